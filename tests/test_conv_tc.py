"""The tcgen05 (TMEM accumulator, TMA operands) 3x3 convolution against the
mma.sync kernel and against PyTorch CPU f32 on the same bf16 operands: several
pixel-block shapes (W >= 128, 64, 32, 16), 64- and 128-wide output tiles, channel
slices, bias, ReLU, f32 and bf16 outputs."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
F = torch.nn.functional


def _bf(t):
    return t.to(torch.bfloat16).to(torch.float32)


def _nhwc(t):
    return t.permute(0, 2, 3, 1).contiguous().reshape(-1)


def _nchw(flat, B, H, W, C_):
    return flat.reshape(B, H, W, C_).permute(0, 3, 1, 2)


def _w_ours(w):
    return w.permute(0, 2, 3, 1).contiguous().reshape(-1)


def test_conv_path_switch_host_checks():
    from pyfastflow_b200 import _lib

    lib = _lib.load()
    assert lib.pff_conv_set_path(3) != 0
    assert lib.pff_conv_set_path(1) == 0
    assert lib.pff_conv_set_path(0) == 0  # back to the default


@pytest.mark.gpu
@pytest.mark.parametrize("B,H,W,Cin,Cout,cs_in,off_in,relu,f32", [
    (2, 16, 16, 64, 64, 64, 0, 1, 0),
    (1, 8, 256, 64, 128, 64, 0, 0, 1),
    (2, 32, 64, 128, 128, 192, 64, 1, 0),
    (1, 16, 32, 192, 64, 192, 0, 0, 1),
    (3, 24, 16, 64, 256, 128, 64, 1, 0),
])
def test_tcgen05_conv_matches(cuda, B, H, W, Cin, Cout, cs_in, off_in, relu, f32):
    from pyfastflow_b200 import _dev, _lib

    lib = _lib.load()
    g = torch.Generator().manual_seed(H * W + Cin + Cout)
    xw = _bf(torch.randn(B, cs_in, H, W, generator=g))
    w = _bf(torch.randn(Cout, Cin, 3, 3, generator=g) * 0.1)
    b = torch.randn(Cout, generator=g)
    ref = F.conv2d(xw[:, off_in:off_in + Cin], w, b, padding=1)
    if relu:
        ref = ref.clamp_min(0)
    xd = _nhwc(xw).to(torch.bfloat16).cuda()
    wd = _w_ours(w).to(torch.bfloat16).cuda()
    bd = b.cuda()
    dt = torch.float32 if f32 else torch.bfloat16
    outs = {}
    try:
        for path in (1, 2):
            assert lib.pff_conv_set_path(path) == 0
            y = torch.zeros(B * H * W * Cout, dtype=dt, device="cuda")
            _lib.call("pff_conv3x3_fwd", xd.data_ptr(), cs_in, off_in, wd.data_ptr(), bd.data_ptr(), y.data_ptr(),
                      Cout, 0, B, H, W, Cin, Cout, relu, f32, _dev.stream())
            torch.cuda.synchronize()
            outs[path] = _nchw(y.float().cpu(), B, H, W, Cout)
        flag = C.c_int(-1)
        _lib.call("pff_conv_tc_status", C.byref(flag))
        assert flag.value == 0, "a tcgen05 pipeline wait gave up"
    finally:
        lib.pff_conv_set_path(0)
    tol = 2e-5 * np.sqrt(9 * Cin) + 1e-5 if f32 else 1e-2
    scale = float(ref.abs().max())
    assert float((outs[2] - ref).abs().max()) / scale < tol
    assert float((outs[2] - outs[1]).abs().max()) / scale < tol


@pytest.mark.gpu
def test_tcgen05_rejects_unsupported(cuda):
    from pyfastflow_b200 import _dev, _lib

    lib = _lib.load()
    x = torch.zeros(2 * 8 * 8 * 32, dtype=torch.bfloat16, device="cuda")
    w = torch.zeros(64 * 9 * 32, dtype=torch.bfloat16, device="cuda")
    y = torch.zeros(2 * 8 * 8 * 64, dtype=torch.bfloat16, device="cuda")
    try:
        lib.pff_conv_set_path(2)
        rc = lib.pff_conv3x3_fwd(x.data_ptr(), 32, 0, w.data_ptr(), None, y.data_ptr(), 64, 0, 2, 8, 8, 32, 64, 0, 0,
                                 _dev.stream())
        assert rc != 0  # Cin = 32 is not a multiple of 64
    finally:
        lib.pff_conv_set_path(0)
