"""The allocation-free fill entry point, through the C ABI.

pff_fill_z_add_delta_noalloc serves callers that cannot allocate device memory:
its scratch is a device array built into the library instead of a caller
workspace.  It must give exactly what pff_fill_z_add_delta gives, call after
call (the shared array keeps the previous call's contents), and refuse grids
larger than its built-in scratch.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from pyfastflow_b200 import synthetic

pytestmark = pytest.mark.gpu


def _case(orc, n, seed):
    rng = np.random.default_rng(seed)
    z = synthetic.spectral_dem(n, n, seed, relief=40.0, npits=15, pit_scale=0.2)
    h = (rng.random(n * n) * 0.3).astype(np.float32)
    zh = (z.ravel() + h).astype(np.float32)
    og = orc.Grid(n, n, 0)
    rcv, _ = orc.compute_receivers(zh, og, 10.0)
    rcv, _, _, _, _ = orc.reroute_flow(rcv, zh, og)
    return zh, h, rcv


def _run(torch, lib, zh, h, rcv, noalloc):
    from pyfastflow_b200 import _dev

    N = zh.size
    zd = torch.from_numpy(zh.copy()).cuda()
    hd = torch.from_numpy(h.copy()).cuda()
    z_ = torch.empty_like(zd)
    r = torch.from_numpy(rcv).cuda()
    r_ = torch.empty_like(r)
    r__ = torch.empty_like(r)
    st = _dev.stream()
    if noalloc:
        rc = lib.pff_fill_z_add_delta_noalloc(zd.data_ptr(), hd.data_ptr(), z_.data_ptr(), r.data_ptr(),
                                              r_.data_ptr(), r__.data_ptr(), 1e-3, N, st)
    else:
        ws = torch.empty(lib.pff_fill_workspace_bytes(N), dtype=torch.uint8, device="cuda")
        rc = lib.pff_fill_z_add_delta(zd.data_ptr(), hd.data_ptr(), z_.data_ptr(), r.data_ptr(), r_.data_ptr(),
                                      r__.data_ptr(), 1e-3, N, ws.data_ptr(), ws.numel(), st)
    assert rc == 0, lib.pff_last_error_string()
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in (zd, hd, z_, r_, r__)]


def test_noalloc_fill_matches_workspace_fill_twice(orc, cuda):
    torch = cuda
    from pyfastflow_b200 import _lib

    lib = _lib.load()
    _lib._sync_device()
    for n, seed in ((200, 1), (131, 2)):  # two calls in a row, different sizes and data
        zh, h, rcv = _case(orc, n, seed)
        ref = _run(torch, lib, zh, h, rcv, noalloc=False)
        got = _run(torch, lib, zh, h, rcv, noalloc=True)
        for a, b in zip(ref, got):
            # the fill is deterministic: same IEEE operations in the same order
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
        # and both equal the CPU oracle's fill (fill_topo.py:99-125, snapshot rounds) bit for bit
        oz, oh, oz_ = orc.fill_z_add_delta(zh.copy(), h.copy(), rcv, 1e-3)
        for want, have in ((oz, got[0]), (oh, got[1]), (oz_, got[2])):
            assert np.array_equal(want.view(np.uint32), have.view(np.uint32))
        # receivers_ after the rounds: the pointers jumped ceil(log2 N) times
        jumped = rcv.copy()
        for _ in range(orc.ceil_log2(rcv.size)):
            jumped = jumped[jumped]
        assert np.array_equal(got[3], jumped)


def test_noalloc_fill_rejects_oversize_grid(cuda):
    torch = cuda
    from pyfastflow_b200 import _lib

    lib = _lib.load()
    _lib._sync_device()
    t = torch.zeros(16, device="cuda")
    ti = torch.zeros(16, dtype=torch.int32, device="cuda")
    too_big = (1 << 22) + 1
    rc = lib.pff_fill_z_add_delta_noalloc(t.data_ptr(), t.data_ptr(), t.data_ptr(), ti.data_ptr(), ti.data_ptr(),
                                          ti.data_ptr(), 1e-3, too_big, C.c_void_p(0))
    assert rc == 1
    assert b"exceed" in lib.pff_last_error_string()
