"""4-level U-Net (3x3 convolutions, 32 -> 256 channels, ReLU, BF16 weights and
activations, FP32 accumulation and FP32 master weights) with an explicit
backward pass, every op a libpff kernel (csrc/pff_conv.cu).

Layout: NHWC, B tiles of H x W (H, W multiples of 8).  Encoder outputs are
written straight into the channel slice of the decoder's concatenation buffer
([upsampled decoder features | skip]), so no copy is needed for the skips.

    enc0  8 -> 32 -> 32        (H)      dec0  96 -> 32 -> 32    head 32 -> 8 (channel 0 = log h)
    enc1  32 -> 64 -> 64       (H/2)    dec1  192 -> 64 -> 64
    enc2  64 -> 128 -> 128     (H/4)    dec2  384 -> 128 -> 128
    bott  128 -> 256 -> 256    (H/8)
Downsampling is 2x2 mean pooling, upsampling nearest 2x.
"""
from __future__ import annotations

import numpy as np
import torch

from .. import _dev, _lib

# name, input buffer, input channel offset, output buffer, output offset, Cin, Cout, relu, level
LAYERS = [
    ("enc0a", "x", 0, "a0", 0, 8, 32, 1, 0),
    ("enc0b", "a0", 0, "cat0", 64, 32, 32, 1, 0),
    ("enc1a", "p0", 0, "a1", 0, 32, 64, 1, 1),
    ("enc1b", "a1", 0, "cat1", 128, 64, 64, 1, 1),
    ("enc2a", "p1", 0, "a2", 0, 64, 128, 1, 2),
    ("enc2b", "a2", 0, "cat2", 256, 128, 128, 1, 2),
    ("bota", "p2", 0, "a3", 0, 128, 256, 1, 3),
    ("botb", "a3", 0, "e3", 0, 256, 256, 1, 3),
    ("dec2a", "cat2", 0, "g2", 0, 384, 128, 1, 2),
    ("dec2b", "g2", 0, "d2", 0, 128, 128, 1, 2),
    ("dec1a", "cat1", 0, "g1", 0, 192, 64, 1, 1),
    ("dec1b", "g1", 0, "d1", 0, 64, 64, 1, 1),
    ("dec0a", "cat0", 0, "g0", 0, 96, 32, 1, 0),
    ("dec0b", "g0", 0, "d0", 0, 32, 32, 1, 0),
    ("head", "d0", 0, "pred", 0, 32, 8, 0, 0),
]
# buffer -> (channels, level)
BUFFERS = {"x": (8, 0), "a0": (32, 0), "cat0": (96, 0), "p0": (32, 1), "a1": (64, 1), "cat1": (192, 1),
           "p1": (64, 2), "a2": (128, 2), "cat2": (384, 2), "p2": (128, 3), "a3": (256, 3), "e3": (256, 3),
           "g2": (128, 2), "d2": (128, 2), "g1": (64, 1), "d1": (64, 1), "g0": (32, 0), "d0": (32, 0),
           "pred": (8, 0)}


def _call(name, *a):
    _lib.call(name, *a)


def check_tensor_core_status():
    """Raise PFFError if a tcgen05 convolution gave up waiting on its pipeline since
    the last check (its outputs are then unspecified).  Synchronizes the device."""
    import ctypes as C

    flag = C.c_int()
    _lib.call("pff_conv_tc_status", C.byref(flag))
    if flag.value:
        raise _lib.PFFError("a tcgen05 convolution timed out waiting on its TMA/MMA pipeline; "
                            "its outputs are unspecified")


class UNet:
    def __init__(self, seed: int = 0, device="cuda"):
        self.device = torch.device(device)
        self.layers = {}
        off = 0
        for L in LAYERS:
            name, _, _, _, _, cin, cout, _, _ = L
            nw = cout * 9 * cin
            self.layers[name] = (off, nw, off + nw, cout)  # weight offset, size, bias offset, Cout
            off += nw + cout
        self.nparams = off
        rng = np.random.default_rng(seed)
        p = np.zeros(off, np.float32)
        for name, _, _, _, _, cin, cout, _, _ in LAYERS:
            wo, nw, bo, _ = self.layers[name]
            std = np.sqrt(2.0 / (9 * cin)) if name != "head" else 1e-3
            p[wo:wo + nw] = rng.standard_normal(nw) * std
        self.p = torch.from_numpy(p).to(self.device)          # f32 master
        self.pb = torch.zeros(off, dtype=torch.bfloat16, device=self.device)  # bf16 copy (weights used)
        self.g = torch.zeros(off, dtype=torch.float32, device=self.device)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.step_count = 0
        self.wt = {}  # flipped weights for the data gradients
        for name, _, _, _, _, cin, cout, _, _ in LAYERS:
            self.wt[name] = torch.zeros(9 * cin * cout, dtype=torch.bfloat16, device=self.device)
        self._sync_bf16()
        self._shape = None
        self.buf = {}
        self.grad = {}

    # ---- parameters -------------------------------------------------------------------
    def _sync_bf16(self):
        _call("pff_f32_to_bf16", self.p.data_ptr(), self.pb.data_ptr(), self.nparams, _dev.stream())
        self._flip()

    def _flip(self):
        st = _dev.stream()
        for name, _, _, _, _, cin, cout, _, _ in LAYERS:
            wo = self.layers[name][0]
            _call("pff_conv3x3_wflip", self.pb.data_ptr() + 2 * wo, self.wt[name].data_ptr(), cin, cout, st)

    def set_head_bias(self, value: float):
        bo = self.layers["head"][2]
        self.p[bo:bo + 8] = value
        self._sync_bf16()

    def state_dict(self):
        return {"p": self.p.cpu().numpy().copy(), "step": self.step_count}

    def load_state_dict(self, sd):
        self.p.copy_(torch.from_numpy(np.asarray(sd["p"], np.float32)))
        self.step_count = int(sd.get("step", 0))
        self._sync_bf16()

    # ---- buffers ----------------------------------------------------------------------
    def _alloc(self, B, H, W):
        if self._shape == (B, H, W):
            return
        if H % 8 or W % 8:
            raise ValueError(f"U-Net tiles need H, W multiples of 8 (got {H} x {W})")
        self._shape = (B, H, W)
        self.buf, self.grad = {}, {}
        for name, (c, lev) in BUFFERS.items():
            n = B * (H >> lev) * (W >> lev) * c
            dt = torch.float32 if name == "pred" else torch.bfloat16
            self.buf[name] = torch.zeros(n, dtype=dt, device=self.device)
            if name != "x":
                self.grad[name] = torch.zeros(n, dtype=torch.bfloat16, device=self.device)

    def _dims(self, lev):
        B, H, W = self._shape
        return B, H >> lev, W >> lev

    # ---- forward ----------------------------------------------------------------------
    def forward(self, x: torch.Tensor, B: int, H: int, W: int, check: bool = True) -> torch.Tensor:
        """x: bf16 NHWC rows of 8 channels, B*H*W rows.  Returns pred (f32 rows of 8,
        channel 0 = predicted log depth).  check: read the tensor-core error flag at
        the end and raise if a convolution timed out (one device synchronisation;
        pass False inside a training step whose backward() checks)."""
        self._alloc(B, H, W)
        st = _dev.stream()
        bf = self.buf
        bf["x"].copy_(x.reshape(-1))

        def conv(L):
            name, src, so, dst, do, cin, cout, relu, lev = L
            wo, _, bo, _ = self.layers[name]
            b, h, w = self._dims(lev)
            _call("pff_conv3x3_fwd", bf[src].data_ptr(), BUFFERS[src][0], so, self.pb.data_ptr() + 2 * wo,
                  self.p.data_ptr() + 4 * bo, bf[dst].data_ptr(), BUFFERS[dst][0], do, b, h, w, cin, cout, relu,
                  1 if dst == "pred" else 0, st)

        def pool(src, so, c, dst, lev):  # lev: the fine level
            b, h, w = self._dims(lev)
            _call("pff_avgpool2", bf[src].data_ptr(), BUFFERS[src][0], so, bf[dst].data_ptr(), BUFFERS[dst][0], 0,
                  b, h, w, c, st)

        def up(src, c, dst, lev):  # lev: the coarse level
            b, h, w = self._dims(lev)
            _call("pff_upsample2", bf[src].data_ptr(), BUFFERS[src][0], 0, bf[dst].data_ptr(), BUFFERS[dst][0], 0,
                  b, h, w, c, st)

        Ls = {L[0]: L for L in LAYERS}
        conv(Ls["enc0a"]); conv(Ls["enc0b"]); pool("cat0", 64, 32, "p0", 0)
        conv(Ls["enc1a"]); conv(Ls["enc1b"]); pool("cat1", 128, 64, "p1", 1)
        conv(Ls["enc2a"]); conv(Ls["enc2b"]); pool("cat2", 256, 128, "p2", 2)
        conv(Ls["bota"]); conv(Ls["botb"]); up("e3", 256, "cat2", 3)
        conv(Ls["dec2a"]); conv(Ls["dec2b"]); up("d2", 128, "cat1", 2)
        conv(Ls["dec1a"]); conv(Ls["dec1b"]); up("d1", 64, "cat0", 1)
        conv(Ls["dec0a"]); conv(Ls["dec0b"]); conv(Ls["head"])
        if check:
            check_tensor_core_status()
        return bf["pred"]

    # ---- backward ---------------------------------------------------------------------
    def backward(self, dpred: torch.Tensor, check: bool = True):
        """dpred: bf16 rows of 8 (gradient of the loss w.r.t. pred).  Accumulates the
        parameter gradients into self.g (zeroed here first).  check: as in forward();
        it covers every convolution since the last check, the forward pass's too."""
        st = _dev.stream()
        bf, gr = self.buf, self.grad
        self.g.zero_()
        gr["pred"].copy_(dpred.reshape(-1))

        def conv_bwd(name, dsrc, dso, need_dx=True):
            L = next(l for l in LAYERS if l[0] == name)
            _, src, so, dst, do, cin, cout, relu, lev = L
            wo, _, bo, _ = self.layers[name]
            b, h, w = self._dims(lev)
            P = b * h * w
            cd = BUFFERS[dst][0]
            if relu:
                _call("pff_relu_bwd", gr[dst].data_ptr(), cd, do, bf[dst].data_ptr(), cd, do, P, cout, st)
            _call("pff_conv3x3_wgrad", bf[src].data_ptr(), BUFFERS[src][0], so, gr[dst].data_ptr(), cd, do,
                  self.g.data_ptr() + 4 * wo, b, h, w, cin, cout, st)
            _call("pff_bias_grad", gr[dst].data_ptr(), cd, do, self.g.data_ptr() + 4 * bo, P, cout, st)
            if need_dx:
                _call("pff_conv3x3_fwd", gr[dst].data_ptr(), cd, do, self.wt[name].data_ptr(), None,
                      gr[dsrc].data_ptr(), BUFFERS[dsrc][0], dso, b, h, w, cout, cin, 0, 0, st)

        def up_bwd(dcat, c, dst, lev):  # lev: coarse level; the upsampled part is channels [0, c)
            b, h, w = self._dims(lev)
            _call("pff_upsample2_bwd", gr[dcat].data_ptr(), BUFFERS[dcat][0], 0, gr[dst].data_ptr(),
                  BUFFERS[dst][0], 0, b, h, w, c, st)

        def pool_bwd(dsrc, dcat, off, c, lev):  # lev: fine level; adds into the skip slice
            b, h, w = self._dims(lev)
            _call("pff_avgpool2_bwd", gr[dsrc].data_ptr(), BUFFERS[dsrc][0], 0, gr[dcat].data_ptr(),
                  BUFFERS[dcat][0], off, b, h, w, c, 1, st)

        conv_bwd("head", "d0", 0)
        conv_bwd("dec0b", "g0", 0)
        conv_bwd("dec0a", "cat0", 0)
        up_bwd("cat0", 64, "d1", 1)
        conv_bwd("dec1b", "g1", 0)
        conv_bwd("dec1a", "cat1", 0)
        up_bwd("cat1", 128, "d2", 2)
        conv_bwd("dec2b", "g2", 0)
        conv_bwd("dec2a", "cat2", 0)
        up_bwd("cat2", 256, "e3", 3)
        conv_bwd("botb", "a3", 0)
        conv_bwd("bota", "p2", 0)
        pool_bwd("p2", "cat2", 256, 128, 2)
        conv_bwd("enc2b", "a2", 0)
        conv_bwd("enc2a", "p1", 0)
        pool_bwd("p1", "cat1", 128, 64, 1)
        conv_bwd("enc1b", "a1", 0)
        conv_bwd("enc1a", "p0", 0)
        pool_bwd("p0", "cat0", 64, 32, 0)
        conv_bwd("enc0b", "a0", 0)
        conv_bwd("enc0a", None, 0, need_dx=False)
        if check:
            check_tensor_core_status()

    def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, weight_decay=0.0):
        self.step_count += 1
        _call("pff_adam", self.p.data_ptr(), self.g.data_ptr(), self.m.data_ptr(), self.v.data_ptr(),
              self.pb.data_ptr(), self.nparams, lr, b1, b2, eps, self.step_count, weight_decay, _dev.stream())
        self._flip()

    # ---- loss -------------------------------------------------------------------------
    def loss_grad(self, target: torch.Tensor, weight: torch.Tensor | None = None) -> torch.Tensor:
        """Weighted MSE of pred channel 0 against target (f32, one per pixel), averaged
        over the weights; leaves d loss / d pred in the gradient buffer, returns the
        loss as a device scalar."""
        P = target.numel()
        wsum = float(weight.sum()) if weight is not None else float(P)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        dp = torch.empty(P * 8, dtype=torch.bfloat16, device=self.device)
        _call("pff_mse_loss", self.buf["pred"].data_ptr(), 8, target.data_ptr(),
              weight.data_ptr() if weight is not None else None, P, dp.data_ptr(), 8, 1.0 / wsum, loss.data_ptr(),
              _dev.stream())
        return loss, dp
