"""Warm start for GraphFlood: features, training data from the plain solver,
training, and the predicted initial depth.

Training data: tiles from the seeded spectral generator with per-tile rainfall
P ~ U(5e-6, 5e-5) m/s and Manning n ~ U(0.02, 0.06); the target is the depth the
plain GraphFlood iteration (all tiles at once, RaggedFlooder) reaches from h = 0
after a fixed number of iterations, as log(h + 1e-3).  The network sees the
features of pff_unet_features (elevation, slope, drainage area, rainfall, n and
the kinematic-wave depth they imply) and predicts log(h0 + 1e-3).
"""
from __future__ import annotations

import numpy as np
import torch

from .. import _dev, _lib, synthetic
from ..flow.ragged import RaggedRouter
from ..graphflood.ragged import RaggedFlooder
from .unet import UNet

EPS = 1e-3


def features(z: torch.Tensor, slope: torch.Tensor, counts: torch.Tensor, prec, manning, dx: float, B: int, N: int):
    """bf16 NHWC input rows (8 channels) for B tiles of N cells (packed f32 z and
    slope, uint32 counts as int32 bits), per-tile rainfall and Manning n."""
    dev = z.device
    P = torch.as_tensor(np.broadcast_to(np.asarray(prec, np.float32), (B,)).copy(), device=dev)
    n = torch.as_tensor(np.broadcast_to(np.asarray(manning, np.float32), (B,)).copy(), device=dev)
    stats = torch.zeros(2 * B, dtype=torch.float32, device=dev)
    x = torch.zeros(B * N * 8, dtype=torch.bfloat16, device=dev)
    _lib.call("pff_unet_features", z.data_ptr(), slope.data_ptr(), counts.data_ptr(), P.data_ptr(), n.data_ptr(),
              float(dx), B, N, stats.data_ptr(), x.data_ptr(), _dev.stream())
    return x


def scenario_tiles(ntiles, side, seed, dx=10.0):
    """Tiles and parameters of a training or evaluation set."""
    rng = np.random.default_rng(seed)
    tiles, P, n = [], [], []
    for k in range(ntiles):
        relief = float(rng.uniform(50.0, 500.0))
        npits = int(rng.integers(0, 1 + side // 16))
        tiles.append(synthetic.spectral_dem(side, side, seed * 7919 + k, relief=relief, dx=dx, npits=npits,
                                            pit_scale=side / 1024.0))
        P.append(float(rng.uniform(5e-6, 5e-5)))
        n.append(float(rng.uniform(0.02, 0.06)))
    return tiles, np.array(P), np.array(n)


def tile_features(tiles, P, n, dx=10.0):
    """Route every tile (one launch) and build the network inputs; returns
    (router, x)."""
    side_y, side_x = tiles[0].shape
    rr = RaggedRouter([t.shape for t in tiles], dx, "normal")
    rr.set_z(tiles)
    rr.seed_constant(1.0, area=False)
    rr.route()
    x = features(rr.z, rr.gradient, rr.counts, P, n, dx, len(tiles), side_x * side_y)
    return rr, x


def make_dataset(ntiles=256, side=128, niter=2000, seed=10, dx=10.0):
    """(x, target, P, n): inputs and log-depth targets of `ntiles` tiles, the
    targets from `niter` plain GraphFlood iterations from h = 0."""
    tiles, P, n = scenario_tiles(ntiles, side, seed, dx)
    rr, x = tile_features(tiles, P, n, dx)
    fl = RaggedFlooder(rr, precipitation_rates=P, manning=n)
    rr.Q.zero_()
    fl.run(niter, stop=None)
    tgt = torch.empty(rr.total, dtype=torch.float32, device=rr.device)
    _lib.call("pff_unet_target", fl.h.data_ptr(), tgt.data_ptr(), rr.total, EPS, _dev.stream())
    return x, tgt, P, n


def train(net: UNet, x, tgt, side, epochs=20, batch=16, lr=2e-3, seed=0, log=None):
    """Minibatch Adam on (x, target) tiles of side x side; returns the loss history."""
    N = side * side
    ntiles = tgt.numel() // N
    rng = np.random.default_rng(seed)
    hist = []
    for ep in range(epochs):
        order = rng.permutation(ntiles)
        tot = torch.zeros(1, dtype=torch.float32, device=tgt.device)
        nb = 0
        for s in range(0, ntiles - batch + 1, batch):
            idx = torch.as_tensor(order[s:s + batch], device=tgt.device)
            xb = x.view(ntiles, N * 8)[idx].reshape(-1)
            tb = tgt.view(ntiles, N)[idx].reshape(-1)
            net.forward(xb, batch, side, side)
            loss, dp = net.loss_grad(tb)
            net.backward(dp)
            cur_lr = lr * 0.5 * (1 + np.cos(np.pi * (ep * ntiles + s) / (epochs * ntiles)))
            net.adam_step(lr=cur_lr)
            tot += loss
            nb += 1
        hist.append(float(tot) / max(nb, 1))
        if log:
            log(f"epoch {ep} loss {hist[-1]:.4f}")
    return hist


def predict_h0(net: UNet, x, B, H, W, z=None, zh=None):
    """Initial depth (f32, B*H*W) predicted from the input rows x.  With the bed z
    and an output zh (f32, B*H*W), also writes the water surface zh = z + h0, the
    GraphFlood state that goes with that depth."""
    pred = net.forward(x, B, H, W)
    h0 = torch.empty(B * H * W, dtype=torch.float32, device=x.device)
    _lib.call("pff_unet_h0", pred.data_ptr(), 8, h0.data_ptr(), B * H * W, EPS,
              z.data_ptr() if zh is not None else None, zh.data_ptr() if zh is not None else None, _dev.stream())
    return h0
