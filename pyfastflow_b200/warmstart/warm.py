"""Warm start for GraphFlood: features, training data from the plain solver,
training, and the warm-started state.

The warm state.  GraphFlood's state is (zh, h, Q): the water surface, the depth
and the discharge.  The reference's update adds the Manning change to h twice
and to zh once (gf_hydrodynamics.py:127-129), and its fill adds every
depression's volume to h in the first iteration (fill_topo.py:94-97), so a cold
run starts with all lakes full and spends tens of thousands of iterations
draining that water.  A warm start therefore runs ONE plain iteration (which
fills the surface zh and starts Q), computes the features on that filled
surface, and replaces h by the network's prediction.  Setting zh = z + h0
instead would let the next fill pour the lake volumes back in.

Training data: tiles from the seeded spectral generator with per-tile rainfall
P ~ U(5e-6, 5e-5) m/s and Manning n ~ U(0.02, 0.06); the target is the depth
the plain iteration (all tiles at once, RaggedFlooder) reaches from h = 0 after
a fixed number of iterations, as log(h + 1e-3), weighted by 1 + h / 5 cm so
that wet cells dominate.  The network sees the features of pff_unet_features
(elevation, slope, drainage area, rainfall, n and the kinematic-wave depth they
imply) computed on the filled surface, and predicts log(h0 + 1e-3).
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


def _surface_features(rr, P, n, dx):
    """Route the router's current surface (one launch; the flooder's Q is kept) and
    build the network inputs."""
    Qs = rr.Q.clone()
    rr.seed_constant(1.0, area=False)
    rr.route()
    x = features(rr.z, rr.gradient, rr.counts, P, n, dx, rr.ntiles, int(rr.ny[0]) * int(rr.nx[0]))
    rr.Q.copy_(Qs)
    return x


def make_dataset(ntiles=512, side=128, niter=30000, seed=10, dx=10.0, log=None):
    """Inputs, log-depth targets and loss weights of the tiles whose run stayed
    finite, the targets from `niter` plain GraphFlood iterations from h = 0 with
    the features taken after the first (the warm start's state)."""
    tiles, P, n = scenario_tiles(ntiles, side, seed, dx)
    rr = RaggedRouter([t.shape for t in tiles], dx, "normal")
    rr.set_z(tiles)
    fl = RaggedFlooder(rr, precipitation_rates=P, manning=n)
    rr.Q.zero_()
    fl.run(1, stop=None)
    x = _surface_features(rr, P, n, dx)
    fl.run(niter - 1, stop=None)
    N = side * side
    h = fl.h.view(ntiles, N)
    ok = ~torch.isnan(h).any(1)
    keep = torch.nonzero(ok).flatten()
    tgt = torch.empty(rr.total, dtype=torch.float32, device=rr.device)
    _lib.call("pff_unet_target", fl.h.data_ptr(), tgt.data_ptr(), rr.total, EPS, _dev.stream())
    xk = x.view(ntiles, N * 8)[keep].reshape(-1).contiguous()
    tk = tgt.view(ntiles, N)[keep].reshape(-1).contiguous()
    wk = (1.0 + h[keep].reshape(-1).clamp_min(0) / 0.05).contiguous()
    if log:
        log(f"dataset: {int(ok.sum())}/{ntiles} tiles kept (the others went NaN in the plain run)")
    return xk, tk, wk


def train(net: UNet, x, tgt, side, weight=None, epochs=100, batch=16, lr=2e-3, seed=0, log=None):
    """Minibatch Adam (cosine learning rate) on (x, target[, weight]) tiles of
    side x side; returns the loss history."""
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
            wb = weight.view(ntiles, N)[idx].reshape(-1).contiguous() if weight is not None else None
            net.forward(xb, batch, side, side, check=False)  # backward() checks the whole step
            loss, dp = net.loss_grad(tb, wb)
            net.backward(dp)
            cur_lr = lr * 0.5 * (1 + np.cos(np.pi * (ep * ntiles + s) / (epochs * ntiles)))
            net.adam_step(lr=cur_lr)
            tot += loss
            nb += 1
        hist.append(float(tot) / max(nb, 1))
        if log and (ep % 10 == 0 or ep == epochs - 1):
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


def warm_start_batch(fl: RaggedFlooder, net: UNet, mode="net"):
    """Warm state for every tile of a RaggedFlooder (equal square tiles): one plain
    iteration, features on the filled surface, then h = the prediction ("net") or
    the kinematic-wave depth of the features ("kinematic", no network)."""
    rr = fl.router
    fl.run(1, stop=None)
    x = _surface_features(rr, fl.P, fl.n, rr.dx[0])
    H, W = int(rr.ny[0]), int(rr.nx[0])
    if mode == "net":
        h0 = predict_h0(net, x, rr.ntiles, H, W)
    else:
        h0 = kinematic_h0(x)
    fl.h.copy_(h0)
    return h0


def kinematic_h0(x):
    """The kinematic-wave depth carried in feature channel 5 (the method without
    the network)."""
    f5 = x.view(-1, 8)[:, 5].float()
    return (torch.exp(3.0 * f5) - EPS).clamp_min(0)


def warm_start_flooder(fl, net: UNet):
    """Warm state for a single-grid Flooder: one plain iteration, route the filled
    surface (the flooder's Q is kept), features, h = the prediction."""
    r = fl.router
    fl.iteration()
    Qs = r.Q.clone()
    r.compute_receivers()
    r.reroute_flow()
    r.accumulate_constant_Q(1.0, area=False)
    x = features(r.z, r.gradient, r.counts, fl.precipitation_rates, fl.manning, r.dx, 1, r.N)
    r.Q.copy_(Qs)
    h0 = predict_h0(net, x, 1, r.ny, r.nx)
    fl.h.copy_(h0)
    return h0
