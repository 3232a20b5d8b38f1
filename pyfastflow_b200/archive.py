"""Legacy downstream tree algorithms of pyfastflow's archive, over torch CUDA tensors.

The reference kept these CUDA-era kernels in archive/fastflow/kernels (with their
drivers in archive/_save_fasftflow/fastflow); they are callers of the same
receiver trees as the hot path:

- tree_accum_downward(rcv, W, p): solves x = p + W * x[rcv] downstream by pointer
  jumping (tree_accum_down.py), e.g. an implicit elevation update;
- tree_max_downward(rcv, p): the largest value on each cell's downstream path, the
  final root's value excluded (tree_max_down.py);
- erode_deposit(...): deposition plus implicit stream-power erosion, whose
  elevation update is a tree_accum_downward solve (erode_deposit.py).

Like the reference's drivers, rcv, W and p are updated in place (rcv ends jumped).
Receivers are int32 cell indices.
"""
from __future__ import annotations

from . import _dev, _lib


def _ws(n):
    return _dev._shared.get(_lib.load().pff_archive_workspace_bytes(n))


def tree_accum_downward(rcv, W, p):
    """In place: p becomes the solution of x = p + W * x[rcv]; returns p."""
    n = p.numel()
    wp, wn = _ws(n)
    _lib.call("pff_tree_accum_down", _dev.ptr(rcv, "i32", n, "rcv"), _dev.ptr(W, "f32", n, "W"),
              _dev.ptr(p, "f32", n, "p"), n, wp, wn, _dev.stream())
    return p


def tree_max_downward(rcv, p):
    """In place: p becomes the largest value on its downstream path (root excluded); returns p."""
    n = p.numel()
    wp, wn = _ws(n)
    _lib.call("pff_tree_max_down", _dev.ptr(rcv, "i32", n, "rcv"), _dev.ptr(p, "f32", n, "p"), n, wp, wn,
              _dev.stream())
    return p


def erode_deposit(z, bound, rcv, drain, Qs, dt, dx, k_spl, k_t, k_h, k_d, m, pe=None, We=None):
    """Deposition on z (in place), then the implicit erosion solve; returns the new
    elevations (pe), as the reference's run_erode_deposit_cuda returns them."""
    import torch

    n = z.numel()
    pe = torch.empty_like(z) if pe is None else pe
    We = torch.empty_like(z) if We is None else We
    wp, wn = _ws(n)
    _lib.call("pff_erode_deposit", _dev.ptr(z, "f32", n, "z"), _dev.ptr(bound, "u8", n, "bound"),
              _dev.ptr(rcv, "i32", n, "rcv"), _dev.ptr(drain, "f32", n, "drain"), _dev.ptr(Qs, "f32", n, "Qs"),
              float(dt), float(dx), float(k_spl), float(k_t), float(k_h), float(k_d), float(m),
              _dev.ptr(pe, "f32", n, "pe"), _dev.ptr(We, "f32", n, "We"), n, wp, wn, _dev.stream())
    return pe
