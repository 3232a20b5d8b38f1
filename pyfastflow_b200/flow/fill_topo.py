"""Topographic fill with delta, mirroring pyfastflow/flow/fill_topo.py:99-125."""
from .. import constants as cte
from .. import _dev, _lib

_scratch = _dev.Scratch()


def fill_z_add_delta(zh, h, z_, receivers, receivers_, receivers__, epsilon=1e-4, workspace=None):
    """ceil(log2 N) pointer-jumping fill rounds on zh, then h += z_ - zh, zh = z_.
    The reference's in-place read of z_ inside a round is a race; it is pinned
    here to snapshot semantics (every read sees the start-of-round value)."""
    n = zh.numel()
    ws = workspace or _scratch
    wp, wn = ws.get(_lib.load().pff_fill_workspace_bytes(n), device=zh.device)
    _lib.call("pff_fill_z_add_delta", _dev.ptr(zh, "f32", n, "zh"), _dev.ptr(h, "f32", n, "h"),
              _dev.ptr(z_, "f32", n, "z_"), _dev.ptr(receivers, "i32", n, "receivers"),
              _dev.ptr(receivers_, "i32", n, "receivers_"), _dev.ptr(receivers__, "i32", n, "receivers__"),
              float(epsilon), n, wp, wn, _dev.stream())
