"""Topographic fills, mirroring pyfastflow/flow/fill_topo.py: topofill (:48-78) and
fill_z_add_delta (:99-125)."""
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


def topofill(flow_field, epsilon=1e-6, custom_z=None):
    """fill_topo.py:48-78: ceil(log2 N) rounds with increments 2^it * epsilon on the
    router's elevation along its receivers.  Without custom_z the router's z is
    replaced by the filled surface (z_ holds it too); with custom_z (a float32 CUDA
    tensor of N cells) the filled surface goes there and z is left as it was.  The
    reference prints each round's increment; this does not."""
    n = flow_field.N
    out = flow_field.z_ if custom_z is None else custom_z
    wp, wn = _scratch.get(_lib.load().pff_fill_workspace_bytes(n), device=flow_field.z.device)
    _lib.call("pff_topofill", _dev.ptr(flow_field.z, "f32", n, "z"), _dev.ptr(out, "f32", n, "z_"),
              _dev.ptr(flow_field.receivers, "i32", n, "receivers"),
              _dev.ptr(flow_field.receivers_, "i32", n, "receivers_"),
              _dev.ptr(flow_field.receivers__, "i32", n, "receivers__"), float(epsilon), n,
              1 if custom_z is None else 0, wp, wn, _dev.stream())
