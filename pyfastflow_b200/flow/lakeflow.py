"""Lake / depression rerouting, mirroring pyfastflow/flow/lakeflow.py.

Basin arrays (basin_saddle, outlet: int64; basin_saddlenode: int32) hold N+1
entries: basin ids run 1..N (cell + 1), and id N exists in custom mode when the
last cell is interior (the reference's N-sized arrays overflow there).
is_border / tag / tag_ are uint8 (or bool) tensors."""
from __future__ import annotations

import ctypes as C

from .. import constants as cte
from .. import _dev, _lib
from .receivers import _codes_ptr


def _grid():
    return cte.NX, cte.NY, cte.BOUND_MODE, _codes_ptr()


def depression_counter(rec) -> int:
    """Number of interior self-receivers (lakeflow.py:25-44)."""
    nx, ny, mode, codes = _grid()
    out = C.c_int()
    _lib.call("pff_depression_counter", _dev.ptr(rec, "i32", nx * ny, "rec"), nx, ny, mode, codes,
              C.byref(out), _dev.stream())
    return out.value


def basin_identification(bid, rec, rec_, N=None):
    """Basin labels by pointer jumping (lakeflow.py:82-101): bid = root+1, or 0
    if the root can leave the domain.  rec_ is scratch."""
    nx, ny, mode, codes = _grid()
    n = nx * ny
    _lib.call("pff_basin_identification", _dev.ptr(bid, "i32", n, "bid"), _dev.ptr(rec, "i32", n, "rec"),
              _dev.ptr(rec_, "i32", n, "rec_"), nx, ny, mode, codes, _dev.stream())


def saddlesort(bid, is_border, z_prime, basin_saddle, basin_saddlenode, outlet, z):
    """Basin saddles and outlets, passes 1-5 (lakeflow.py:106-281)."""
    nx, ny, mode, codes = _grid()
    n = nx * ny
    _lib.call("pff_saddlesort", _dev.ptr(bid, "i32", n, "bid"), _dev.ptr(is_border, "u8", n, "is_border"),
              _dev.ptr(z_prime, "f32", n, "z_prime"), _dev.ptr(basin_saddle, "i64", n + 1, "basin_saddle"),
              _dev.ptr(basin_saddlenode, "i32", n + 1, "basin_saddlenode"), _dev.ptr(outlet, "i64", n + 1, "outlet"),
              _dev.ptr(z, "f32", n, "z"), nx, ny, mode, codes, _dev.stream())


_scratch = _dev.Scratch()


def reroute_flow(bid, rec, rec_, rec__, z, z_prime, is_border, outlet, basin_saddle, basin_saddlenode, tag, tag_,
                 change=None, carve=True, workspace: _dev.Scratch | None = None) -> int:
    """Depression rerouting (lakeflow.py:466-538).  carve=True reroutes ``rec`` in
    place; carve=False leaves the result in ``rec_`` as the reference does.
    Returns the number of outer iterations run.  ``change`` is accepted for
    signature compatibility (convergence flags live on the device)."""
    nx, ny, mode, codes = _grid()
    n = nx * ny
    ws = workspace or _scratch
    wp, wn = ws.get(_lib.load().pff_reroute_workspace_bytes(n), device=rec.device)
    nout = C.c_int()
    _lib.call("pff_reroute_flow", _dev.ptr(bid, "i32", n, "bid"), _dev.ptr(rec, "i32", n, "rec"),
              _dev.ptr(rec_, "i32", n, "rec_"), _dev.ptr(rec__, "i32", n, "rec__"), _dev.ptr(z, "f32", n, "z"),
              _dev.ptr(z_prime, "f32", n, "z_prime"), _dev.ptr(is_border, "u8", n, "is_border"),
              _dev.ptr(outlet, "i64", n + 1, "outlet"), _dev.ptr(basin_saddle, "i64", n + 1, "basin_saddle"),
              _dev.ptr(basin_saddlenode, "i32", n + 1, "basin_saddlenode"), _dev.ptr(tag, "u8", n, "tag"),
              _dev.ptr(tag_, "u8", n, "tag_"), int(bool(carve)), nx, ny, mode, codes, wp, wn, C.byref(nout),
              _dev.stream())
    return nout.value
