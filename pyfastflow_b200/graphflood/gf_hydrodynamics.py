"""GraphFlood kernels, mirroring pyfastflow/graphflood/gf_hydrodynamics.py."""
from __future__ import annotations

import numpy as np

from .. import constants as cte
from .. import _dev, _lib
from ..flow.receivers import _codes_ptr

_scratch = _dev.Scratch()


def _f32(x) -> float:
    return float(np.float32(x))


def diffuse_Q_constant_prec(zh, Q, temp, nsweeps: int = 1, workspace=None):
    """MFD discharge diffusion (gf_hydrodynamics.py:23-75): Q_new[j] = PREC*DX^2 +
    sum of slope-weighted Q of the cells draining into j.  ``nsweeps`` repeats the
    sweep on the same zh (the Flooder runs 5).  Contributions are summed in the
    reference's serial order, so the result is deterministic."""
    n = cte.NX * cte.NY
    ws = workspace or _scratch
    wp, wn = ws.get(_lib.load().pff_diffuse_workspace_bytes(n), device=Q.device)
    _lib.call("pff_diffuse_q", _dev.ptr(zh, "f32", n, "zh"), _dev.ptr(Q, "f32", n, "Q"),
              _dev.ptr(temp, "f32", n, "temp"), int(nsweeps), cte.NX, cte.NY, _f32(cte.DX),
              _f32(cte.PREC * cte.DX * cte.DX), cte.BOUND_MODE, _codes_ptr(), wp, wn, _dev.stream())


def graphflood_core_cte_mannings(h, zh, dh, rec, Q, h_ref=None, dhmax=None):
    """Manning outflow and explicit depth update (gf_hydrodynamics.py:78-129),
    reproduced as written: h receives the depth change twice, zh once."""
    n = h.numel()
    _lib.call("pff_graphflood_core", _dev.ptr(h, "f32", n, "h"), _dev.ptr(zh, "f32", n, "zh"),
              _dev.ptr(dh, "f32", n, "dh"), _dev.ptr(rec, "i32", n, "rec"), _dev.ptr(Q, "f32", n, "Q"), n,
              _f32(cte.DX), _f32(cte.DX ** 2), _f32(cte.MANNING), _f32(cte.EDGESW), _f32(cte.DT_HYDRO),
              _dev.ptr(h_ref, "f32", n, "h_ref") if h_ref is not None else None,
              _dev.ptr(dhmax, "f32", 1, "dhmax") if dhmax is not None else None, _dev.stream())
