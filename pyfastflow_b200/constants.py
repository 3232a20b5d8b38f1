"""Grid and hydrodynamic parameters, mirroring ``pyfastflow.constants``.

Same names and defaults as pyfastflow/constants.py:20-103.  The reference bakes
these into each Taichi kernel at JIT time; here every kernel takes them as
runtime arguments, read from this module when a kernel-level function is
called (FlowRouter and Flooder hold their own copies).
"""
from __future__ import annotations

import numpy as np

INITIALISED = False

DX = 1.0          # cell size (constants.py:28)
NX = 512          # columns (:31)
NY = 512          # rows (:34)
RAND_RCV = False  # stochastic receivers (:37)
RAND_SEED = 0  # base seed of the stochastic receivers' counter-based draws (no reference counterpart)

# 0 normal (all edges outlets), 1 periodic east-west, 2 periodic north-south,
# 3 custom per-cell codes: 0 nodata, 1 normal, 3 outlet, 7 inlet, 9 periodic (:39-50)
BOUND_MODE = 0

boundaries = None  # torch.uint8 CUDA tensor of N codes in custom mode (:53)

PREC = 10 * 1e-3 / 3600  # precipitation rate, m/s (:94)
MANNING = 0.033          # Manning roughness (:97)
EDGESW = 1e-2            # slope used for cells draining out of the domain (:100)
DT_HYDRO = 5e-3          # explicit time step, s (:103)

BOUND_MODES = {"normal": 0, "periodic_EW": 1, "periodic_NS": 2, "custom": 3}


def init_custom_boundaries(tboundaries: np.ndarray):
    """Upload per-cell boundary codes (uint8, NX*NY) and switch to custom mode
    (constants.py:56-83)."""
    import torch

    global boundaries, BOUND_MODE
    arr = np.ascontiguousarray(np.asarray(tboundaries, dtype=np.uint8).ravel())
    boundaries = torch.from_numpy(arr.copy()).to("cuda")
    BOUND_MODE = 3
    return boundaries
