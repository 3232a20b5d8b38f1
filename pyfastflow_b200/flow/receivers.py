"""Steepest-descent receivers, mirroring pyfastflow/flow/receivers.py."""
from .. import constants as cte
from .. import _dev, _lib


def _codes_ptr():
    if cte.BOUND_MODE == 3:
        if cte.boundaries is None:
            raise RuntimeError("custom boundary mode needs constants.init_custom_boundaries()")
        return _dev.ptr(cte.boundaries, "u8", cte.NX * cte.NY, "boundaries")
    return None


def compute_receivers(z, receivers, gradient):
    """D4 steepest-descent receivers and gradients (receivers.py:15-58), grid from
    ``constants`` (NX, NY, DX, BOUND_MODE, boundaries)."""
    if cte.RAND_RCV:
        raise NotImplementedError("stochastic receivers are not supported")
    N = cte.NX * cte.NY
    _lib.call("pff_compute_receivers", _dev.ptr(z, "f32", N, "z"), _dev.ptr(receivers, "i32", N, "receivers"),
              _dev.ptr(gradient, "f32", N, "gradient"), cte.NX, cte.NY, float(cte.DX), cte.BOUND_MODE,
              _codes_ptr(), _dev.stream())
