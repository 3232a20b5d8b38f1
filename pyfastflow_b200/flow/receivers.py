"""Steepest-descent receivers, mirroring pyfastflow/flow/receivers.py."""
from .. import constants as cte
from .. import _dev, _lib


def _codes_ptr():
    if cte.BOUND_MODE == 3:
        if cte.boundaries is None:
            raise RuntimeError("custom boundary mode needs constants.init_custom_boundaries()")
        return _dev.ptr(cte.boundaries, "u8", cte.NX * cte.NY, "boundaries")
    return None


_draws = [0]  # calls to the stochastic form so far: each call draws new numbers


def next_seed(base: int | None = None) -> int:
    """Seed of the next stochastic draw: RAND_SEED (constants) mixed with a call
    counter, so that successive calls differ and a run is reproducible."""
    _draws[0] += 1
    b = cte.RAND_SEED if base is None else base
    return (int(b) * 1000003 + _draws[0]) & 0xFFFFFFFFFFFFFFFF


def compute_receivers(z, receivers, gradient):
    """D4 steepest-descent receivers and gradients (receivers.py:15-58), grid from
    ``constants`` (NX, NY, DX, BOUND_MODE, boundaries).  With RAND_RCV the slopes are
    scaled by uniform draws (receivers.py:46-47; see pff_compute_receivers_stochastic)."""
    N = cte.NX * cte.NY
    if cte.RAND_RCV:
        _lib.call("pff_compute_receivers_stochastic", _dev.ptr(z, "f32", N, "z"),
                  _dev.ptr(receivers, "i32", N, "receivers"), _dev.ptr(gradient, "f32", N, "gradient"), cte.NX,
                  cte.NY, float(cte.DX), cte.BOUND_MODE, _codes_ptr(), next_seed(), _dev.stream())
        return
    _lib.call("pff_compute_receivers", _dev.ptr(z, "f32", N, "z"), _dev.ptr(receivers, "i32", N, "receivers"),
              _dev.ptr(gradient, "f32", N, "gradient"), cte.NX, cte.NY, float(cte.DX), cte.BOUND_MODE,
              _codes_ptr(), _dev.stream())
