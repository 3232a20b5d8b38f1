"""pyfastflow_b200 -- pyfastflow's flow-routing and GraphFlood hot path on NVIDIA B200.

``import pyfastflow_b200 as pf`` gives the reference's layout (pyfastflow/__init__.py:
``pf.constants``, ``pf.flow``, ``pf.graphflood``) over torch CUDA tensors; the
compute runs in hand-written sm_100a CUDA kernels in ``libpff.so`` (C ABI in
include/pff.h), loaded with ctypes.  There is no CPU fallback.
"""
__version__ = "0.1.0"

from . import constants
from . import flow
from . import graphflood
from . import archive

__all__ = ["constants", "flow", "graphflood", "archive"]
