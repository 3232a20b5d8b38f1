"""GraphFlood: ``pyfastflow.graphflood`` on B200 (graphflood/__init__.py:35-49)."""
from .gf_fields import Flooder
from .gf_hydrodynamics import diffuse_Q_constant_prec, graphflood_core_cte_mannings
from .ragged import RaggedFlooder
from . import gf_fields, gf_hydrodynamics, ragged

__all__ = ["Flooder", "RaggedFlooder", "diffuse_Q_constant_prec", "graphflood_core_cte_mannings", "gf_fields",
           "gf_hydrodynamics", "ragged"]
