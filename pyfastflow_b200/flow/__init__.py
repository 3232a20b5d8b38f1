"""Flow routing: ``pyfastflow.flow`` on B200 (hand-written sm_100a CUDA via libpff).

Same module layout and names as pyfastflow/flow/__init__.py:26-47; kernel-level
functions take torch CUDA tensors where the reference takes Taichi fields."""
from .. import constants
from ..constants import *  # noqa: F401,F403  (the reference re-exports the constants)
from .environment import initialise, reboot
from .receivers import compute_receivers
from .downstream_propag import rcv2donor, rake_compress_accum, fuse
from .lakeflow import depression_counter, basin_identification, saddlesort, reroute_flow
from .f32_i32_struct import pack_float_index, unpack_float_index
from .fill_topo import fill_z_add_delta, topofill
from .flowfields import FlowRouter
from .ragged import RaggedRouter
from . import environment, receivers, downstream_propag, lakeflow, f32_i32_struct, fill_topo, flowfields, ragged

__all__ = [
    "environment", "receivers", "downstream_propag", "lakeflow", "f32_i32_struct", "fill_topo", "flowfields",
    "ragged",
    "FlowRouter", "RaggedRouter", "compute_receivers", "rcv2donor", "rake_compress_accum", "fuse", "depression_counter",
    "basin_identification", "saddlesort", "reroute_flow", "fill_z_add_delta", "topofill", "pack_float_index",
    "unpack_float_index", "initialise", "reboot",
]
