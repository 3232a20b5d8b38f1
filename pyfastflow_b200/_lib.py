"""Loader for ``libpff.so``, the sm_100a CUDA library behind this package.

The library is built in-tree (``pyfastflow_b200/libpff.so``) by
``pyfastflow_b200.build.build()``.  There is no fallback: if the library is
missing every call raises, so a run can never silently compute on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpff.so")

_vp, _i32, _i64, _f32, _f64, _sz = C.c_void_p, C.c_int, C.c_int64, C.c_float, C.c_double, C.c_size_t

# name -> (restype, argtypes); mirrors include/pff.h
SIGNATURES = {
    "pff_version": (_i32, []),
    "pff_last_error_string": (C.c_char_p, []),
    "pff_launch_count": (C.c_longlong, []),
    "pff_probe_enable": (_i32, [_i32]),
    "pff_probe_read": (_i32, [C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "pff_reroute_use_graphs": (_i32, [_i32]),
    "pff_reroute_flow_async": (_i32, [_vp] * 12 + [_i32, _i32, _i32, _vp, _vp, _sz, _vp, _vp]),
    "pff_reroute_flow_finish": (_i32, [_vp] * 12 + [_i32, _i32, _i32, _vp, _vp, _sz, _vp, _vp, _vp]),
    "pff_guard_begin": (_i32, [_vp, _vp, _vp, _vp]),
    "pff_guard_end": (_i32, [_i32, _vp]),
    "pff_guard_launch": (_i32, [_i32, _vp]),
    "pff_guard_destroy": (_i32, [_i32]),
    "pff_residual_flag": (_i32, [_vp, _f64, _f64, _vp, _vp]),
    "pff_value_store": (_i32, [_vp, _vp, _vp, _vp]),
    "pff_set_device": (_i32, [_i32]),
    "pff_compute_receivers": (_i32, [_vp, _vp, _vp, _i32, _i32, _f32, _i32, _vp, _vp]),
    "pff_compute_receivers_stochastic": (_i32, [_vp, _vp, _vp, _i32, _i32, _f32, _i32, _vp, C.c_uint64, _vp]),
    "pff_rcv2donor": (_i32, [_vp, _vp, _vp, _i32, _vp]),
    "pff_rake_compress_accum": (_i32, [_vp] * 7 + [_i32, _i32, _vp]),
    "pff_fuse": (_i32, [_vp, _vp, _vp, _i32, _i32, _vp]),
    "pff_accumulate_workspace_bytes": (_sz, [_i32]),
    "pff_accumulate": (_i32, [_vp, _vp, _vp, _i32, _vp, _sz, _vp]),
    "pff_accumulate_grid": (_i32, [_vp, _vp, _vp, _i32, _i32, _i32, _vp, _i32, _vp, _sz, _vp]),
    "pff_accumulate_set_front": (_i32, [_i32]),
    "pff_accumulate_tree_workspace_bytes": (_sz, [_i32, _i32, _i32]),
    "pff_accumulate_tree": (_i32, [_vp, _vp, _f32, _vp, _vp, _i32, _i32, _i32, _vp, _sz, _vp]),
    "pff_accumulate_tree_status": (_i32, [_i32, _i32, _i32, _vp, _sz, C.POINTER(C.c_int), _vp]),
    "pff_reroute_workspace_bytes": (_sz, [_i32]),
    "pff_reroute_flow": (_i32, [_vp] * 12 + [_i32, _i32, _i32, _i32, _vp, _vp, _sz, C.POINTER(C.c_int), _vp]),
    "pff_basin_identification": (_i32, [_vp, _vp, _vp, _i32, _i32, _i32, _vp, _vp]),
    "pff_depression_counter": (_i32, [_vp, _i32, _i32, _i32, _vp, C.POINTER(C.c_int), _vp]),
    "pff_saddlesort": (_i32, [_vp] * 7 + [_i32, _i32, _i32, _vp, _vp]),
    "pff_fill_workspace_bytes": (_sz, [_i32]),
    "pff_fill_z_add_delta": (_i32, [_vp] * 6 + [_f64, _i32, _vp, _sz, _vp]),
    "pff_fill_z_add_delta_noalloc": (_i32, [_vp] * 6 + [_f64, _i32, _vp]),
    "pff_topofill": (_i32, [_vp] * 5 + [_f64, _i32, _i32, _vp, _sz, _vp]),
    "pff_diffuse_workspace_bytes": (_sz, [_i32]),
    "pff_diffuse_q": (_i32, [_vp, _vp, _vp, _i32, _i32, _i32, _f32, _f32, _i32, _vp, _vp, _sz, _vp]),
    "pff_graphflood_core": (_i32, [_vp] * 5 + [_i32] + [_f32] * 5 + [_vp, _vp, _vp]),
    "pff_graphflood_core_filled": (_i32, [_vp] * 6 + [_i32] + [_f32] * 5 + [_vp, _vp, _vp]),
    "pff_abs_diff_stats": (_i32, [_vp, _vp, _i32, _vp, _vp]),
    "pff_archive_workspace_bytes": (_sz, [_i32]),
    "pff_tree_accum_down": (_i32, [_vp, _vp, _vp, _i32, _vp, _sz, _vp]),
    "pff_tree_max_down": (_i32, [_vp, _vp, _i32, _vp, _sz, _vp]),
    "pff_erode_deposit": (_i32, [_vp] * 5 + [_f32] * 7 + [_vp, _vp, _i32, _vp, _sz, _vp]),
    "pff_batch_workspace_bytes": (_sz, [_i64, _i32]),
    "pff_batch_plan": (_i64, [_vp, _vp, _vp, _vp, _i32, _vp, _vp, _vp, _sz, _vp]),
    "pff_batch_route": (_i32, [_vp] * 6 + [_i64, _i32, _i32, _i32, _vp, _sz, _vp]),
    "pff_batch_status": (_i32, [_i64, _i32, _vp, _sz, C.POINTER(C.c_int), _vp]),
    "pff_batch_graphflood": (_i32, [_vp, _vp, _vp, _vp, _vp, _f32, _f32, _i32, _i32, _vp, _vp, _vp, _i64, _i32,
                                    _i32, _i32, _vp, _sz, _vp]),
    "pff_conv3x3_fwd": (_i32, [_vp, _i32, _i32, _vp, _vp, _vp, _i32, _i32] + [_i32] * 7 + [_vp]),
    "pff_receivers_set_path": (_i32, [_i32]),
    "pff_receivers_div_selfcheck": (_i32, [_f32, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "pff_conv_set_path": (_i32, [_i32]),
    "pff_conv_tc_status": (_i32, [C.POINTER(C.c_int)]),
    "pff_conv3x3_wflip": (_i32, [_vp, _vp, _i32, _i32, _vp]),
    "pff_conv3x3_wgrad": (_i32, [_vp, _i32, _i32, _vp, _i32, _i32, _vp] + [_i32] * 5 + [_vp]),
    "pff_bias_grad": (_i32, [_vp, _i32, _i32, _vp, _i64, _i32, _vp]),
    "pff_relu_bwd": (_i32, [_vp, _i32, _i32, _vp, _i32, _i32, _i64, _i32, _vp]),
    "pff_avgpool2": (_i32, [_vp, _i32, _i32, _vp, _i32, _i32] + [_i32] * 4 + [_vp]),
    "pff_avgpool2_bwd": (_i32, [_vp, _i32, _i32, _vp, _i32, _i32] + [_i32] * 5 + [_vp]),
    "pff_upsample2": (_i32, [_vp, _i32, _i32, _vp, _i32, _i32] + [_i32] * 4 + [_vp]),
    "pff_upsample2_bwd": (_i32, [_vp, _i32, _i32, _vp, _i32, _i32] + [_i32] * 4 + [_vp]),
    "pff_mse_loss": (_i32, [_vp, _i32, _vp, _vp, _i64, _vp, _i32, _f32, _vp, _vp]),
    "pff_adam": (_i32, [_vp, _vp, _vp, _vp, _vp, _i64, _f32, _f32, _f32, _f32, _i32, _f32, _vp]),
    "pff_f32_to_bf16": (_i32, [_vp, _vp, _i64, _vp]),
    "pff_unet_features": (_i32, [_vp, _vp, _vp, _vp, _vp, _f32, _i32, _i64, _vp, _vp, _vp]),
    "pff_unet_h0": (_i32, [_vp, _i32, _vp, _i64, _f32, _vp, _vp, _vp]),
    "pff_unet_target": (_i32, [_vp, _vp, _i64, _f32, _vp]),
}

_lib = None


class PFFError(RuntimeError):
    pass


def load():
    """Load libpff.so (raises ImportError if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with pyfastflow_b200.build.build() "
                          "(nvcc, sm_100a); there is no CPU fallback")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


_tls = threading.local()


def _sync_device():
    """Keep the library's current device equal to torch's (per host thread)."""
    import torch

    if not torch.cuda.is_available():
        return  # host-side argument checks still run and report through the status
    d = torch.cuda.current_device()
    if getattr(_tls, "device", None) != d:
        rc = load().pff_set_device(d)
        if rc != 0:
            raise PFFError(f"pff_set_device({d}) failed: {load().pff_last_error_string().decode()}")
        _tls.device = d


def call(name: str, *args):
    """Call a libpff entry point and raise PFFError on a nonzero status."""
    _sync_device()
    fn = getattr(load(), name)
    rc = fn(*args)
    if rc != 0:
        msg = load().pff_last_error_string().decode(errors="replace")
        raise PFFError(f"{name} failed with status {rc}: {msg}")
    return rc
