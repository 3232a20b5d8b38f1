"""Packed (f32, i32) lexicographic keys, mirroring pyfastflow/flow/f32_i32_struct.py.

Key layout (f32_i32_struct.py:15-103): high 32 bits = raw float bits for
non-negative floats, (~bits) | 0x80000000 for negative ones; low 32 bits = the
index bits; keys compare as signed 64-bit integers, i.e. by (float, unsigned
index).  The GPU kernels use the same layout for their atomicMin.
"""
from __future__ import annotations

import numpy as np


def pack_float_index(f, i):
    """Pack float32 value(s) f and int32 index(es) i into int64 key(s)."""
    f = np.asarray(f, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    hi = np.where(u & 0x80000000, (~u & 0xFFFFFFFF) | 0x80000000, u)
    lo = np.asarray(i, dtype=np.int32).view(np.uint32).astype(np.uint64)
    k = ((hi << np.uint64(32)) | lo).astype(np.uint64).view(np.int64)
    return k if k.ndim else np.int64(k)


def unpack_float_index(k):
    """Inverse of pack_float_index: returns (float32, int32)."""
    k = np.asarray(k, dtype=np.int64).view(np.uint64)
    hi = (k >> np.uint64(32)) & np.uint64(0xFFFFFFFF)
    u = np.where(hi & 0x80000000, (~hi & 0xFFFFFFFF) | 0x80000000, hi).astype(np.uint32)
    f = u.view(np.float32)
    i = (k & np.uint64(0xFFFFFFFF)).astype(np.uint32).view(np.int32)
    if f.ndim == 0:
        return np.float32(f), np.int32(i)
    return f, i


INVALID_KEY = int(pack_float_index(np.float32(1e8), 42))  # lakeflow.py:127
