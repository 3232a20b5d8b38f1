"""ctypes wrapper around the CPU oracle (``libpff_oracle.so``).

TEST INFRASTRUCTURE ONLY.  tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline / reference legs import this module as the checker (and as the timed
CPU implementation of the reference algorithm); the product package never does.

Every function restates a pyfastflow kernel or driver with serial ascending-index
semantics; the C source cites the reference file:line for each one.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "libpff_oracle.so")


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, no fast-math, no FP contraction)."""
    src = [os.path.join(_HERE, f) for f in ("pff_oracle.c", "pff_oracle_real.h", "Makefile")]
    if force or not os.path.exists(_SO) or any(os.path.getmtime(s) > os.path.getmtime(_SO) for s in src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


class _Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("mode", C.c_int), ("codes", C.c_void_p)]


class _GFParams(C.Structure):
    _fields_ = [("dx", C.c_double), ("prec", C.c_double), ("manning", C.c_double),
                ("edgesw", C.c_double), ("dt", C.c_double), ("min_slope", C.c_double),
                ("fill_eps", C.c_double), ("serial_fill", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_SO)
        _lib.orc_pack_float_index.restype = C.c_int64
        _lib.orc_pack_float_index.argtypes = [C.c_float, C.c_int32]
        _lib.orc_unpack_float_index.argtypes = [C.c_int64, C.POINTER(C.c_float), C.POINTER(C.c_int32)]
        _lib.orc_neighbour.argtypes = [C.POINTER(_Grid), C.c_int, C.c_int]
        _lib.orc_can_leave.argtypes = [C.POINTER(_Grid), C.c_int]
        _lib.orc_compute_receivers_f32.argtypes = [C.c_void_p] * 3 + [C.POINTER(_Grid), C.c_float]
        _lib.orc_compute_receivers_f64.argtypes = [C.c_void_p] * 3 + [C.POINTER(_Grid), C.c_double]
        _lib.orc_saddlesort_f32.argtypes = [C.c_void_p] * 7 + [C.POINTER(_Grid)]
        _lib.orc_reroute_flow_f32.argtypes = [C.c_void_p] * 12 + [C.POINTER(_Grid), C.c_int, C.c_void_p]
        _lib.orc_fill_z_add_delta_f32.argtypes = [C.c_void_p] * 7 + [C.c_int, C.c_int, C.c_int, C.c_void_p]
        _lib.orc_diffuse_q_f32.argtypes = [C.c_void_p] * 3 + [C.POINTER(_Grid), C.c_float, C.c_float]
        _lib.orc_graphflood_core_f32.argtypes = [C.c_void_p] * 5 + [C.c_int] + [C.c_float] * 6
        _lib.orc_graphflood_run_f32.argtypes = [C.c_void_p] * 3 + [C.POINTER(_Grid), C.POINTER(_GFParams), C.c_int, C.c_void_p]
        _lib.orc_graphflood_run_f64.argtypes = [C.c_void_p] * 3 + [C.POINTER(_Grid), C.POINTER(_GFParams), C.c_int, C.c_void_p]
        _lib.orc_depression_counter.argtypes = [C.c_void_p, C.POINTER(_Grid)]
        _lib.orc_basin_identification.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(_Grid)]
        _lib.orc_rcv2donor.argtypes = [C.c_void_p] * 3 + [C.c_int]
        _lib.orc_rake_compress_accum.argtypes = [C.c_void_p] * 7 + [C.c_int, C.c_int]
        _lib.orc_fuse.argtypes = [C.c_void_p] * 3 + [C.c_int, C.c_int]
        _lib.orc_accumulate.argtypes = [C.c_void_p] * 3 + [C.c_int, C.c_void_p, C.c_void_p]
        _lib.orc_topo_accumulate_u32.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        _lib.orc_count_cycle_nodes.argtypes = [C.c_void_p, C.c_int]
        _lib.orc_neighbour_table.argtypes = [C.POINTER(_Grid), C.c_void_p, C.c_void_p]
        _lib.orc_set_threads.argtypes = [C.c_int]
        _lib.orc_tree_accum_down_f32.argtypes = [C.c_void_p] * 3 + [C.c_int] + [C.c_void_p] * 3
        _lib.orc_tree_max_down_f32.argtypes = [C.c_void_p] * 2 + [C.c_int] + [C.c_void_p] * 2
        _lib.orc_erode_deposit_f32.argtypes = [C.c_void_p] * 5 + [C.c_float] * 7 + [C.c_void_p] * 2 + [C.c_int] + \
            [C.c_void_p] * 3
        _lib.orc_ceil_log2.argtypes = [C.c_longlong]
    return _lib


def set_threads(n: int) -> int:
    """OpenMP threads for the race-free loops (CPU-baseline timing); returns the count."""
    return lib().orc_set_threads(int(n))


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Grid:
    """Grid geometry + boundary mode (0 normal, 1 periodic EW, 2 periodic NS, 3 custom)."""

    def __init__(self, nx: int, ny: int, mode: int = 0, codes: np.ndarray | None = None):
        self.nx, self.ny, self.mode = int(nx), int(ny), int(mode)
        self.N = self.nx * self.ny
        self.codes = None
        if mode == 3:
            if codes is None:
                raise ValueError("custom mode needs codes")
            self.codes = np.ascontiguousarray(codes, dtype=np.uint8).ravel()
            assert self.codes.size == self.N
        self._g = _Grid(self.nx, self.ny, self.mode, _p(self.codes) if self.codes is not None else None)

    @property
    def ref(self):
        return C.byref(self._g)


def ceil_log2(n: int) -> int:
    return lib().orc_ceil_log2(int(n))


def pack_float_index(f: float, i: int) -> int:
    return lib().orc_pack_float_index(float(np.float32(f)), int(i))


def unpack_float_index(k: int):
    f = C.c_float()
    i = C.c_int32()
    lib().orc_unpack_float_index(int(k), C.byref(f), C.byref(i))
    return np.float32(f.value), int(i.value)


def neighbour_table(g: Grid):
    nb = np.empty(4 * g.N, np.int32)
    lv = np.empty(g.N, np.uint8)
    lib().orc_neighbour_table(g.ref, _p(nb), _p(lv))
    return nb.reshape(g.N, 4), lv.astype(bool)


def compute_receivers(z: np.ndarray, g: Grid, dx: float, f64: bool = False):
    dt = np.float64 if f64 else np.float32
    z = np.ascontiguousarray(z, dtype=dt).ravel()
    rcv = np.empty(g.N, np.int32)
    grad = np.empty(g.N, dt)
    if f64:
        lib().orc_compute_receivers_f64(_p(z), _p(rcv), _p(grad), g.ref, float(dx))
    else:
        lib().orc_compute_receivers_f32(_p(z), _p(rcv), _p(grad), g.ref, float(np.float32(dx)))
    return rcv, grad


def depression_counter(rec: np.ndarray, g: Grid) -> int:
    rec = np.ascontiguousarray(rec, np.int32)
    return lib().orc_depression_counter(_p(rec), g.ref)


def basin_labels(rec: np.ndarray, g: Grid) -> np.ndarray:
    """basin_identification (lakeflow.py:82-101): bid = root+1, or 0 for outlet roots."""
    rec = np.ascontiguousarray(rec, np.int32)
    bid = np.empty(g.N, np.int32)
    tmp = np.empty(g.N, np.int32)
    lib().orc_basin_identification(_p(bid), _p(rec), _p(tmp), g.ref)
    return bid


class LakeState:
    """The router's lake-flow fields (flowfields.py:119-159); basin arrays sized N+1."""

    def __init__(self, N: int):
        self.bid = np.zeros(N, np.int32)
        self.rec_ = np.zeros(N, np.int32)
        self.rec__ = np.zeros(N, np.int32)
        self.z_prime = np.zeros(N, np.float32)
        self.is_border = np.zeros(N, np.uint8)
        self.outlet = np.zeros(N + 1, np.int64)
        self.basin_saddle = np.zeros(N + 1, np.int64)
        self.basin_saddlenode = np.zeros(N + 1, np.int32)
        self.tag = np.zeros(N, np.uint8)
        self.tag_ = np.zeros(N, np.uint8)


def saddlesort(bid, z, g: Grid, st: LakeState | None = None) -> LakeState:
    st = st or LakeState(g.N)
    bid = np.ascontiguousarray(bid, np.int32)
    z = np.ascontiguousarray(z, np.float32)
    lib().orc_saddlesort_f32(_p(bid), _p(st.is_border), _p(st.z_prime), _p(st.basin_saddle),
                             _p(st.basin_saddlenode), _p(st.outlet), _p(z), g.ref)
    return st


def reroute_flow(rec: np.ndarray, z: np.ndarray, g: Grid, carve: bool = True, st: LakeState | None = None):
    """lakeflow.reroute_flow; returns (rec_after, rec__after, state, Ndep, n_outer).

    carve=True: the rerouted receivers are in ``rec`` (first return value).
    carve=False: the reference leaves its result in ``rec_`` (second value)."""
    st = st or LakeState(g.N)
    rec = np.array(rec, np.int32, copy=True)
    z = np.ascontiguousarray(z, np.float32)
    nout = C.c_int()
    nd = lib().orc_reroute_flow_f32(_p(st.bid), _p(rec), _p(st.rec_), _p(st.rec__), _p(z),
                                    _p(st.z_prime), _p(st.is_border), _p(st.outlet),
                                    _p(st.basin_saddle), _p(st.basin_saddlenode), _p(st.tag),
                                    _p(st.tag_), g.ref, int(bool(carve)), C.byref(nout))
    return rec, st.rec_.copy(), st, nd, nout.value


def rcv2donor(rcv, dnr, ndnr):
    lib().orc_rcv2donor(_p(rcv), _p(dnr), _p(ndnr), rcv.size)


def rake_compress_accum(dnr, ndnr, p, src, dnr_, ndnr_, p_, iteration: int):
    lib().orc_rake_compress_accum(_p(dnr), _p(ndnr), _p(p), _p(src), _p(dnr_), _p(ndnr_), _p(p_),
                                  int(iteration), p.size)


def fuse(A, src, B, iteration: int):
    lib().orc_fuse(_p(A), _p(src), _p(B), int(iteration), A.size)


def accumulate(rcv: np.ndarray, seed: np.ndarray | float = 1.0, with_counts: bool = True,
               return_active: bool = False):
    """accumulate_constant_Q's rake-and-compress chain (flowfields.py:272-292) with an
    arbitrary per-cell f32 seed; also exact uint32 counts through the same rounds."""
    rcv = np.ascontiguousarray(rcv, np.int32)
    N = rcv.size
    if np.isscalar(seed):
        Q = np.full(N, np.float32(seed), np.float32)
    else:
        Q = np.array(seed, np.float32, copy=True).ravel()
    cnt = np.empty(N, np.uint32) if with_counts else None
    ws = np.zeros(10 * N, np.int32)
    act = np.zeros(64, np.int32)
    rounds = lib().orc_accumulate(_p(rcv), _p(Q), _p(cnt) if cnt is not None else None, N, _p(ws), _p(act))
    if return_active:
        return Q, cnt, act[: ceil_log2(N) + 2].copy(), rounds
    return Q, cnt


def topo_accumulate(rcv: np.ndarray) -> np.ndarray:
    """Independent exact drainage count (Kahn topological order)."""
    rcv = np.ascontiguousarray(rcv, np.int32)
    cnt = np.empty(rcv.size, np.uint32)
    rc = lib().orc_topo_accumulate_u32(_p(rcv), _p(cnt), rcv.size)
    if rc != 0:
        raise ValueError("receivers contain a cycle")
    return cnt


def count_cycle_nodes(rcv: np.ndarray) -> int:
    rcv = np.ascontiguousarray(rcv, np.int32)
    return lib().orc_count_cycle_nodes(_p(rcv), rcv.size)


def fill_increments(N: int, eps: float) -> np.ndarray:
    """float32(2**(it-1) * eps) for it = 0..ceil(log2 N)-1 (fill_topo.py:36,121)."""
    return np.array([np.float32(2.0 ** (it - 1) * eps) for it in range(ceil_log2(N))], np.float32)


def fill_z_add_delta(zh, h, rec, eps: float = 1e-3, serial: bool = False):
    """fill_topo.fill_z_add_delta in place on (zh, h); returns (zh, h, z_)."""
    N = zh.size
    inc = fill_increments(N, eps)
    z_ = np.empty(N, np.float32)
    r_ = np.empty(N, np.int32)
    r__ = np.empty(N, np.int32)
    tmp = np.empty(N, np.float32)
    rec = np.ascontiguousarray(rec, np.int32)
    lib().orc_fill_z_add_delta_f32(_p(zh), _p(h), _p(z_), _p(rec), _p(r_), _p(r__), _p(inc),
                                   inc.size, N, int(serial), _p(tmp))
    return zh, h, z_


def topofill(z, rec, eps: float = 1e-6, serial: bool = False):
    """fill_topo.topofill (fill_topo.py:48-78 with _topofill :17-45): the same rounds as
    fill_z_add_delta with increments float32(2**it * eps), it = 0..ceil(log2 N)-1
    (the reference passes iteration it+1 and adds 2**(iteration-1) * eps); returns the
    filled surface z_."""
    z = np.array(z, np.float32, copy=True).ravel()
    N = z.size
    inc = np.array([np.float32(2.0 ** it * eps) for it in range(ceil_log2(N))], np.float32)
    h = np.zeros(N, np.float32)
    z_ = np.empty(N, np.float32)
    r_ = np.empty(N, np.int32)
    r__ = np.empty(N, np.int32)
    tmp = np.empty(N, np.float32)
    rec = np.ascontiguousarray(rec, np.int32)
    lib().orc_fill_z_add_delta_f32(_p(z), _p(h), _p(z_), _p(rec), _p(r_), _p(r__), _p(inc), inc.size, N,
                                   int(serial), _p(tmp))
    return z_


def diffuse_q(zh, Q, g: Grid, dx: float, prec: float):
    temp = np.empty_like(Q)
    lib().orc_diffuse_q_f32(_p(zh), _p(Q), _p(temp), g.ref, float(np.float32(dx)),
                            float(np.float32(prec * dx * dx)))
    return Q


def graphflood_core(h, zh, rec, Q, dx, manning, edgesw, dt=5e-3):
    dh = np.empty_like(h)
    lib().orc_graphflood_core_f32(_p(h), _p(zh), _p(dh), _p(rec), _p(Q), h.size,
                                  float(np.float32(dx)), float(np.float32(dx * dx)),
                                  float(np.float32(manning)), float(np.float32(edgesw)),
                                  float(np.float32(dt)), float(np.float32(1e-4)))
    return h, zh, dh


def graphflood_run(zh, h, Q, g: Grid, dx, prec, manning=0.033, edgesw=1e-2, dt=5e-3, niter=1,
                   f64=False, serial_fill=False, fill_eps=1e-3):
    """Flooder.run_graphflood (gf_fields.py:111-141) in place on (zh, h, Q).
    Returns the per-iteration max |dh| trace."""
    dt_ = np.float64 if f64 else np.float32
    for a in (zh, h, Q):
        assert a.dtype == dt_ and a.flags.c_contiguous
    prm = _GFParams(float(dx), float(prec), float(manning), float(edgesw), float(dt), 1e-4,
                    float(fill_eps), int(serial_fill))
    trace = np.zeros(niter, dt_)
    fn = lib().orc_graphflood_run_f64 if f64 else lib().orc_graphflood_run_f32
    fn(_p(zh), _p(h), _p(Q), g.ref, C.byref(prm), int(niter), _p(trace))
    return trace


# ---- legacy downstream tree algorithms (archive/fastflow/kernels) ------------
def tree_accum_down(rcv, W, p):
    """tree_accum_down rounds; returns (rcv, W, p) as the reference leaves them."""
    rcv = np.array(rcv, np.int32, copy=True)
    W = np.array(W, np.float32, copy=True)
    p = np.array(p, np.float32, copy=True)
    N = p.size
    r2, W2, p2 = np.empty_like(rcv), np.empty_like(W), np.empty_like(p)
    lib().orc_tree_accum_down_f32(_p(rcv), _p(W), _p(p), N, _p(r2), _p(W2), _p(p2))
    return rcv, W, p


def tree_max_down(rcv, p):
    """tree_max_down rounds; returns (rcv, p) as the reference leaves them."""
    rcv = np.array(rcv, np.int32, copy=True)
    p = np.array(p, np.float32, copy=True)
    r2, p2 = np.empty_like(rcv), np.empty_like(p)
    lib().orc_tree_max_down_f32(_p(rcv), _p(p), p.size, _p(r2), _p(p2))
    return rcv, p


def erode_deposit(z, bound, rcv, drain, Qs, dt, dx, k_spl, k_t, k_h, k_d, m):
    """erode_deposit kernel + downstream solve; returns (z after deposition, new
    elevations pe, We after the rounds)."""
    z = np.array(z, np.float32, copy=True).ravel()
    N = z.size
    bound = np.ascontiguousarray(bound, np.uint8).ravel()
    rcv = np.array(rcv, np.int32, copy=True).ravel()
    drain = np.ascontiguousarray(drain, np.float32).ravel()
    Qs = np.ascontiguousarray(Qs, np.float32).ravel()
    pe, We = np.empty(N, np.float32), np.empty(N, np.float32)
    r2, W2, p2 = np.empty(N, np.int32), np.empty(N, np.float32), np.empty(N, np.float32)
    f = lambda x: float(np.float32(x))  # noqa: E731
    lib().orc_erode_deposit_f32(_p(z), _p(bound), _p(rcv), _p(drain), _p(Qs), f(dt), f(dx), f(k_spl), f(k_t), f(k_h),
                                f(k_d), f(m), _p(pe), _p(We), N, _p(r2), _p(W2), _p(p2))
    return z, pe, We
