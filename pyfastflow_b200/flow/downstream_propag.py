"""Rake-and-compress accumulation kernels, mirroring pyfastflow/flow/downstream_propag.py.

Same arguments and in-place semantics as the reference's Taichi kernels, taking
torch CUDA tensors instead of fields.  Donor slots are filled in ascending donor
index (the reference's serial order), which makes every round deterministic."""
from .. import _dev, _lib


def rcv2donor(rcv, dnr, ndnr):
    """downstream_propag.py:77-96; ndnr must be zero on entry."""
    N = rcv.numel()
    _lib.call("pff_rcv2donor", _dev.ptr(rcv, "i32", N, "rcv"), _dev.ptr(dnr, "i32", 4 * N, "dnr"),
              _dev.ptr(ndnr, "i32", N, "ndnr"), N, _dev.stream())


def rake_compress_accum(dnr, ndnr, p, src, dnr_, ndnr_, p_, iteration):
    """One rake-and-compress round (downstream_propag.py:99-179)."""
    N = p.numel()
    _lib.call("pff_rake_compress_accum", _dev.ptr(dnr, "i32", 4 * N, "dnr"), _dev.ptr(ndnr, "i32", N, "ndnr"),
              _dev.ptr(p, "f32", N, "p"), _dev.ptr(src, "i32", N, "src"), _dev.ptr(dnr_, "i32", 4 * N, "dnr_"),
              _dev.ptr(ndnr_, "i32", N, "ndnr_"), _dev.ptr(p_, "f32", N, "p_"), int(iteration), N, _dev.stream())


def fuse(A, src, B, iteration):
    """Select the final ping-pong buffer (downstream_propag.py:59-74)."""
    N = A.numel()
    _lib.call("pff_fuse", _dev.ptr(A, "f32", N, "A"), _dev.ptr(src, "i32", N, "src"), _dev.ptr(B, "f32", N, "B"),
              int(iteration), N, _dev.stream())
