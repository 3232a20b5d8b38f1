"""Torch tensor plumbing for the C ABI: pointer/dtype checks, stream, scratch."""
from __future__ import annotations

import torch

_DT = {
    "f32": torch.float32,
    "i32": torch.int32,
    "i64": torch.int64,
    "u8": torch.uint8,
    "bool": torch.bool,
}


def ptr(t, kind: str, n: int | None = None, name: str = "tensor") -> int:
    """Device pointer of a contiguous CUDA tensor of the expected dtype and size."""
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name}: expected a torch CUDA tensor, got {type(t).__name__}")
    if not t.is_cuda:
        raise TypeError(f"{name}: tensor must live on a CUDA device")
    want = _DT[kind]
    if t.dtype != want and not (kind == "u8" and t.dtype == torch.bool):
        raise TypeError(f"{name}: dtype {t.dtype}, expected {want}")
    if not t.is_contiguous():
        raise ValueError(f"{name}: tensor must be contiguous")
    if n is not None and t.numel() < n:
        raise ValueError(f"{name}: {t.numel()} elements, need at least {n}")
    return t.data_ptr()


def stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def resolve_device(device):
    """torch.device with an explicit index ("cuda" -> the current CUDA device): tensors
    always report an index, so comparisons need one."""
    if device is None:
        return None
    device = torch.device(device)
    if device.type == "cuda" and device.index is None and torch.cuda.is_available():
        device = torch.device("cuda", torch.cuda.current_device())
    return device


class Scratch:
    """Grow-only device scratch buffer (one per owner), handed to the C ABI as workspace."""

    def __init__(self):
        self.buf = None

    def get(self, nbytes: int, device=None) -> tuple[int, int]:
        """The buffer (at least nbytes) as (pointer, size).  It is reallocated only when it
        is too small or on another device, so graphs that captured its address stay valid;
        "cuda" without an index means the current device."""
        nbytes = max(int(nbytes), 256)
        device = resolve_device(device)
        if self.buf is None or self.buf.numel() < nbytes or (device is not None and self.buf.device != device):
            self.buf = torch.empty(nbytes, dtype=torch.uint8, device=device or "cuda")
        return self.buf.data_ptr(), self.buf.numel()


_shared = Scratch()


def shared_scratch(nbytes: int, device=None) -> tuple[int, int]:
    """Module-level scratch for the kernel-level functions (one call at a time)."""
    return _shared.get(nbytes, device)
