"""Device buffers and streams as the C ABI sees them: (pointer, length in elements) and a
cudaStream_t handle.  torch provides the memory and the streams; it is plumbing only."""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class DevicePtr:
    """A raw device pointer with a length in elements (a DeviceSlice of the reference)."""
    ptr: int
    len: int
    elem_size: int = 8


def as_slice(x, elem_size: int = 8) -> tuple[int, int]:
    """(device address, length in elements) of a torch CUDA tensor or a DevicePtr."""
    if isinstance(x, DevicePtr):
        if x.elem_size != elem_size:
            raise TypeError("expected %d-byte elements" % elem_size)
        return x.ptr, x.len
    if hasattr(x, "data_ptr") and hasattr(x, "element_size"):
        if not x.is_cuda:
            raise TypeError("device buffer expected, got a host tensor")
        if x.element_size() != elem_size:
            raise TypeError("expected %d-byte elements, got %d-byte" % (elem_size, x.element_size()))
        if not x.is_contiguous():
            raise TypeError("device buffer must be contiguous")
        return x.data_ptr(), x.numel()
    raise TypeError("unsupported buffer type %r" % type(x))


def stream_handle(stream) -> int | None:
    """cudaStream_t of a torch stream, an int handle, or the current torch stream for None."""
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream or None
    if isinstance(stream, int):
        return stream or None
    return stream.cuda_stream or None
