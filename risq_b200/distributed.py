"""Row-block partition of sigma over several GPUs, one process per GPU.

Every rank holds the whole determinant set and a handle of its own; with
GpuHam.set_partition(rank, nranks, make_allreduce()) an upper-triangle build keeps
the rank's share of the row panels, and every sigma adds the ranks' 64-bit
fixed-point partial sums through the all-reduce made here (torch.distributed:
NCCL on the device buffer, or gloo through host memory).  Integer sums are exact,
so each rank gets the full sigma bit for bit and the Davidson solves, replicated
on the ranks, stay identical without any further exchange.  The reference splits
no work at all (it is single-threaded); its matrix_vector_prod
(src/var/sparse.rs:64-78) is what is divided here, by rows.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A


class _DeviceInt64:
    """A device buffer of int64 seen through __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<i8", "data": (int(ptr), False),
                                         "version": 3, "strides": None, "stream": None}


def reduce_host_array(arr: np.ndarray, group=None) -> None:
    """Sum an int64 host array in place across the ranks of `group`."""
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(arr)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)


def make_allreduce(group=None, host_buffers: bool = False):
    """A risqgpu_allreduce_fn over torch.distributed.

    Device buffers (the library's case): with NCCL the sum runs on the device, ordered
    on the library's stream; with gloo the buffer goes through host memory.  With
    host_buffers the pointer addresses host memory (for callers that hold their
    partial sums on the host).  The returned object must stay alive while the handle
    uses it (GpuHam.set_partition keeps it)."""
    import torch.distributed as dist
    backend = dist.get_backend(group)

    def fn(ptr, count, stream, user):
        try:
            if host_buffers:
                arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_int64)), shape=(int(count),))
                reduce_host_array(arr, group)
                return 0
            import torch
            s = torch.cuda.ExternalStream(stream) if stream else torch.cuda.current_stream()
            with torch.cuda.stream(s):
                t = torch.as_tensor(_DeviceInt64(ptr, count), device="cuda")
                if backend == "nccl":
                    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
                else:
                    h = t.cpu()
                    reduce_host_array(h.numpy(), group)
                    t.copy_(h)
            return 0
        except Exception:  # reported to the library as a failed call
            return 1

    return A.ALLREDUCE_FN(fn)
