"""The halo exchange of a rank of a decomposed domain over NCCL.

OLAM exchanges the border columns of every tracer between MPI ranks after
each RK stage but the last (omodel/scalar_transport_rk.F90:315-322, 343,
379, through olam_mpi_atm.F90).  The library packs the columns a rank sends
into one device buffer per neighbour and calls an exchange hook
(``olamgpu_set_halo``); this module gives that hook for torch.distributed's
NCCL backend: one grouped send/receive per neighbour, ordered on the
library's own stream, so the unpack the library enqueues after the hook
waits for the receive without the host waiting for anything.
"""
from __future__ import annotations


class _DeviceArray:
    """A float32 device buffer described by __cuda_array_interface__."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False),
                                         "version": 3, "strides": None}


def device_view(ptr: int, n: int):
    """A torch tensor viewing n float32 values of device memory at ptr (no copy)."""
    import torch
    return torch.as_tensor(_DeviceArray(ptr, n), device="cuda")


def host_view(ptr: int, n: int):
    """A torch tensor viewing n float32 values of host memory at ptr (no copy)."""
    import ctypes

    import numpy as np
    import torch
    if n == 0:
        return torch.zeros(0, dtype=torch.float32)
    return torch.from_numpy(np.ctypeslib.as_array((ctypes.c_float * n).from_address(ptr)))


def nccl_exchange(dist, view=None, on_stream=None):
    """The exchange hook for abi.make_halo_device: sends each neighbour its
    packed columns and receives its own, as one batch of point-to-point
    operations on the library's stream.  view(ptr, n) wraps a buffer and
    on_stream(stream) orders the operations; both default to device
    memory and the library's CUDA stream (with host views and no stream
    the same hook runs over gloo, which is how the pairing is tested
    without a GPU)."""
    import torch
    if view is None:
        view = device_view
    if on_stream is None:
        def on_stream(stream):
            return torch.cuda.stream(torch.cuda.ExternalStream(stream))

    def fn(ranks, sbufs, rbufs, stream):
        with on_stream(stream):
            ops = []
            for r, (sp, sn), (rp, rn) in zip(ranks, sbufs, rbufs):
                if sn:
                    ops.append(dist.P2POp(dist.isend, view(sp, sn), r))
                if rn:
                    ops.append(dist.P2POp(dist.irecv, view(rp, rn), r))
            if ops:
                for req in dist.batch_isend_irecv(ops):
                    req.wait()   # with a CUDA stream: the stream waits, the host does not
        return 0

    return fn
