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


def nccl_exchange(dist):
    """The exchange hook for abi.make_halo_device: sends each neighbour its
    packed columns and receives its own, as one batch of NCCL point-to-point
    operations on the library's stream."""
    import torch

    def fn(ranks, sbufs, rbufs, stream):
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            ops = []
            for r, (sp, sn), (rp, rn) in zip(ranks, sbufs, rbufs):
                if sn:
                    ops.append(dist.P2POp(dist.isend, device_view(sp, sn), r))
                if rn:
                    ops.append(dist.P2POp(dist.irecv, device_view(rp, rn), r))
            if ops:
                for req in dist.batch_isend_irecv(ops):
                    req.wait()   # the library stream waits; the host does not
        return 0

    return fn
