"""Collectives for one solve sharded over several GPUs (vhci_set_comm).

The library splits the Hamiltonian's rows and the eigensolver's Krylov basis over the ranks and
asks its caller for two collectives on device buffers: a sum all-reduce of doubles and an
all-gather of equal-sized byte blocks (include/vhci_gpu.h, "one solve sharded over several GPUs").
`Comm` provides them from a torch.distributed process group — NCCL over NVLink between GPUs in
production; gloo also accepts CUDA tensors, and CPU buffers (device="cpu") for testing the
plumbing without a GPU.  A callback completes its collective (and synchronises the device)
before returning, as the library requires.

    import torch.distributed as dist
    from vhci_b200 import api, shard
    dist.init_process_group("nccl")                     # one process per GPU
    with api.VHCI("input.inp", device=local_rank) as v:
        v.set_comm(shard.Comm())                         # every rank, same input, same calls
        v.hci(); dE, n_pert = v.pt2()
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch
import torch.distributed as dist

from vhci_b200 import api


class _DeviceBuffer:
    """A device pointer presented through the CUDA array interface, so torch can view it."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"data": (int(ptr), False), "shape": tuple(shape),
                                         "typestr": typestr, "strides": None, "version": 2}


def _view(ptr: int, count: int, dtype, device: str) -> torch.Tensor:
    """A tensor sharing `count` elements of memory at ptr (device memory, or host for "cpu")."""
    if device == "cpu":
        ctype = ctypes.c_double if dtype == torch.float64 else ctypes.c_uint8
        arr = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctype)), shape=(count,))
        return torch.from_numpy(arr)
    typestr = "<f8" if dtype == torch.float64 else "|u1"
    return torch.as_tensor(_DeviceBuffer(ptr, (count,), typestr), device=device)


class Comm:
    """vhci_comm over a torch.distributed process group (the default group unless given)."""

    def __init__(self, group=None, device: str | None = None):
        self.group = group
        self.rank = dist.get_rank(group)
        self.nranks = dist.get_world_size(group)
        self.device = device or ("cuda" if torch.cuda.is_available() else "cpu")
        self.errors = []
        self._ar = api.ALLREDUCE_CB(self._allreduce)
        self._ag = api.ALLGATHER_CB(self._allgather)
        self.struct = api.Comm(self.rank, self.nranks, None, self._ar, self._ag)

    def _sync(self):
        if self.device != "cpu":
            torch.cuda.synchronize()

    def _allreduce(self, user, buf, count) -> int:
        try:
            t = _view(buf, int(count), torch.float64, self.device)
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
            self._sync()
            return 0
        except Exception as e:  # reported to the library as a failed collective
            self.errors.append(repr(e))
            return 1

    def _allgather(self, user, send, recv, nbytes) -> int:
        try:
            nbytes = int(nbytes)
            src = _view(send, nbytes, torch.uint8, self.device)
            dst = _view(recv, nbytes * self.nranks, torch.uint8, self.device)
            dist.all_gather(list(dst.split(nbytes)), src, group=self.group)
            self._sync()
            return 0
        except Exception as e:
            self.errors.append(repr(e))
            return 1
