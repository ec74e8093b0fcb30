"""The collectives of a sharded solve (vhci_b200.shard.Comm) on two gloo ranks over CPU buffers:
the callbacks the library calls (through the vhci_comm function pointers) sum doubles in place
and gather equal-sized byte blocks in rank order."""
import ctypes
import os
import socket
from datetime import timedelta

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=60))
    from vhci_b200 import shard
    comm = shard.Comm(device="cpu")
    assert comm.struct.rank == rank and comm.struct.nranks == world
    # all-reduce through the C function pointer, as the library calls it
    buf = np.arange(5, dtype=np.float64) + 10.0 * rank
    rc1 = comm.struct.allreduce_sum(None, buf.ctypes.data, buf.size)
    # all-gather of 24-byte blocks
    send = np.full(3, rank + 0.5)
    recv = np.zeros(3 * world)
    rc2 = comm.struct.allgather(None, send.ctypes.data, recv.ctypes.data, send.nbytes)
    out[rank] = (rc1, rc2, buf.tolist(), recv.tolist(), list(comm.errors))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_sum_and_gather():
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    expect_sum = (np.arange(5) * world + 10.0 * sum(range(world))).tolist()
    expect_gather = [r + 0.5 for r in range(world) for _ in range(3)]
    for r in range(world):
        rc1, rc2, s, g, errors = res[r]
        assert rc1 == 0 and rc2 == 0, errors
        assert s == expect_sum
        assert g == expect_gather
