"""The N-GPU replica path's host logic on two gloo ranks (CPU): ranks share nothing but the
barriers and the max-reduction of their timed regions, and the whole-job seconds per solve is the
slowest rank's time over all ranks' solves."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from vhci_b200.replicas import Replicas, job_seconds_per_solve
    rep = Replicas(backend="gloo", timeout_s=60)
    rep.barrier()
    t = 1.5 + rank                      # rank 1 is the slow one
    t_max = rep.allmax(t)
    total = rep.allsum(3.0)             # 3 solves per rank
    out[rank] = (t_max, total, job_seconds_per_solve(t_max, 3, world))
    rep.barrier()
    rep.close()


def test_two_gloo_ranks_max_and_job_value():
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        t_max, total, value = res[r]
        assert t_max == 2.5 and total == 6.0
        assert value == pytest.approx(2.5 / 6.0)


def test_single_process_needs_no_group(monkeypatch):
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE"):
        monkeypatch.delenv(k, raising=False)
    from vhci_b200.replicas import Replicas
    rep = Replicas(backend="gloo")
    assert rep.world == 1 and rep.allmax(4.0) == 4.0
    rep.barrier()
    rep.close()
