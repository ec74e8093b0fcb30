"""One solve sharded over two ranks (vhci_set_comm) equals the same solve on one rank.

The two ranks run as two processes on the same GPU and exchange their collectives through
torch.distributed's gloo backend, which moves the CUDA buffers through host memory: every wait is
on the host, no kernel waits for another rank.  Each rank holds half of the Hamiltonian's rows
and of the Krylov basis; the vector blocks are all-gathered, the projections all-reduced, and PT2
splits the perturber range.  The 24-mode, two-word-key fixture takes the sparse eigensolver path
(up to 47,176 states, three heat-bath iterations, 229,316 perturbers).  The sums run in a
different order than on one rank, so energies agree to 1e-8 cm^-1 rather than bit for bit; the
basis sizes and |P| are identical.
"""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

CASE = os.path.join(GOLDEN, "syn_m24_w2", "input.inp")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _solve(v):
    sizes = []
    v.hci(callback=lambda it, n, zpe: sizes.append(n) if it > 0 else None)
    E_var = v.energies().copy()
    dE, npert = v.pt2()
    return {"sizes": sizes, "n": v.n, "E_var": E_var.tolist(), "E": v.energies().tolist(),
            "n_pert": npert}


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=300))
    from vhci_b200 import api, shard
    comm = shard.Comm(device="cuda")
    with api.VHCI(CASE, device=0) as v:
        v.set_comm(comm)
        r = _solve(v)
        # the held Hamiltonian is this rank's row block, not the whole matrix
        try:
            v.h_csr()
            r["h_sharded"] = False
        except api.VhciError as e:
            r["h_sharded"] = e.code == api.E_STATE
    r["errors"] = list(comm.errors)
    out[rank] = r
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_solve_equals_single_rank():
    from vhci_b200 import api
    with api.VHCI(CASE) as v:
        ref = _solve(v)
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        got = res[r]
        assert not got["errors"], got["errors"]
        assert got["h_sharded"]
        assert got["sizes"] == ref["sizes"] and got["n"] == ref["n"]
        assert got["n_pert"] == ref["n_pert"]
        assert np.abs(np.array(got["E_var"]) - np.array(ref["E_var"])).max() < 1e-8
        assert np.abs(np.array(got["E"]) - np.array(ref["E"])).max() < 1e-8
    assert res[0]["E"] == res[1]["E"]  # every rank holds the same result
