"""Request server (vhci_serve): continuous batching of independent solves on one GPU.  Each
request's result must be the same when it runs alone and when it runs in the mix (concurrent
contexts on separate CUDA streams share the device but no state), and the per-request size limits
must reject a request before it builds the oversized step."""
import numpy as np
import pytest

from conftest import load_golden
from vhci_b200 import pes as P

pytestmark = pytest.mark.gpu


def small_requests(tmp_path, n=10):
    """Small admissible requests of mixed sizes (Nm 6..10, Nstate 5..29, PT2 on)."""
    reqs = []
    for r in range(n):
        rng = np.random.default_rng(900 + r)
        nm = int(rng.integers(6, 11))
        run = P.RunSettings(eps1=float("%.4f" % rng.uniform(1.0, 3.0)),
                            nstate=int(rng.integers(5, 30)), pt2=1, eps2=0.3)
        for j in range(200):
            pes = P.generate(P.PESSpec(nm), 777000 + 1000 * r + j)
            if P.admissible(pes):
                break
        path = str(tmp_path / f"req{r}.inp")
        P.write_input(path, pes, run)
        reqs.append(path)
    return reqs


def test_results_identical_alone_and_in_the_mix(tmp_path):
    from vhci_b200 import api
    paths = small_requests(tmp_path)
    alone = [api.solve(p) for p in paths]
    arrivals = [0.02 * i for i in range(len(paths))]
    summ, res = api.serve(list(zip(paths, arrivals)), slots=4, reserve_bytes=2e9)
    assert summ["failed"] == 0 and summ["completed"] == len(paths)
    assert summ["peak_in_flight"] >= 2          # requests really overlapped
    for a, r in zip(alone, res):
        assert r["status"] == 0, r["message"]
        assert r["n_basis"] == a["n_basis"] and r["n_pert"] == a["n_pert"]
        assert len(r["E"]) == len(a["E"])
        assert np.allclose(r["E"], a["E"], rtol=0, atol=1e-8)
        assert r["t_admit"] >= r["arrival"] - 1e-6 and r["t_done"] >= r["t_admit"]


def test_single_slot_runs_in_arrival_order(tmp_path):
    from vhci_b200 import api
    paths = small_requests(tmp_path, n=4)
    summ, res = api.serve([(p, 0.01 * (3 - i)) for i, p in enumerate(paths)], slots=1)
    assert summ["failed"] == 0 and summ["peak_in_flight"] == 1
    order = sorted(range(4), key=lambda i: res[i]["t_admit"])
    assert order == [3, 2, 1, 0]


def test_size_limits_reject_before_building():
    from vhci_b200 import api
    g = load_golden("syn_m8_sextic_pt2")
    sizes = g["log"]["sizes"]
    with api.VHCI(g["input"], max_basis=sizes[0] - 1) as v:
        with pytest.raises(api.VhciError) as e:
            v.hci()
        assert e.value.code == api.E_LIMIT and "max_basis" in str(e.value)
        assert v.n < sizes[0]                   # the oversized basis was never appended
    ref = api.solve(g["input"])
    with api.VHCI(g["input"], max_pert=ref["n_pert"] - 1) as v:
        v.hci()
        with pytest.raises(api.VhciError) as e:
            v.pt2()
        assert e.value.code == api.E_LIMIT and "max_pert" in str(e.value)
    summ, res = api.serve([(g["input"], 0.0)], slots=1, max_pert=ref["n_pert"] - 1)
    assert summ["failed"] == 1 and res[0]["status"] == api.E_LIMIT
    with api.VHCI(g["input"], max_basis=sizes[-1], max_pert=ref["n_pert"]) as v:
        v.hci()
        _, npert = v.pt2()
        assert v.n == ref["n_basis"] and npert == ref["n_pert"]   # limits at the size pass
