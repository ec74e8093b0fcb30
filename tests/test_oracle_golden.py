"""Pins the CPU oracle (oracle/) to the reference program's own outputs (tests/golden/, produced
by running the shipped reference binary; see tests/golden/make_golden.py), and checks that the
oracle's connection-driven forms equal its literal pair-loop forms bit for bit."""
import numpy as np
import pytest

from conftest import golden_cases, levels_of, load_golden
from oracle import oracle as O

FAST = ["clo2_vhci", "clo2_vhci_pt2", "clo2_vci", "syn_m6_pt2", "syn_m8_sextic_pt2",
        "syn_m5_cubic_pt2", "syn_m10_vci_pt2", "syn_m9_eps0_pt2"]


@pytest.mark.parametrize("case", FAST)
def test_oracle_matches_reference_outputs(case):
    g = load_golden(case)
    r = O.solve(g["input"])
    lev = levels_of(r.E)
    ref = np.array(g["levels"])
    assert np.abs(lev[:len(ref)] - ref).max() < 1e-6
    assert r.sizes == g["log"]["sizes"]
    assert r.n_pert == g["log"]["n_pert"]


@pytest.mark.slow
def test_oracle_matches_reference_workload0():
    g = load_golden("workload0")
    r = O.solve(g["input"])
    lev = levels_of(r.E)
    ref = np.array(g["levels"])
    assert np.abs(lev[:len(ref)] - ref).max() < 1e-6
    assert r.sizes == g["log"]["sizes"]


@pytest.mark.parametrize("case", ["syn_m6_pt2", "syn_m8_sextic_pt2", "syn_m5_cubic_pt2",
                                  "clo2_vhci_pt2"])
def test_connection_forms_equal_pair_forms(case):
    g = load_golden(case)
    o = O.Oracle(g["input"])
    w, C = np.linalg.eigh(o.dense_h())
    o.append_basis(o.select(C, min(o.neig, o.n), o.eps1))
    Hp = o.sparse_h("pairs").tocsr()
    Hc = o.sparse_h("conn").tocsr()
    # the pair loop also stores gated pairs with no connecting FC (structural zeros)
    Hp_nz = Hp.multiply(abs(Hp) > 0).tocsr()
    Hc_nz = Hc.multiply(abs(Hc) > 0).tocsr()
    assert (Hp_nz != Hc_nz).nnz == 0
    assert Hc.nnz <= Hp.nnz
    E, V = np.linalg.eigh(Hc.toarray())
    nopt = min(o.neig, o.n)
    d0, P0 = o.pt2(V, E, nopt, max(o.eps2, 0.05), "pairs")
    d1, P1 = o.pt2(V, E, nopt, max(o.eps2, 0.05), "conn")
    assert np.array_equal(P0, P1)
    assert np.array_equal(d0, d1)


def test_dense_equals_sparse_pairs():
    g = load_golden("clo2_vhci")
    o = O.Oracle(g["input"])
    D = o.dense_h()
    S = o.sparse_h("pairs").toarray()
    assert np.array_equal(D, S)


@pytest.mark.parametrize("p,n,d,expect", [
    (1, 0, 1, 1.0), (1, 3, 1, 2.0), (1, 3, -1, np.sqrt(3)), (2, 0, 0, 1.0), (2, 4, 0, 9.0),
    (2, 1, 2, np.sqrt(6)), (3, 0, 3, np.sqrt(6)), (4, 0, 0, 3.0), (4, 1, 0, 15.0),
])
def test_ladder_factors(p, n, d, expect):
    # <n+d| (a + a^dag)^p |n> against closed forms
    assert abs(O.ladder(p, n, d) - expect) < 1e-12 * max(1.0, expect)


def test_golden_fixture_inventory():
    names = golden_cases()
    for must in FAST + ["workload0"]:
        assert must in names
