"""GPU parity on multi-word basis keys, wide PT2 and reproducible PT2 sums.

With 4 bits per mode one 64-bit key word holds 16 modes: the 24-mode case needs two words and the
44-mode case three (the 48-mode benchmark shape), and a 10-mode basis holding a state with more
than 15 quanta in one mode switches to 8-bit fields, i.e. two words.  Each is checked against the
CPU oracle with the same bars as the one-word fixtures (tests/test_gpu_parity.py):

  * selected state sets and Hamiltonian patterns bit-exact, Hamiltonian values within 1e-12
    relative (diagonal bit-exact), with the oracle's own vectors injected;
  * PT2 with injected vectors: the same |P|, corrections within 1e-9 relative;
  * end to end: the basis size after every heat-bath iteration and |P| equal to the oracle's,
    variational levels within 1e-4 cm^-1 and PT2-corrected levels within 1e-3 cm^-1.

PT2 for Nstate > 256 (the reference has no limit on N_opt = min(NEig, N), PT2.cpp:29-37) runs as
column tiles; its corrections are checked against the oracle.  PT2 orders each perturber row's
entries before summing, so two runs give bit-identical corrections.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MULTI = {"syn_m24_w2": 2, "syn_m44_w3": 3}
E_TOL = 1e-4
PT2_TOL = 1e-3


@pytest.fixture(scope="module")
def api():
    from vhci_b200 import api
    return api


def _input(case):
    return os.path.join(GOLDEN, case, "input.inp")


def _oracle_json(case):
    with open(os.path.join(GOLDEN, case, "oracle.json")) as fh:
        return json.load(fh)


def rows_sorted(q):
    q = np.asarray(q, np.int64)
    return q[np.lexsort(q.T[::-1])] if len(q) else q


def _first_selection(o):
    """Oracle state after the dense first step and one heat-bath selection."""
    w, C = np.linalg.eigh(o.dense_h())
    new = o.select(C, min(o.neig, o.n), o.eps1)
    return w, C, new


@pytest.mark.parametrize("case", sorted(MULTI))
def test_multiword_key_layout(api, case):
    with api.VHCI(_input(case)) as v:
        assert v.info.key_words == MULTI[case] and v.info.key_bits == 4


@pytest.mark.parametrize("case", sorted(MULTI))
def test_multiword_selection_injected_vectors(api, case):
    """Two heat-bath selections with the oracle's vectors: identical new-state sets."""
    o = O.Oracle(_input(case))
    w, C = np.linalg.eigh(o.dense_h())
    for it in range(2):
        nopt = min(o.neig, o.n)
        ref = o.select(C, nopt, o.eps1)
        with api.VHCI(_input(case)) as v:
            v.set_basis(o.basis().astype(np.uint8))
            k = min(C.shape[1], nopt)
            v.set_vectors(C[:, :k], w[:k])
            got = v.select(o.eps1)
        assert got.shape == ref.shape, (case, it, got.shape, ref.shape)
        assert np.array_equal(rows_sorted(got), rows_sorted(ref))
        o.append_basis(ref)
        w, C = O.sparse_eigs(o.sparse_h(), o.neig)


@pytest.mark.parametrize("case", sorted(MULTI))
def test_multiword_hamiltonian_matches_oracle(api, case):
    o = O.Oracle(_input(case))
    _, _, new = _first_selection(o)
    o.append_basis(new)
    Href = o.sparse_h().tocsr()
    with api.VHCI(_input(case)) as v:
        v.set_basis(o.basis().astype(np.uint8))
        Hg = v.h_csr().tocsr()
    Href.sort_indices()
    Hg.sort_indices()
    assert np.array_equal(Hg.indptr, Href.indptr)
    assert np.array_equal(Hg.indices, Href.indices)
    assert np.array_equal(Hg.diagonal(), Href.diagonal())
    d = np.abs(Hg.data - Href.data)
    assert np.all(d <= 1e-12 * np.abs(Href.data) + 1e-300), d.max()


@pytest.mark.parametrize("case", sorted(MULTI))
def test_multiword_pt2_injected_vectors(api, case):
    o = O.Oracle(_input(case))
    _, _, new = _first_selection(o)
    o.append_basis(new)
    E, C = O.sparse_eigs(o.sparse_h(), o.neig)
    nopt = min(o.neig, o.n)
    dE_ref, P_ref = o.pt2(C, E, nopt, o.eps2)
    with api.VHCI(_input(case)) as v:
        v.set_basis(o.basis().astype(np.uint8))
        v.set_vectors(C[:, :nopt], E[:nopt])
        dE, npert = v.pt2(o.eps2)
    assert npert == len(P_ref)
    assert np.allclose(dE, dE_ref, rtol=1e-9, atol=1e-12), np.abs(dE - dE_ref).max()


@pytest.mark.parametrize("case", sorted(MULTI))
def test_multiword_end_to_end_vs_oracle(api, case):
    ref = _oracle_json(case)
    sizes = []
    with api.VHCI(_input(case)) as v:
        v.hci(callback=lambda it, n, zpe: sizes.append(n) if it > 0 else None)
        n_basis = v.n
        E_var = v.energies().copy()
        dE, npert = v.pt2()
        E = v.energies().copy()
    assert sizes == ref["sizes"]
    assert n_basis == ref["final_basis"] and npert == ref["n_pert"]
    k = len(ref["E_var"])
    assert np.abs(E_var[:k] - np.array(ref["E_var"])).max() <= E_TOL
    assert np.abs(E[:k] - np.array(ref["E"])).max() <= PT2_TOL


def _with_high_quanta(o):
    """The initial basis plus one state with 16 quanta in mode 0 (needs 8-bit fields)."""
    q = o.basis()
    extra = np.zeros((1, o.nm), np.int32)
    extra[0, 0] = 16
    return np.vstack([q, extra])


def test_eight_bit_two_word_layout_matches_oracle(api):
    """10 modes with a 16-quanta state: 8-bit fields over two words.  Selection, Hamiltonian and
    PT2 with injected vectors against the oracle."""
    g = load_golden("syn_m10_vci_pt2")
    o = O.Oracle(g["input"])
    o.set_basis(_with_high_quanta(o))
    H0 = o.sparse_h().toarray()
    w, C = np.linalg.eigh(H0)
    nopt = min(o.neig, o.n)
    eps = 0.5
    ref_sel = o.select(C, nopt, eps)
    with api.VHCI(g["input"]) as v:
        v.set_basis(o.basis().astype(np.uint8))
        assert v.info.key_bits == 8 and v.info.key_words == 2
        Hg = v.h_csr().toarray()
        assert np.array_equal(Hg != 0, H0 != 0)
        assert np.array_equal(np.diag(Hg), np.diag(H0))
        assert np.allclose(Hg, H0, rtol=1e-12, atol=0)
        v.set_vectors(C[:, :nopt], w[:nopt])
        got = v.select(eps)
        assert np.array_equal(rows_sorted(got), rows_sorted(ref_sel))
        dE, npert = v.pt2(o.eps2)
    dE_ref, P_ref = o.pt2(C, w, nopt, o.eps2)
    assert npert == len(P_ref)
    assert np.allclose(dE, dE_ref, rtol=1e-9, atol=1e-12), np.abs(dE - dE_ref).max()


def test_pt2_more_than_256_states(api, tmp_path):
    """Nstate = 300 (two column tiles in the EN reduction) against the oracle."""
    g = load_golden("syn_m10_vci_pt2")
    lines = open(g["input"]).read().splitlines()
    assert lines[2].split()[0].startswith(("Nstate", "HBOptimization"))
    lines[2] = lines[2].split()[0] + " 300"
    path = str(tmp_path / "wide.inp")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    o = O.Oracle(path)
    assert o.neig == 300
    o.append_basis(o.select(np.linalg.eigh(o.dense_h())[1], min(o.neig, o.n), 0.5))
    w, C = np.linalg.eigh(o.sparse_h().toarray())
    nopt = 300
    dE_ref, P_ref = o.pt2(C, w, nopt, o.eps2)
    with api.VHCI(path) as v:
        v.set_basis(o.basis().astype(np.uint8))
        v.set_vectors(C[:, :nopt], w[:nopt])
        dE, npert = v.pt2(o.eps2)
    assert len(dE) == 300 and npert == len(P_ref)
    assert np.allclose(dE, dE_ref, rtol=1e-9, atol=1e-12), np.abs(dE - dE_ref).max()


def test_pt2_is_bit_reproducible(api):
    """Two PT2 runs over the same vectors give bit-identical corrections (rows are summed in one
    fixed entry order whatever order the fill pass produced)."""
    o = O.Oracle(_input("syn_m24_w2"))
    _, _, new = _first_selection(o)
    o.append_basis(new)
    E, C = O.sparse_eigs(o.sparse_h(), o.neig)
    nopt = min(o.neig, o.n)
    out = []
    for _ in range(2):
        with api.VHCI(_input("syn_m24_w2")) as v:
            v.set_basis(o.basis().astype(np.uint8))
            v.set_vectors(C[:, :nopt], E[:nopt])
            out.append(v.pt2(o.eps2)[0])
    assert np.array_equal(out[0], out[1])
