"""Checkpoint files (reference: WriteCheckpoint / ReadCheckpoint, src/Core_functions.cpp:94-167):
the written layout, validation on read, and restart of the heat-bath procedure from a checkpoint
written part-way (src/VHCI.cpp:39-48, src/HB.cpp:180)."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from vhci_b200 import api
    return api


def read_reference_layout(path, nm, neig):
    """Reads a checkpoint the way the reference does: 'N M NEig', M frequencies, NEig eigenvalues,
    then N rows of M quanta and NEig coefficients."""
    tok = open(path).read().split()
    n, m, k = int(tok[0]), int(tok[1]), int(tok[2])
    assert (m, k) == (nm, neig)
    p = 3
    freqs = np.array(tok[p:p + m], float); p += m
    E = np.array(tok[p:p + k], float); p += k
    rows = np.array(tok[p:], float).reshape(n, m + k)
    return freqs, E, rows[:, :m].astype(int), rows[:, m:]


def test_checkpoint_layout(api, tmp_path):
    g = load_golden("syn_m6_pt2")
    path = str(tmp_path / "ck.txt")
    with api.VHCI(g["input"]) as v:
        v.hci()
        v.write_checkpoint(path)
        C, E = v.vectors(v.info.nstate)
        q = v.basis()
        f = v.freqs()
    freqs, Ek, quanta, coeffs = read_reference_layout(path, len(f), len(E))
    assert np.array_equal(freqs, f)
    assert np.array_equal(quanta, q.astype(int))
    assert np.allclose(Ek, E, rtol=0, atol=1e-12)
    assert np.allclose(coeffs, C, rtol=0, atol=1e-15)
    first = open(path).readline().split()
    assert first == [str(len(q)), str(len(f)), str(len(E))]
    assert "%.17f " % f[0] in open(path).read()


def test_restart_from_midway_checkpoint(api, tmp_path):
    """One heat-bath iteration, checkpoint, then restart: same final result as one uninterrupted
    run."""
    g = load_golden("syn_m8_sextic_pt2")
    ref = api.solve(g["input"])
    path = str(tmp_path / "mid.txt")
    with api.VHCI(g["input"]) as v:
        k = v.info.nstate
        v.eigs(k)                       # dense first step over the initial basis
        v.select(v.info.eps1, append=True)
        v.build_h()
        v.eigs(k)
        v.write_checkpoint(path)
    with api.VHCI(g["input"], restart=True) as v:
        assert v.n == 1                 # restart builds only the ground state before reading
        v.read_checkpoint(path)
        v.hci()
        dE, npert = v.pt2()
        E = v.energies()
        n = v.n
    assert n == ref["n_basis"]
    assert npert == ref["n_pert"]
    assert np.abs(E - ref["E"][:len(E)]).max() < 1e-6


def test_checkpoint_validation(api, tmp_path):
    g = load_golden("syn_m6_pt2")
    good = str(tmp_path / "ck.txt")
    with api.VHCI(g["input"]) as v:
        v.hci()
        v.write_checkpoint(good)
    txt = open(good).read().split("\n")
    head = txt[0].split()
    bad_modes = str(tmp_path / "bad1.txt")
    open(bad_modes, "w").write("\n".join([f"{head[0]} {int(head[1]) + 1} {head[2]}"] + txt[1:]))
    bad_freq = str(tmp_path / "bad2.txt")
    f = txt[1].split()
    f[0] = "%.17f" % (float(f[0]) + 1e-6)
    open(bad_freq, "w").write("\n".join([txt[0], " ".join(f) + " "] + txt[2:]))
    for p, msg in [(bad_modes, "wrong number of fundamental modes"),
                   (bad_freq, "wrong fundamental frequencies")]:
        with api.VHCI(g["input"], restart=True) as v:
            with pytest.raises(api.VhciError) as e:
                v.read_checkpoint(p)
            assert msg in str(e.value)


def test_checkpoint_text_is_byte_identical_to_printf(api, tmp_path):
    """The parallel writer produces exactly the reference's text: 'N M NEig', then '%.17f '
    fields (Core_functions.cpp:94-117), checked against Python's correctly rounded formatting;
    and the parallel reader restores the same basis and vectors."""
    g = load_golden("syn_m9_eps0_pt2")
    path = str(tmp_path / "ck.txt")
    with api.VHCI(g["input"], host_threads=7) as v:
        v.hci()
        v.write_checkpoint(path)
        k = v.info.nstate
        C, E = v.vectors(k)
        q = v.basis().astype(int)
        f = v.freqs()
    n, nm = q.shape
    want = [f"{n} {nm} {k}\n", "".join("%.17f " % x for x in f) + "".join("%.17f " % x for x in E) + "\n"]
    for i in range(n):
        want.append("".join("%d " % x for x in q[i]) + "".join("%.17f " % x for x in C[i]) + "\n")
    assert open(path).read() == "".join(want)
    with api.VHCI(g["input"], restart=True, host_threads=5) as v:
        v.read_checkpoint(path)
        C2, E2 = v.vectors(k)
        assert np.array_equal(v.basis().astype(int), q)
    C_txt = np.array([[float("%.17f" % x) for x in row] for row in C])
    assert np.array_equal(C2, C_txt)
    assert np.array_equal(E2, np.array([float("%.17f" % x) for x in E]))
