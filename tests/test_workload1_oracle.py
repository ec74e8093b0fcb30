"""Workload 1 at full size (Nm 15, HCI_Eps 0.5, Nstate 200, PT2_Eps 0.01: 380,418 states,
6,583,465 perturbers) against the CPU oracle's solve of the same input
(tests/golden/workload1_oracle.json, made by tests/golden/make_oracle_workload.py; the oracle's
agreement with the reference program is pinned by test_oracle_golden.py).  Basis size after every
heat-bath iteration and |P| must be equal; variational energies within 1e-4 cm^-1 and PT2
corrections within 1e-3 cm^-1 (the path's FP64 tolerances)."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(ROOT, "tests", "golden", "workload1_oracle.json")


def test_workload1_full_size_matches_oracle(tmp_path):
    from vhci_b200 import api, pes
    ref = json.load(open(FIXTURE))
    path = str(tmp_path / "w1.inp")
    pes.write_workload(path, 1)
    sizes = []
    with api.VHCI(path) as v:
        v.hci(callback=lambda it, n, zpe: sizes.append(n))
        E_var = v.energies().copy()
        dE, npert = v.pt2()
    assert sizes[1:] == ref["sizes"]
    assert npert == ref["n_pert"]
    k = len(ref["E_var"])
    assert np.abs(E_var[:k] - np.array(ref["E_var"])).max() <= 1e-4
    assert np.abs(np.asarray(dE)[:k] - np.array(ref["dE"])).max() <= 1e-3
