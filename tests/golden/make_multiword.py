"""Seeded synthetic PESs whose basis keys span two and three 64-bit words, solved by the oracle.

With 4 bits per mode a key word holds 16 modes, so 17-32 modes need two words and 33-48 three.
Every reference example and the other synthetic fixtures have at most 15 modes (one word); these
two cases exercise the multi-word key paths (selection, Hamiltonian build, PT2) against the CPU
oracle at sizes the oracle solves in under a minute:

    tests/golden/<case>/input.inp     the input file (reference format)
    tests/golden/<case>/oracle.json   the oracle's full solve: basis size after each heat-bath
                                      iteration, variational energies, PT2 corrections, |P|

The oracle's agreement with the reference program is pinned separately (tests/test_oracle_golden.py).

Usage:  python tests/golden/make_multiword.py [case ...]
"""
from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from vhci_b200 import pes as P  # noqa: E402

# (spec, run settings, seed): value ranges narrower than the benchmark generator's so the sparse
# force fields stay bound without the admissibility search
CASES = {
    "syn_m24_w2": (P.PESSpec(24, p3=0.15, p4=0.03, r3=(0.0, 2.0), r4=(-1.0, 1.0)),
                   P.RunSettings(eps1=0.5, nstate=60, pt2=1, eps2=0.1), 31004),
    "syn_m44_w3": (P.PESSpec(44, p3=0.04, p4=0.004, r3=(0.0, 2.0), r4=(-1.0, 1.0)),
                   P.RunSettings(eps1=0.5, nstate=40, pt2=1, eps2=0.2), 31003),
}


def run_case(name: str) -> None:
    spec, run, seed = CASES[name]
    out = os.path.join(HERE, name)
    os.makedirs(out, exist_ok=True)
    inp = os.path.join(out, "input.inp")
    P.write_input(inp, P.generate(spec, seed), run, comment=f"synthetic PES seed {seed}")
    t0 = time.time()
    r = O.solve(inp)
    info = {
        "sizes": [int(x) for x in r.sizes],
        "final_basis": int(len(r.basis)),
        "n_pert": int(r.n_pert),
        "E_var": [float(x) for x in r.E_var],
        "dE": [float(x) for x in r.dE] if r.dE is not None else [],
        "E": [float(x) for x in r.E],
        "oracle_s": round(time.time() - t0, 1),
    }
    with open(os.path.join(out, "oracle.json"), "w") as fh:
        json.dump(info, fh, indent=1)
    print(name, info["sizes"], info["n_pert"], info["oracle_s"])


if __name__ == "__main__":
    for n in sys.argv[1:] or list(CASES):
        run_case(n)
