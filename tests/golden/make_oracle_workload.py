"""Solve a benchmark workload with the CPU oracle (oracle/) and store the result as a fixture.

The reference program itself cannot finish these workloads in a practical time (its Hamiltonian
build and PT2 are pair-quadratic: about 2.7e12 pair evaluations for workload 1), so the full-size
parity fixture comes from the oracle, whose agreement with the reference is pinned separately by
tests/test_oracle_golden.py.  Output: tests/golden/workload<N>_oracle.json with the basis size
after each heat-bath iteration, the variational energies, the PT2 corrections and |P|.

Usage:  python tests/golden/make_oracle_workload.py 1        (several hours on 8 cores)
"""
from __future__ import annotations

import json
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from oracle import oracle as O  # noqa: E402
from vhci_b200 import pes as P  # noqa: E402


def main(workload: int) -> None:
    out = os.path.join(HERE, f"workload{workload}_oracle.json")
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "workload.inp")
        P.write_workload(path, workload)
        t0 = time.time()
        o = O.Oracle(path)
        w, C = np.linalg.eigh(o.dense_h())
        E, sizes, log = w, [], []
        while True:
            nopt = min(o.neig, o.n)
            new = o.select(C, nopt, o.eps1)
            if len(new) / o.n <= 0.01:
                break
            o.append_basis(new)
            sizes.append(o.n)
            H = o.sparse_h()
            E, C = O.sparse_eigs(H, o.neig)
            log.append({"n": o.n, "nnz": int(H.nnz), "E0": float(E[0]), "t": time.time() - t0})
            print(json.dumps(log[-1]), flush=True)
        res = {"workload": workload, "sizes": sizes, "E_var": [float(x) for x in E[:o.neig]],
               "log": log}
        if o.perturb:
            nopt = min(o.neig, o.n)
            dE, Pq = o.pt2(C, E, nopt, o.eps2)
            res["dE"] = [float(x) for x in dE]
            res["n_pert"] = int(len(Pq))
        res["wall_s"] = time.time() - t0
        res["threads"] = int(O.lib().orc_num_threads())
    with open(out, "w") as fh:
        json.dump(res, fh, indent=1)
    print("wrote", out, flush=True)


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 1)
