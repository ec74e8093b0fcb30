"""Generate the golden fixtures under tests/golden/ by running the reference VHCI program.

This script runs only where the reference tree (with its shipped `vhci` executable) is present;
its location is given with --reference PATH or the VHCI_REFERENCE environment variable.  The
executable is run as a black box in a scratch directory (`vhci -n <threads> -i case.inp -o freqs.dat`); its frequency file and the numbers
printed in its log are stored per case:

    tests/golden/<case>/input.inp    the input file (reference example or seeded synthetic PES)
    tests/golden/<case>/freqs.dat    the reference's frequency/assignment output
    tests/golden/<case>/log.json     basis size after each HCI iteration, perturber count,
                                     "% sparse" per Hamiltonian build, ZPE and wall time

The tests read these files only; they never need the reference tree.

Usage:  python tests/golden/make_golden.py --reference PATH [case ...]
"""
from __future__ import annotations

import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from vhci_b200 import pes as P  # noqa: E402

# location of the reference tree; set from --reference / VHCI_REFERENCE in main
REF = os.environ.get("VHCI_REFERENCE", "")
BIN = ""


def _example(mol, method, fname):
    return ("file", os.path.join("examples", mol, method, fname))


def _synthetic(spec, run, seed):
    return ("synthetic", spec, run, seed)


CASES = {
    # reference examples (their own known-answer fixtures)
    "clo2_vci": _example("CLO2", "VCI", "CLO2.inp"),
    "clo2_vhci": _example("CLO2", "VHCI", "CLO2.inp"),
    "clo2_vhci_pt2": _example("CLO2", "VHCI+PT2", "CLO2.inp"),
    "acetonitrile_vhci": _example("Acetonitrile", "VHCI", "acetonitrile.inp"),
    # seeded synthetic PESs
    "workload0": _synthetic(P.WORKLOADS[0][0], P.WORKLOADS[0][1], P.base_seed(0)),
    "syn_m6_pt2": _synthetic(P.PESSpec(6), P.RunSettings(0.5, 20, 1, 0.05), 101),
    "syn_m8_sextic_pt2": _synthetic(P.PESSpec(8, p5=0.05, p6=0.2), P.RunSettings(1.0, 15, 1, 0.1),
                                    102),
    "syn_m5_cubic_pt2": _synthetic(P.PESSpec(5, p4=0.0), P.RunSettings(0.5, 10, 1, 0.05), 103),
    "syn_m10_vci_pt2": _synthetic(P.PESSpec(10), P.RunSettings(0.0, 20, 1, 0.5, ntot=3), 104),
    "syn_m9_eps0_pt2": _synthetic(P.PESSpec(9), P.RunSettings(2.0, 12, 1, 0.0), 105),
    "syn_m12_pt2": _synthetic(P.PESSpec(12), P.RunSettings(2.0, 30, 1, 0.2), 106),
    "workload1_small": _synthetic(P.WORKLOADS[1][0], P.RunSettings(3.0, 50, 1, 0.3),
                                  P.base_seed(1)),
}


def parse_log(text: str) -> dict:
    sizes = [int(x) for x in re.findall(r"Basis size after iteration \d+ is: (\d+)", text)]
    sparse = [float(x) for x in re.findall(r"The Hamiltonian is ([0-9.]+)% sparse", text)]
    npert = re.findall(r"Perturbative space contains (\d+) states", text)
    init = re.findall(r"Initial basis size is: (\d+)", text)
    basis_fn = re.findall(r"Basis functions: (\d+)", text)
    conv = re.findall(r"contains (\d+) product states", text)
    return {
        "sizes": sizes,
        "sparse_percent": sparse,
        "n_pert": int(npert[0]) if npert else 0,
        "initial_basis": int(init[0]) if init else (int(basis_fn[0]) if basis_fn else None),
        "final_basis": int(conv[0]) if conv else (sizes[-1] if sizes else None),
    }


def run_case(name: str, threads: int = 8) -> None:
    spec = CASES[name]
    out = os.path.join(HERE, name)
    os.makedirs(out, exist_ok=True)
    inp = os.path.join(out, "input.inp")
    if spec[0] == "file":
        shutil.copyfile(os.path.join(REF, spec[1]), inp)
    else:
        _, pspec, run, seed = spec
        P.write_input(inp, P.generate(pspec, seed), run, comment=f"synthetic PES seed {seed}")
    with tempfile.TemporaryDirectory() as td:
        shutil.copyfile(inp, os.path.join(td, "case.inp"))
        t0 = time.time()
        r = subprocess.run([BIN, "-n", str(threads), "-i", "case.inp", "-o", "freqs.dat"], cwd=td,
                           capture_output=True, text=True)
        wall = time.time() - t0
        shutil.copyfile(os.path.join(td, "freqs.dat"), os.path.join(out, "freqs.dat"))
    info = parse_log(r.stdout)
    info["wall_s"] = round(wall, 2)
    info["threads"] = threads
    info["source"] = spec[0]
    with open(os.path.join(out, "log.json"), "w") as fh:
        json.dump(info, fh, indent=1)
    print(name, json.dumps(info))


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=REF, help="reference tree (default: $VHCI_REFERENCE)")
    ap.add_argument("cases", nargs="*")
    a = ap.parse_args()
    if not a.reference:
        sys.exit("give the reference tree with --reference PATH or VHCI_REFERENCE")
    REF = a.reference
    BIN = os.path.join(REF, "vhci")
    for n in a.cases or list(CASES):
        run_case(n)
