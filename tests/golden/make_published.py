"""Collect the reference project's published result files as golden fixtures.

The reference tree ships real-molecule inputs (`input/<mol>.inp`) and the frequency files its
authors obtained from them (`results/freq_<mol>_eps1-<e1>_nstate-<k>_perturb-<p>_eps2-<e2>_
nmax-<cap>_ntot-<ntot>.dat`).  The run parameters of each result are in its file name; several
inputs carry other header values (e.g. naphthalene's has HCI_Eps 0, Max_quanta 3), so a test
rewrites the header from the parameters before solving.  This script copies, for the selected
molecules, the input once and every matching result file:

    tests/golden/published/<mol>.inp
    tests/golden/published/<result file name>.dat
    tests/golden/published/index.json     result name -> molecule and run parameters

Nothing is run.  The tests read only these files.

Usage:  python tests/golden/make_published.py --reference PATH      (or VHCI_REFERENCE=PATH)
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "published")

# Molecules taken: naphthalene (48 modes: three 64-bit key words), ethylene oxide (15 modes,
# the reference's own largest logged run), C2H4 with sextic terms and its quartic variant.
# Acetonitrile has degenerate mode pairs, so its selected basis depends on the eigensolver's
# rotation of degenerate eigenvectors; it is left out of the level-by-level comparison.
MOLECULES = ("naphthalene", "ethylene_oxide", "C2H4", "C2H4_quartic")

NAME = re.compile(r"^freq_(?P<mol>.+)_eps1-(?P<e1>[0-9.]+)_nstate-(?P<k>\d+)_perturb-(?P<p>[01])"
                  r"_eps2-(?P<e2>[0-9.]+)_nmax-(?P<cap>\d+)_ntot-(?P<ntot>\d+)\.dat$")


def parse_name(fname: str) -> dict | None:
    m = NAME.match(fname)
    if not m:
        return None
    return {"molecule": m["mol"], "eps1": float(m["e1"]), "nstate": int(m["k"]),
            "pt2": int(m["p"]), "eps2": float(m["e2"]), "cap": int(m["cap"]),
            "ntot": int(m["ntot"])}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("VHCI_REFERENCE", ""))
    a = ap.parse_args()
    if not a.reference:
        sys.exit("give the reference tree with --reference PATH or VHCI_REFERENCE")
    os.makedirs(OUT, exist_ok=True)
    index = {}
    for fname in sorted(os.listdir(os.path.join(a.reference, "results"))):
        meta = parse_name(fname)
        if not meta or meta["molecule"] not in MOLECULES:
            continue
        shutil.copyfile(os.path.join(a.reference, "results", fname), os.path.join(OUT, fname))
        index[fname[:-4]] = meta
    for mol in sorted({m["molecule"] for m in index.values()}):
        shutil.copyfile(os.path.join(a.reference, "input", mol + ".inp"),
                        os.path.join(OUT, mol + ".inp"))
    with open(os.path.join(OUT, "index.json"), "w") as fh:
        json.dump(index, fh, indent=1, sort_keys=True)
    print(f"{len(index)} result files for {sorted({m['molecule'] for m in index.values()})}")


if __name__ == "__main__":
    main()
