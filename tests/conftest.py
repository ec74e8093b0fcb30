import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running case")


def golden_cases():
    out = []
    for name in sorted(os.listdir(GOLDEN)):
        d = os.path.join(GOLDEN, name)
        if os.path.isdir(d) and os.path.exists(os.path.join(d, "log.json")):
            out.append(name)
    return out


def load_golden(name):
    d = os.path.join(GOLDEN, name)
    with open(os.path.join(d, "log.json")) as fh:
        log = json.load(fh)
    freqs = [l.split("   ", 1) for l in open(os.path.join(d, "freqs.dat")).read().splitlines()]
    energies = [float(f[0]) for f in freqs]
    assigns = [f[1] if len(f) > 1 else "" for f in freqs]
    return {"input": os.path.join(d, "input.inp"), "log": log, "levels": energies,
            "assign": assigns, "dir": d}


def levels_of(E):
    """Reference output convention: E_0, then E_n - E_0."""
    import numpy as np
    E = np.asarray(E, float)
    return np.r_[E[0], E[1:] - E[0]]
