"""Mixed precision (vhci_opts.precision = 1) against the FP64 path on the 44-mode, three-word-key
fixture: FP32 Hamiltonian values and FP32 vector gathers with FP64 accumulation in the
eigensolver's products, the Lanczos stopped at 1e-7, then an FP64 Rayleigh-Ritz sweep over the
Ritz block before every selection and before PT2; PT2 denominators and sums stay FP64.

Bars: the selected basis after every heat-bath iteration and |P| identical to the FP64 run, every
variational and PT2-corrected level within 0.01 cm^-1 of it, and the FP64 sweep's relative
residuals reported."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

CASE = os.path.join(GOLDEN, "syn_m44_w3", "input.inp")
TOL_CM = 0.01


def _run(precision):
    from vhci_b200 import api
    sizes = []
    with api.VHCI(CASE, precision=precision) as v:
        v.hci(callback=lambda it, n, zpe: sizes.append(n) if it > 0 else None)
        E_var = v.energies().copy()
        _, npert = v.pt2()
        return sizes, E_var, v.energies().copy(), npert, v.stats()


def test_mixed_precision_matches_fp64():
    s64, ev64, e64, p64, _ = _run(0)
    s32, ev32, e32, p32, st = _run(1)
    assert s32 == s64 and p32 == p64
    assert np.abs(ev32 - ev64).max() <= TOL_CM, np.abs(ev32 - ev64).max()
    assert np.abs(e32 - e64).max() <= TOL_CM, np.abs(e32 - e64).max()
    assert 0.0 < st["mixed_max_residual"] < 1e-6
