"""The incremental Hamiltonian build against a build from scratch.

Every heat-bath iteration of the reference rebuilds H over the whole basis (Ham.cpp:203-344, called
from HB.cpp:176-265).  Here the iterations after the first build only the rows of the states
added since, and take the new columns of the old rows from the new rows' entries (H is symmetric to
the bit).  After a complete heat-bath run, the stored matrix must equal, entry for entry and bit
for bit, the matrix a fresh context builds from scratch over the same final basis: the same
pattern, the same FP64 (or FP32) values, the same diagonal.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from vhci_b200 import api
    return api


def _scratch_csr(api, path, basis, precision):
    with api.VHCI(path, precision=precision) as w:
        w.set_basis(basis)
        w.build_h()
        assert w.stats()["hbuild_incremental"] == 0
        return w.h_csr()


@pytest.mark.parametrize("case,precision", [("workload0", 0), ("syn_m24_w2", 0),
                                            ("syn_m12_pt2", 1)])
def test_incremental_build_equals_scratch(api, case, precision):
    path = os.path.join(GOLDEN, case, "input.inp")
    with api.VHCI(path, precision=precision) as v:
        v.hci()
        assert v.stats()["hbuild_incremental"] >= 1, "no incremental build happened"
        H = v.h_csr()
        basis = v.basis()
    R = _scratch_csr(api, path, basis, precision)
    assert H.shape == R.shape
    assert np.array_equal(H.indptr, R.indptr)
    assert np.array_equal(H.indices, R.indices)
    assert np.array_equal(H.data, R.data)  # bit-identical values, diagonal included
