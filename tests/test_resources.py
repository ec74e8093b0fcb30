"""Device resources across many contexts: every buffer a context allocates (column panels,
segment tables, gate-pattern tables included) goes back to the stream-ordered pool on destroy, and
pooled library handles are reused."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _pool_used(device=0):
    from cuda.bindings import runtime as cudart
    err, pool = cudart.cudaDeviceGetDefaultMemPool(device)
    assert int(err) == 0
    err, used = cudart.cudaMemPoolGetAttribute(
        pool, cudart.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
    assert int(err) == 0
    return int(used)


def test_no_device_memory_left_after_destroy(monkeypatch):
    from vhci_b200 import api
    g = load_golden("syn_m8_sextic_pt2")
    monkeypatch.setenv("VHCI_PANEL_MB", "0.03")       # build column panels too
    first = api.solve(g["input"])                       # warm: module, pooled handles
    base = _pool_used()
    for _ in range(3):
        with api.VHCI(g["input"]) as v:
            v.hci()
            v.pt2()
            v.structural_nnz()
            E = v.energies().copy()
        assert np.array_equal(E, first["E"])
    assert _pool_used() == base
