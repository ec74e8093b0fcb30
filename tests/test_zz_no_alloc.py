"""The no-allocation residual-norm entry point (vhci_residual_norms_noalloc).

It exists for callers that cannot allocate device memory when they need the check — a serving
process whose device memory belongs to its own pool, or code that must not trigger the implicit
device-wide synchronisation of cudaMalloc/cudaFree.  Its scratch is a fixed array in the library's
device memory, shared by every call.  This file is collected last so that a run stopping at the
first failure has already run every other test; it must also pass alone in a fresh process (the
first call on the device does the array's address set-up).
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_residual_norms_noalloc_matches_allocating_call():
    import torch
    from vhci_b200 import api
    g = load_golden("workload0")
    rng = np.random.default_rng(7)
    with api.VHCI(g["input"]) as v:
        v.build_h()
        n, k = v.n, 45
        X = rng.standard_normal((n, k))
        th = rng.uniform(1.0e4, 2.0e4, k)
        ref = v.residual_norms(X, th)  # the existing call: host buffers, allocates per call
        Xd = torch.tensor(X, dtype=torch.float64, device="cuda").contiguous()  # n x k row-major
        thd = torch.tensor(th, dtype=torch.float64, device="cuda")
        for _ in range(2):  # two calls in a row share (and reuse) the fixed scratch array
            rd = torch.full((k,), float("nan"), dtype=torch.float64, device="cuda")
            # the library's stream does not wait for torch's: the inputs must be complete first
            torch.cuda.synchronize()
            v.residual_norms_noalloc(Xd.data_ptr(), thd.data_ptr(), rd.data_ptr(), k)
            got = rd.cpu().numpy()
            assert np.allclose(got, ref, rtol=1e-12, atol=0), np.abs(got - ref).max()
        with pytest.raises(api.VhciError) as e:  # beyond the fixed array: a clear refusal
            v.residual_norms_noalloc(Xd.data_ptr(), thd.data_ptr(), rd.data_ptr(), 257)
        assert e.value.code == api.E_INPUT
        host = np.zeros(k)  # a host buffer is refused before anything runs on the device
        with pytest.raises(api.VhciError) as e:
            v.residual_norms_noalloc(Xd.data_ptr(), thd.data_ptr(), host.ctypes.data, k)
        assert e.value.code == api.E_INPUT
        assert torch.cuda.current_device() == 0
