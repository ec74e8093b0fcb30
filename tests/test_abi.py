"""The C-ABI library loads without a GPU and exports every function include/vhci_gpu.h declares;
without a device it refuses to run (there is no CPU path)."""
import os
import re

import pytest

from conftest import ROOT


def header_functions():
    src = open(os.path.join(ROOT, "include", "vhci_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(vhci_[a-z_0-9]+)\s*\(", src)) - {"vhci_iter_cb"})


def test_library_exports_every_declared_symbol():
    from vhci_b200 import api
    L = api.lib()
    names = header_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
    assert sorted(api.EXPORTS) == names


def test_no_cpu_fallback_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from vhci_b200 import api
    with pytest.raises(api.VhciError) as e:
        api.VHCI(os.path.join(ROOT, "tests", "golden", "clo2_vhci", "input.inp"))
    assert e.value.code == api.E_CUDA
