"""vhci_b200: heat-bath VCI + Epstein-Nesbet PT2 on NVIDIA B200 (sm_100a).

The compute path is the C ABI library `libvhci_gpu.so` (include/vhci_gpu.h); `vhci_b200.api`
binds it for Python, `vhci_b200.pes` writes seeded synthetic input files, and `bin/vhci` is the
drop-in command-line tool.
"""
from .api import VHCI, VhciError, solve  # noqa: F401
