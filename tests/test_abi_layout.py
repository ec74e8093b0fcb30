"""The ctypes mirrors in vhci_b200/api.py have exactly the C layout of include/vhci_gpu.h: size and
every field offset, checked against a small C program compiled with the header (CPU only)."""
import ctypes
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

STRUCTS = {"vhci_opts": "Opts", "vhci_problem": "Problem", "vhci_info": "Info",
           "vhci_stats": "Stats", "vhci_request": "Request", "vhci_serve_opts": "ServeOpts",
           "vhci_result": "Result", "vhci_serve_summary": "ServeSummary"}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    from vhci_b200 import api
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "vhci_gpu.h"', "int main(void) {"]
    for cname, pyname in STRUCTS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in getattr(api, pyname)._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("  return 0;\n}")
    d = tmp_path_factory.mktemp("abi")
    src = d / "layout.c"
    src.write_text("\n".join(lines))
    exe = d / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    lay = {}
    for ln in out.splitlines():
        s, f, v = ln.split()
        lay[(s, f)] = int(v)
    return lay


@pytest.mark.parametrize("cname", list(STRUCTS))
def test_ctypes_layout_matches_header(c_layout, cname):
    from vhci_b200 import api
    py = getattr(api, STRUCTS[cname])
    assert ctypes.sizeof(py) == c_layout[(cname, "size")]
    for fname, _ in py._fields_:
        assert getattr(py, fname).offset == c_layout[(cname, fname)], fname


def test_serving_requests_are_deterministic_and_admissible():
    """The serving stream's request generator: same request index, same PES and settings; the
    settings follow the stream's distributions; the PES passes the admissibility screen."""
    from vhci_b200 import pes as P
    for r in (2, 5):
        a, ra = P.serving_request(r)
        b, rb = P.serving_request(r)
        assert a.freqs == b.freqs and a.fcs == b.fcs and ra == rb
        assert 6 <= len(a.freqs) <= 24 and 10 <= ra.nstate <= 100
        assert 0.3 <= ra.eps1 <= 3.0 and ra.pt2 == 1 and abs(ra.eps2 - 0.1 * ra.eps1) < 1e-6
        assert P.admissible(a)
