"""Host-side tables on the CPU (vhci_b200/csrc/model.cpp built with g++ through tests/host/
model_shim.cpp): the connection groups and the reference's pair-gate patterns are ordered by
lowered-mode key with a correct segment index, and the gate patterns are exactly the change
vectors the reference's gates admit (|delta|_1 = s, s even <= fcmax or odd <= fcmax - 1)."""
import ctypes
import os
import shutil
import subprocess

import pytest

from conftest import ROOT, load_golden


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    d = tmp_path_factory.mktemp("shim")
    so = d / "libmodelshim.so"
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC",
                    "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "vhci_b200", "csrc"),
                    os.path.join(ROOT, "tests", "host", "model_shim.cpp"),
                    os.path.join(ROOT, "vhci_b200", "csrc", "model.cpp"),
                    "-o", str(so)], check=True)
    L = ctypes.CDLL(str(so))
    L.shim_load.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_longlong]
    for f in ("shim_ngroups", "shim_nseg", "shim_seg_begin"):
        getattr(L, f).restype = ctypes.c_longlong
    L.shim_seg_begin.argtypes = [ctypes.c_longlong]
    L.shim_seg_key.restype = ctypes.c_ulonglong
    L.shim_seg_key.argtypes = [ctypes.c_longlong]
    L.shim_group.argtypes = [ctypes.c_longlong, ctypes.POINTER(ctypes.c_int)]
    L.shim_lowered_key.restype = ctypes.c_ulonglong
    L.shim_lowered_key.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    return L


def _groups(L):
    out = (ctypes.c_int * 12)()
    res = []
    for u in range(L.shim_ngroups()):
        k = L.shim_group(u, out)
        res.append(tuple((out[2 * i], out[2 * i + 1]) for i in range(k)))
    return res


def _key(L, g):
    low = [m for m, d in g if d < 0]
    arr = (ctypes.c_int * max(1, len(low)))(*low)
    return L.shim_lowered_key(len(low), arr)


def _check_segments(L, groups):
    keys = [_key(L, g) for g in groups]
    assert keys == sorted(keys)                       # ordered by lowered-mode key
    nseg = L.shim_nseg()
    assert nseg == len(set(keys))
    for s in range(nseg):
        b, e = L.shim_seg_begin(s), L.shim_seg_begin(s + 1)
        assert b < e and all(keys[u] == L.shim_seg_key(s) for u in range(b, e))
    assert L.shim_seg_begin(nseg) == len(groups)
    assert L.shim_max_lowered() == max(sum(d < 0 for _, d in g) for g in groups)


@pytest.mark.parametrize("case", ["syn_m8_sextic_pt2", "syn_m5_cubic_pt2", "clo2_vhci"])
def test_connection_groups_segment_index(shim, case):
    assert shim.shim_load(load_golden(case)["input"].encode(), 0, 0) == 0
    groups = _groups(shim)
    assert len(groups) == len(set(groups))            # one group per change vector
    assert all(all(d != 0 for _, d in g) for g in groups)
    _check_segments(shim, groups)


@pytest.mark.parametrize("case", ["syn_m8_sextic_pt2", "syn_m5_cubic_pt2", "clo2_vhci"])
def test_gate_patterns_are_the_admitted_change_vectors(shim, case):
    assert shim.shim_load(load_golden(case)["input"].encode(), 1, 2_000_000) == 0
    nm, fcmax = shim.shim_nm(), shim.shim_fcmax()
    got = _groups(shim)
    want = set()

    def walk(m, rem, vec):                            # every vector with |d|_1 <= fcmax
        if m == nm:
            s = sum(abs(x) for _, x in vec)
            if s and ((s % 2 == 0 and s <= fcmax) or (s % 2 == 1 and s <= fcmax - 1)):
                want.add(tuple(vec))
            return
        for x in range(-rem, rem + 1):
            walk(m + 1, rem - abs(x), vec + [(m, x)] if x else vec)

    walk(0, fcmax, [])
    assert len(got) == len(set(got)) and set(got) == want
    _check_segments(shim, got)


def test_subset_walk_visits_exactly_the_applicable_groups(shim):
    """The device enumerator's walk (for_each_group in csrc/conn.cuh), restated: subsets of a
    state's excited modes of size 0..max lowered, unranked in the combinatorial number system, each
    looked up by its lowered-mode key in the segment index. It must visit every group whose lowered
    modes are all excited, once, and nothing else."""
    from math import comb
    import numpy as np
    assert shim.shim_load(load_golden("syn_m8_sextic_pt2")["input"].encode(), 0, 0) == 0
    nm = shim.shim_nm()
    groups = _groups(shim)
    seg = {shim.shim_seg_key(s): (shim.shim_seg_begin(s), shim.shim_seg_begin(s + 1))
           for s in range(shim.shim_nseg())}
    maxl = shim.shim_max_lowered()
    rng = np.random.default_rng(7)
    for _ in range(200):
        q = np.zeros(nm, int)
        k = int(rng.integers(0, nm + 1))
        q[rng.choice(nm, k, replace=False)] = rng.integers(1, 4, k)
        exc = [m for m in range(nm) if q[m] > 0]
        e = len(exc)
        nsub = sum(comb(e, r) for r in range(min(maxl, e) + 1))
        seen = []
        for s in range(nsub):
            r, rem = 0, s
            while rem >= comb(e, r):
                rem -= comb(e, r)
                r += 1
            modes, hi = [0] * r, e
            for i in range(r, 0, -1):        # largest c < hi with C(c, i) <= rem
                c = hi - 1
                while comb(c, i) > rem:
                    c -= 1
                rem -= comb(c, i)
                modes[i - 1] = exc[c]
                hi = c
            arr = (ctypes.c_int * max(1, r))(*modes)
            key = shim.shim_lowered_key(r, arr)
            if key in seg:
                seen.extend(range(*seg[key]))
        want = [u for u, g in enumerate(groups) if all(q[m] > 0 for m, d in g if d < 0)]
        assert len(seen) == len(set(seen)) and sorted(seen) == want
