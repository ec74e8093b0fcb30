"""CPU ORACLE driver — test infrastructure only (never part of the product path).

Loads the C++ restatement in oracle/oracle.cpp (built into oracle/_build/liboracle.so by
oracle/Makefile) and runs the reference's full VHCI(+PT2) procedure with LAPACK/ARPACK
eigen-steps through numpy/scipy:

* `src/HB.cpp:176-265` (Perform_HCI): dense first step over the initial basis
  (`Eigen::SelfAdjointEigenSolver` there, LAPACK `syevd` here), then heat-bath iterations until
  the basis grows by at most 1 %, each followed by a sparse eigensolve;
* `src/Ham.cpp:347-370` (SparseDiagonalize): implicitly restarted Lanczos for the `Nstate` smallest
  eigenvalues, ncv = max(2*Nstate+1, 20), tolerance 1e-10 (Spectra there, ARPACK here);
* `src/VHCI.cpp:49-76` (HCI_Eps == 0): one sparse eigensolve over the initial basis;
* `src/PT2.cpp:16-154` (DoPT2): Epstein-Nesbet correction over the eps2-screened perturber space.

Parity of this driver with the reference itself is pinned by tests/test_oracle_golden.py against
outputs of the shipped reference binary stored under tests/golden/.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, i64, i32p, dp, i64p = (ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int32),
                                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64))
        L.orc_load.restype = vp
        L.orc_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
        L.orc_free.argtypes = [vp]
        L.orc_info.argtypes = [vp, i64p, dp]
        L.orc_freqs.argtypes = [vp, dp]
        L.orc_hb_list.argtypes = [vp, dp, i32p, i32p]
        L.orc_fc_list.argtypes = [vp, dp, i32p, i32p]
        L.orc_basis_size.restype = i64
        L.orc_basis_size.argtypes = [vp]
        L.orc_get_basis.argtypes = [vp, i32p]
        L.orc_set_basis.argtypes = [vp, i32p, i64]
        L.orc_append_basis.argtypes = [vp, i32p, i64]
        L.orc_select.restype = i64
        L.orc_select.argtypes = [vp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.orc_get_selected.argtypes = [vp, i32p]
        L.orc_dense_h.argtypes = [vp, dp]
        L.orc_build_h_pairs.restype = i64
        L.orc_build_h_pairs.argtypes = [vp]
        L.orc_build_h_conn.restype = i64
        L.orc_build_h_conn.argtypes = [vp]
        L.orc_get_csr.argtypes = [vp, i64p, i32p, dp]
        L.orc_pt2.restype = i64
        L.orc_pt2.argtypes = [vp, dp, ctypes.c_int, dp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                              dp]
        L.orc_pair_rows.restype = i64
        L.orc_pair_rows.argtypes = [vp, i64, i64, i64, dp]
        L.orc_ladder.restype = ctypes.c_double
        L.orc_ladder.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


class Oracle:
    """One parsed input file plus the current basis (the reference's global state)."""

    def __init__(self, path: str):
        L = lib()
        err = ctypes.create_string_buffer(256)
        self.h = L.orc_load(path.encode(), err, 256)
        if not self.h:
            raise ValueError(err.value.decode())
        info = np.zeros(8, np.int64)
        dinfo = np.zeros(2, np.float64)
        L.orc_info(self.h, _p(info, ctypes.c_int64), _p(dinfo, ctypes.c_double))
        (self.nm, self.ntot, self.neig, self.perturb, _, self.nfc, self.nhb, self.fcmax) = map(
            int, info)
        self.eps1, self.eps2 = float(dinfo[0]), float(dinfo[1])
        self.freqs = np.zeros(self.nm)
        L.orc_freqs(self.h, _p(self.freqs, ctypes.c_double))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_free(self.h)
            self.h = None

    # ---- basis ----
    @property
    def n(self) -> int:
        return int(lib().orc_basis_size(self.h))

    def basis(self) -> np.ndarray:
        q = np.zeros((self.n, self.nm), np.int32)
        lib().orc_get_basis(self.h, _p(q, ctypes.c_int32))
        return q

    def set_basis(self, q: np.ndarray) -> None:
        q = np.ascontiguousarray(q, np.int32)
        lib().orc_set_basis(self.h, _p(q, ctypes.c_int32), q.shape[0])

    def append_basis(self, q: np.ndarray) -> None:
        q = np.ascontiguousarray(q, np.int32)
        lib().orc_append_basis(self.h, _p(q, ctypes.c_int32), q.shape[0])

    def hb_list(self):
        fc = np.zeros(self.nhb)
        modes = np.zeros((self.nhb, 6), np.int32)
        powers = np.zeros((self.nhb, 6), np.int32)
        lib().orc_hb_list(self.h, _p(fc, ctypes.c_double), _p(modes, ctypes.c_int32),
                          _p(powers, ctypes.c_int32))
        return fc, modes, powers

    def fc_list(self):
        fc = np.zeros(self.nfc)
        modes = np.zeros((self.nfc, 6), np.int32)
        powers = np.zeros((self.nfc, 6), np.int32)
        lib().orc_fc_list(self.h, _p(fc, ctypes.c_double), _p(modes, ctypes.c_int32),
                          _p(powers, ctypes.c_int32))
        return fc, modes, powers

    # ---- kernels ----
    def select(self, C: np.ndarray, nopt: int, eps: float) -> np.ndarray:
        C = np.asfortranarray(C, np.float64)
        assert C.shape[0] == self.n
        cnt = lib().orc_select(self.h, _p(C, ctypes.c_double), C.shape[1], nopt, eps)
        q = np.zeros((cnt, self.nm), np.int32)
        lib().orc_get_selected(self.h, _p(q, ctypes.c_int32))
        return q

    def dense_h(self) -> np.ndarray:
        H = np.zeros((self.n, self.n))
        lib().orc_dense_h(self.h, _p(H, ctypes.c_double))
        return H

    def sparse_h(self, mode: str = "conn"):
        import scipy.sparse as sp
        n = self.n
        nnz = (lib().orc_build_h_pairs(self.h) if mode == "pairs" else
               lib().orc_build_h_conn(self.h))
        rowptr = np.zeros(n + 1, np.int64)
        col = np.zeros(nnz, np.int32)
        val = np.zeros(nnz)
        lib().orc_get_csr(self.h, _p(rowptr, ctypes.c_int64), _p(col, ctypes.c_int32),
                          _p(val, ctypes.c_double))
        return sp.csr_matrix((val, col, rowptr), shape=(n, n))

    def pt2(self, C: np.ndarray, E: np.ndarray, nopt: int, eps2: float, mode: str = "conn"):
        C = np.asfortranarray(C, np.float64)
        E = np.ascontiguousarray(E, np.float64)
        dE = np.zeros(nopt)
        npert = lib().orc_pt2(self.h, _p(C, ctypes.c_double), C.shape[1], _p(E, ctypes.c_double),
                              nopt, eps2, 0 if mode == "pairs" else 1, _p(dE, ctypes.c_double))
        q = np.zeros((npert, self.nm), np.int32)
        lib().orc_get_selected(self.h, _p(q, ctypes.c_int32))
        return dE, q


def pair_rows(o: "Oracle", r0: int, r1: int, stride: int):
    """Reference pair loop over rows r0, r0+stride, ... < r1 against all j >= i; returns
    (pairs evaluated, checksum)."""
    cs = ctypes.c_double()
    n = lib().orc_pair_rows(o.h, r0, r1, stride, ctypes.byref(cs))
    return int(n), cs.value


def ladder(p: int, n: int, delta: int) -> float:
    return float(lib().orc_ladder(p, n, delta))


def sparse_eigs(H, k: int, tol: float = 1e-10):
    """Lowest k eigenpairs, implicitly restarted Lanczos as src/Ham.cpp:347-370."""
    import scipy.sparse.linalg as sla
    n = H.shape[0]
    ncv = max(2 * k + 1, 20)
    if k >= n - 1 or ncv > n:
        w, v = np.linalg.eigh(H.toarray())
        return w[:k], v[:, :k]
    v0 = np.random.Generator(np.random.PCG64(12345)).standard_normal(n)
    w, v = sla.eigsh(H, k=k, which="SA", tol=tol, ncv=ncv, maxiter=1000 * n, v0=v0)
    o = np.argsort(w)
    return w[o], v[:, o]


@dataclass
class Result:
    E: np.ndarray
    C: np.ndarray
    basis: np.ndarray
    sizes: list = field(default_factory=list)   # basis size after each HCI iteration
    n_pert: int = 0
    dE: np.ndarray | None = None
    E_var: np.ndarray | None = None


def solve(path: str, h_mode: str = "conn", pt2_mode: str = "conn", max_iter: int = 100) -> Result:
    """Full reference procedure (src/VHCI.cpp:5-120) on one input file."""
    o = Oracle(path)
    sizes = []
    if o.eps1 == 0.0:
        H = o.sparse_h(h_mode)
        E, C = sparse_eigs(H, o.neig)
    else:
        w, v = np.linalg.eigh(o.dense_h())
        E, C = w, v
        for _ in range(max_iter):
            nopt = min(o.neig, o.n)
            new = o.select(C, nopt, o.eps1)
            if len(new) / o.n <= 0.01:
                break
            o.append_basis(new)
            sizes.append(o.n)
            H = o.sparse_h(h_mode)
            E, C = sparse_eigs(H, o.neig)
    res = Result(E=np.array(E), C=C, basis=o.basis(), sizes=sizes)
    res.E_var = res.E.copy()
    if o.perturb:
        nopt = min(o.neig, o.n)
        dE, P = o.pt2(C, E, nopt, o.eps2, pt2_mode)
        res.E = res.E.copy()
        res.E[:nopt] += dE
        res.dE = dE
        res.n_pert = len(P)
    return res
