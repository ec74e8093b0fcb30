"""Python binding of the C ABI in include/vhci_gpu.h (ctypes).

This is the interface the tests, the benchmark and Python users call.  It mirrors the reference
program's seams (input parsing, heat-bath selection, Hamiltonian build, eigensolve, PT2, output and
checkpoint files) one call each; every call goes to the sm_100a library `libvhci_gpu.so`, which
has no CPU path — without a CUDA device, `VHCI(...)` raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libvhci_gpu.so")

(OK, E_INPUT, E_OOM, E_TABLE_FULL, E_KEY_OVERFLOW, E_NOT_CONVERGED, E_CUDA, E_STATE, E_NEG_ZPE,
 E_LIMIT) = range(10)
_NAMES = {0: "OK", 1: "E_INPUT", 2: "E_OOM", 3: "E_TABLE_FULL", 4: "E_KEY_OVERFLOW",
          5: "E_NOT_CONVERGED", 6: "E_CUDA", 7: "E_STATE", 8: "E_NEG_ZPE",
          9: "E_LIMIT"}

# Every symbol declared in include/vhci_gpu.h.
EXPORTS = [
    "vhci_default_opts", "vhci_create_from_file", "vhci_create", "vhci_destroy",
    "vhci_last_error", "vhci_get_info", "vhci_get_stats", "vhci_reset_stats", "vhci_get_fc_list",
    "vhci_get_hb_list", "vhci_get_freqs", "vhci_set_basis", "vhci_get_basis", "vhci_set_vectors",
    "vhci_get_vectors", "vhci_select", "vhci_get_selected", "vhci_build_h", "vhci_get_h_csr",
    "vhci_structural_nnz", "vhci_eigs", "vhci_hci", "vhci_pt2", "vhci_write_freqs",
    "vhci_write_checkpoint", "vhci_read_checkpoint", "vhci_get_energies", "vhci_apply_h",
    "vhci_residual_norms", "vhci_residual_norms_noalloc", "vhci_default_serve_opts", "vhci_serve",
    "vhci_set_comm",
]


class VhciError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_NAMES.get(code, code)}: {msg}")
        self.code = code


class Opts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("precision", ctypes.c_int), ("eig_tol", ctypes.c_double),
                ("eig_maxit", ctypes.c_int), ("verbose", ctypes.c_int),
                ("host_threads", ctypes.c_int), ("pt2_chunk", ctypes.c_int64),
                ("structural_nnz", ctypes.c_int), ("max_basis", ctypes.c_int64),
                ("max_pert", ctypes.c_int64), ("stream_priority", ctypes.c_int)]


class Problem(ctypes.Structure):
    _fields_ = [("nmodes", ctypes.c_int), ("freq", ctypes.POINTER(ctypes.c_double)),
                ("cap", ctypes.POINTER(ctypes.c_int)), ("max_quanta", ctypes.c_int),
                ("nfc", ctypes.c_int), ("fc_order", ctypes.POINTER(ctypes.c_int)),
                ("fc_modes", ctypes.POINTER(ctypes.c_int)),
                ("fc_value", ctypes.POINTER(ctypes.c_double)), ("eps1", ctypes.c_double),
                ("nstate", ctypes.c_int), ("pt2", ctypes.c_int), ("eps2", ctypes.c_double)]


class Info(ctypes.Structure):
    _fields_ = [("nmodes", ctypes.c_int), ("nstate", ctypes.c_int), ("pt2", ctypes.c_int),
                ("key_bits", ctypes.c_int), ("key_words", ctypes.c_int),
                ("eps1", ctypes.c_double), ("eps2", ctypes.c_double),
                ("n_basis", ctypes.c_int64), ("n_fc", ctypes.c_int64), ("n_hb", ctypes.c_int64),
                ("n_groups", ctypes.c_int64), ("n_vectors", ctypes.c_int64),
                ("h_nnz", ctypes.c_int64)]


# void (*vhci_iter_cb)(void* user, int iteration, int64_t n_basis, double zpe)
ITER_CB = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double)


# int (*allreduce_sum)(void* user, double* buf, int64_t count)
ALLREDUCE_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64)
# int (*allgather)(void* user, const void* send, void* recv, int64_t bytes)
ALLGATHER_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_int64)


class Comm(ctypes.Structure):
    _fields_ = [("rank", ctypes.c_int), ("nranks", ctypes.c_int), ("user", ctypes.c_void_p),
                ("allreduce_sum", ALLREDUCE_CB), ("allgather", ALLGATHER_CB)]


class Request(ctypes.Structure):
    _fields_ = [("input_path", ctypes.c_char_p), ("problem", ctypes.c_void_p),
                ("arrival_s", ctypes.c_double)]


class ServeOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("slots", ctypes.c_int),
                ("reserve_bytes", ctypes.c_double), ("max_states", ctypes.c_int),
                ("max_basis", ctypes.c_int64), ("max_pert", ctypes.c_int64),
                ("fifo_priority", ctypes.c_int)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("worker", ctypes.c_int), ("retries", ctypes.c_int),
                ("n_energies", ctypes.c_int), ("n_basis", ctypes.c_int64),
                ("n_pert", ctypes.c_int64), ("t_admit", ctypes.c_double),
                ("t_done", ctypes.c_double), ("message", ctypes.c_char * 160)]


class ServeSummary(ctypes.Structure):
    _fields_ = [("wall_s", ctypes.c_double), ("completed", ctypes.c_int),
                ("failed", ctypes.c_int), ("peak_in_flight", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("ms_select", ctypes.c_double), ("ms_hbuild", ctypes.c_double),
                ("ms_eigs", ctypes.c_double), ("ms_pt2", ctypes.c_double),
                ("ms_total", ctypes.c_double), ("ms_spmm", ctypes.c_double),
                ("spmm_calls", ctypes.c_int64), ("spmm_cols", ctypes.c_int64),
                ("spmm_bytes", ctypes.c_int64), ("hbuild_probes", ctypes.c_int64),
                ("select_candidates", ctypes.c_int64), ("pt2_entries", ctypes.c_int64),
                ("pt2_perturbers", ctypes.c_int64), ("ms_pt2_reduce", ctypes.c_double),
                ("pt2_reduce_bytes", ctypes.c_int64), ("eig_iterations", ctypes.c_int),
                ("hci_iterations", ctypes.c_int), ("h2d_bytes", ctypes.c_int64),
                ("d2h_bytes", ctypes.c_int64), ("kernel_launches", ctypes.c_int64),
                ("spmm_gather_bytes", ctypes.c_int64), ("mixed_max_residual", ctypes.c_double),
                ("hbuild_incremental", ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def lib():
    """Load libvhci_gpu.so; raises if it has not been built (there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C vhci_b200/csrc`")
        L = ctypes.CDLL(LIB_PATH)
        vp, i64, i64p = ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)
        dp, i32p, u8p = (ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32),
                         ctypes.POINTER(ctypes.c_uint8))
        sig = {
            "vhci_default_opts": (None, [ctypes.POINTER(Opts)]),
            "vhci_create_from_file": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(Opts),
                                                     ctypes.c_int, ctypes.POINTER(vp)]),
            "vhci_create": (ctypes.c_int, [ctypes.POINTER(Problem), ctypes.POINTER(Opts),
                                           ctypes.c_int, ctypes.POINTER(vp)]),
            "vhci_destroy": (ctypes.c_int, [vp]),
            "vhci_last_error": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_size_t]),
            "vhci_get_info": (ctypes.c_int, [vp, ctypes.POINTER(Info)]),
            "vhci_get_stats": (ctypes.c_int, [vp, ctypes.POINTER(Stats)]),
            "vhci_reset_stats": (ctypes.c_int, [vp]),
            "vhci_get_fc_list": (ctypes.c_int, [vp, dp, i32p, i32p]),
            "vhci_get_hb_list": (ctypes.c_int, [vp, dp, i32p, i32p]),
            "vhci_get_freqs": (ctypes.c_int, [vp, dp]),
            "vhci_set_basis": (ctypes.c_int, [vp, u8p, i64]),
            "vhci_get_basis": (ctypes.c_int, [vp, u8p, i64, i64p]),
            "vhci_set_vectors": (ctypes.c_int, [vp, dp, dp, ctypes.c_int]),
            "vhci_get_vectors": (ctypes.c_int, [vp, dp, dp, ctypes.c_int]),
            "vhci_select": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int, i64p]),
            "vhci_get_selected": (ctypes.c_int, [vp, u8p, i64, i64p]),
            "vhci_build_h": (ctypes.c_int, [vp, i64p]),
            "vhci_get_h_csr": (ctypes.c_int, [vp, i64p, i32p, dp]),
            "vhci_structural_nnz": (ctypes.c_int, [vp, i64p]),
            "vhci_eigs": (ctypes.c_int, [vp, ctypes.c_int, dp]),
            "vhci_apply_h": (ctypes.c_int, [vp, dp, dp, ctypes.c_int]),
            "vhci_default_serve_opts": (None, [ctypes.POINTER(ServeOpts)]),
            "vhci_serve": (ctypes.c_int, [ctypes.POINTER(Request), ctypes.c_int,
                                          ctypes.POINTER(ServeOpts), ctypes.POINTER(Result), dp,
                                          ctypes.POINTER(ServeSummary)]),
            "vhci_residual_norms": (ctypes.c_int, [vp, dp, dp, dp, ctypes.c_int]),
            "vhci_residual_norms_noalloc": (ctypes.c_int, [vp, vp, vp, vp, ctypes.c_int]),
            "vhci_hci": (ctypes.c_int, [vp, ctypes.c_char_p, vp, vp]),
            "vhci_pt2": (ctypes.c_int, [vp, ctypes.c_double, dp, i64p]),
            "vhci_write_freqs": (ctypes.c_int, [vp, ctypes.c_char_p]),
            "vhci_write_checkpoint": (ctypes.c_int, [vp, ctypes.c_char_p]),
            "vhci_read_checkpoint": (ctypes.c_int, [vp, ctypes.c_char_p]),
            "vhci_get_energies": (ctypes.c_int, [vp, dp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
            "vhci_set_comm": (ctypes.c_int, [vp, ctypes.POINTER(Comm)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def default_opts(**kw) -> Opts:
    o = Opts()
    lib().vhci_default_opts(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class VHCI:
    """One solve context (the reference program's global state, held on one GPU)."""

    def __init__(self, path: str | None = None, *, problem: dict | None = None, precision: int = 0,
                 device: int = 0, restart: bool = False, verbose: bool = False, **opts):
        self.h = ctypes.c_void_p()
        o = default_opts(precision=precision, device=device, verbose=int(verbose), **opts)
        L = lib()
        if path is not None:
            st = L.vhci_create_from_file(path.encode(), ctypes.byref(o), int(restart),
                                         ctypes.byref(self.h))
        else:
            self._keep = _problem_struct(problem)
            st = L.vhci_create(ctypes.byref(self._keep[0]), ctypes.byref(o), int(restart),
                               ctypes.byref(self.h))
        if st != OK:
            msg = self.last_error()
            self.close()
            raise VhciError(st, msg)

    # ---- lifetime / errors ----
    def close(self):
        if self.h:
            lib().vhci_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def last_error(self) -> str:
        if not self.h:
            return ""
        b = ctypes.create_string_buffer(512)
        lib().vhci_last_error(self.h, b, 512)
        return b.value.decode(errors="replace")

    def _check(self, st):
        if st != OK:
            raise VhciError(st, self.last_error())

    # ---- info ----
    @property
    def info(self) -> Info:
        i = Info()
        self._check(lib().vhci_get_info(self.h, ctypes.byref(i)))
        return i

    @property
    def n(self) -> int:
        return int(self.info.n_basis)

    def stats(self) -> dict:
        s = Stats()
        self._check(lib().vhci_get_stats(self.h, ctypes.byref(s)))
        return s.as_dict()

    def reset_stats(self):
        self._check(lib().vhci_reset_stats(self.h))

    def _fc(self, fn, count):
        v = np.zeros(count)
        m = np.zeros((count, 6), np.int32)
        p = np.zeros((count, 6), np.int32)
        self._check(fn(self.h, _ptr(v, ctypes.c_double), _ptr(m, ctypes.c_int32),
                       _ptr(p, ctypes.c_int32)))
        return v, m, p

    def fc_list(self):
        return self._fc(lib().vhci_get_fc_list, int(self.info.n_fc))

    def hb_list(self):
        return self._fc(lib().vhci_get_hb_list, int(self.info.n_hb))

    def freqs(self) -> np.ndarray:
        f = np.zeros(self.info.nmodes)
        self._check(lib().vhci_get_freqs(self.h, _ptr(f, ctypes.c_double)))
        return f

    # ---- basis / vectors ----
    def basis(self) -> np.ndarray:
        n = self.n
        q = np.zeros((n, self.info.nmodes), np.uint8)
        nn = ctypes.c_int64()
        self._check(lib().vhci_get_basis(self.h, _ptr(q, ctypes.c_uint8), n, ctypes.byref(nn)))
        return q

    def set_basis(self, q: np.ndarray):
        q = np.ascontiguousarray(q, np.uint8)
        self._check(lib().vhci_set_basis(self.h, _ptr(q, ctypes.c_uint8), q.shape[0]))

    def set_vectors(self, C: np.ndarray, E: np.ndarray):
        C = np.asfortranarray(C, np.float64)
        E = np.ascontiguousarray(E, np.float64)
        self._check(lib().vhci_set_vectors(self.h, _ptr(C, ctypes.c_double),
                                           _ptr(E, ctypes.c_double), C.shape[1]))

    def vectors(self, k: int | None = None):
        if k is None:
            k = int(self.info.n_vectors)
        C = np.zeros((self.n, k), order="F")
        E = np.zeros(k)
        self._check(lib().vhci_get_vectors(self.h, _ptr(C, ctypes.c_double),
                                           _ptr(E, ctypes.c_double), k))
        return C, E

    def energies(self) -> np.ndarray:
        k = int(self.info.nstate)
        E = np.zeros(k)
        n = ctypes.c_int()
        self._check(lib().vhci_get_energies(self.h, _ptr(E, ctypes.c_double), k, ctypes.byref(n)))
        return E[: n.value]

    # ---- hot path ----
    def select(self, eps: float, append: bool = False) -> np.ndarray:
        nn = ctypes.c_int64()
        self._check(lib().vhci_select(self.h, eps, int(append), ctypes.byref(nn)))
        q = np.zeros((nn.value, self.info.nmodes), np.uint8)
        if nn.value and not append:
            m = ctypes.c_int64()
            self._check(lib().vhci_get_selected(self.h, _ptr(q, ctypes.c_uint8), nn.value,
                                                ctypes.byref(m)))
        return q

    def build_h(self) -> int:
        nnz = ctypes.c_int64()
        self._check(lib().vhci_build_h(self.h, ctypes.byref(nnz)))
        return nnz.value

    def structural_nnz(self) -> int:
        """Entries of the reference's stored pattern on the current basis (vhci_structural_nnz)."""
        x = ctypes.c_int64()
        self._check(lib().vhci_structural_nnz(self.h, ctypes.byref(x)))
        return x.value

    def h_csr(self):
        import scipy.sparse as sp
        n = self.n
        nnz = self.build_h() if self.info.h_nnz == 0 else int(self.info.h_nnz) + n
        rp = np.zeros(n + 1, np.int64)
        col = np.zeros(nnz, np.int32)
        val = np.zeros(nnz)
        self._check(lib().vhci_get_h_csr(self.h, _ptr(rp, ctypes.c_int64), _ptr(col, ctypes.c_int32),
                                         _ptr(val, ctypes.c_double)))
        return sp.csr_matrix((val, col, rp), shape=(n, n))

    def apply_h(self, X: np.ndarray) -> np.ndarray:
        X = np.asfortranarray(X, np.float64)
        Y = np.zeros_like(X, order="F")
        self._check(lib().vhci_apply_h(self.h, _ptr(X, ctypes.c_double), _ptr(Y, ctypes.c_double),
                                       X.shape[1]))
        return Y

    def residual_norms(self, X: np.ndarray, theta: np.ndarray) -> np.ndarray:
        X = np.asfortranarray(X, np.float64)
        theta = np.ascontiguousarray(theta, np.float64)
        r = np.zeros(X.shape[1])
        self._check(lib().vhci_residual_norms(self.h, _ptr(X, ctypes.c_double),
                                              _ptr(theta, ctypes.c_double),
                                              _ptr(r, ctypes.c_double), X.shape[1]))
        return r

    def residual_norms_noalloc(self, x_dev: int, theta_dev: int, rnorm_dev: int, k: int) -> None:
        """Residual norms over caller-owned DEVICE buffers (addresses as integers): X n x k
        row-major, theta k, rnorm k.  Allocates nothing (see include/vhci_gpu.h)."""
        self._check(lib().vhci_residual_norms_noalloc(self.h, ctypes.c_void_p(x_dev),
                                                      ctypes.c_void_p(theta_dev),
                                                      ctypes.c_void_p(rnorm_dev), k))

    def set_comm(self, comm) -> None:
        """Shard this context's solve over the ranks of `comm` (a vhci_b200.shard.Comm, or None to
        solve alone).  Every rank must create its context from the same input and make the same
        calls."""
        self._comm = comm  # the callbacks must outlive the context's use of them
        self._check(lib().vhci_set_comm(self.h, ctypes.byref(comm.struct) if comm else None))

    def eigs(self, k: int) -> np.ndarray:
        E = np.zeros(k)
        self._check(lib().vhci_eigs(self.h, k, _ptr(E, ctypes.c_double)))
        return E

    def hci(self, checkpoint: str | None = None, callback=None):
        """The heat-bath procedure (vhci_hci).  callback(iteration, n_basis, zpe) runs after the
        first dense step (iteration 0) and after every heat-bath iteration's eigensolve."""
        cb = None
        if callback is not None:
            cb = ITER_CB(lambda user, it, n, zpe: callback(int(it), int(n), float(zpe)))
        self._check(lib().vhci_hci(self.h, checkpoint.encode() if checkpoint else None,
                                   ctypes.cast(cb, ctypes.c_void_p) if cb else None, None))

    def pt2(self, eps2: float | None = None):
        if eps2 is None:
            eps2 = self.info.eps2
        k = min(int(self.info.nstate), self.n)
        dE = np.zeros(k)
        npert = ctypes.c_int64()
        self._check(lib().vhci_pt2(self.h, eps2, _ptr(dE, ctypes.c_double), ctypes.byref(npert)))
        return dE, npert.value

    # ---- files ----
    def write_freqs(self, path: str):
        self._check(lib().vhci_write_freqs(self.h, path.encode()))

    def write_checkpoint(self, path: str):
        self._check(lib().vhci_write_checkpoint(self.h, path.encode()))

    def read_checkpoint(self, path: str):
        self._check(lib().vhci_read_checkpoint(self.h, path.encode()))


def _problem_struct(p: dict):
    nm = len(p["freq"])
    freq = np.ascontiguousarray(p["freq"], np.float64)
    cap = np.ascontiguousarray(p.get("cap", [8] * nm), np.int32)
    fcs = p["fcs"]  # list of (modes tuple, value)
    order = np.array([len(m) for m, _ in fcs], np.int32)
    modes = np.full((max(len(fcs), 1), 6), 0, np.int32)
    for i, (m, _) in enumerate(fcs):
        modes[i, :len(m)] = m
    vals = np.array([v for _, v in fcs], np.float64)
    s = Problem(nmodes=nm, freq=_ptr(freq, ctypes.c_double), cap=_ptr(cap, ctypes.c_int),
                max_quanta=int(p.get("ntot", 2)), nfc=len(fcs),
                fc_order=_ptr(order, ctypes.c_int), fc_modes=_ptr(modes, ctypes.c_int),
                fc_value=_ptr(vals, ctypes.c_double), eps1=float(p.get("eps1", 1.0)),
                nstate=int(p.get("nstate", 10)), pt2=int(p.get("pt2", 0)),
                eps2=float(p.get("eps2", 0.0)))
    return (s, freq, cap, order, modes, vals)


def serve(requests, slots: int = 8, reserve_bytes: float = 8e9, device: int = 0,
          max_states: int = 256, max_basis: int = 0, max_pert: int = 0,
          fifo_priority: bool = True):
    """Run many independent solves on one GPU with continuous batching (vhci_serve).
    `requests` is a list of (input_path, arrival_seconds).  Returns (summary dict, list of
    per-request dicts: status, energies, basis size, |P|, arrival/admit/done times, message)."""
    n = len(requests)
    reqs = (Request * n)()
    keep = []
    for i, (path, t) in enumerate(requests):
        b = str(path).encode()
        keep.append(b)
        reqs[i].input_path = b
        reqs[i].problem = None
        reqs[i].arrival_s = float(t)
    so = ServeOpts()
    lib().vhci_default_serve_opts(ctypes.byref(so))
    so.device, so.slots, so.reserve_bytes, so.max_states = device, slots, reserve_bytes, max_states
    so.max_basis, so.max_pert = max_basis, max_pert
    so.fifo_priority = 1 if fifo_priority else 0
    res = (Result * n)()
    E = np.zeros(n * max_states)
    summ = ServeSummary()
    st = lib().vhci_serve(reqs, n, ctypes.byref(so), res, _ptr(E, ctypes.c_double),
                          ctypes.byref(summ))
    if st not in (OK, E_STATE):
        raise VhciError(st, "vhci_serve")
    out = []
    for i in range(n):
        r = res[i]
        out.append({"status": r.status, "worker": r.worker, "retries": r.retries,
                    "E": E[i * max_states: i * max_states + r.n_energies].copy(),
                    "n_basis": r.n_basis, "n_pert": r.n_pert, "t_admit": r.t_admit,
                    "t_done": r.t_done, "arrival": float(requests[i][1]),
                    "message": r.message.decode(errors="replace")})
    return ({"status": st, "wall_s": summ.wall_s, "completed": summ.completed,
             "failed": summ.failed, "peak_in_flight": summ.peak_in_flight}, out)


def solve(path: str, precision: int = 0, **opts) -> dict:
    """The reference program's full procedure on one input file: heat-bath iterations (or one VCI
    eigensolve) and, when the input asks for it, PT2.  Returns energies and counters."""
    with VHCI(path, precision=precision, **opts) as v:
        v.hci()
        E_var = v.energies().copy()
        dE, npert = (None, 0)
        if v.info.pt2:
            dE, npert = v.pt2()
        return {"E": v.energies().copy(), "E_var": E_var, "dE": dE, "n_pert": npert,
                "n_basis": v.n, "stats": v.stats()}
