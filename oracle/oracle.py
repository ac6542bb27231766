"""ORACLE -- test infrastructure only.

ctypes front end of ``oracle/_ref/libgiporacle.so`` (the plain-C restatement of GIP's
CPU path in ``oracle/gip_oracle.c``).  Only tests, the smoke check and the CPU leg of
the benchmark use it, as the checker; the product never imports it.

Parity is pinned: on C100K merged to one rank it prints GIP's README.md:73-82 lines
digit for digit and matches GIP's own CPU build bit for bit (tests/test_oracle.py).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libgiporacle.so")
REF_BIN = os.path.join(_HERE, "_ref", "gip_ref_cpu")

OP_ORDER = ("D", "Ec", "L", "Lb", "Mx", "My", "Mz", "Mres", "Gx", "Gy", "Gz",
            "SFx", "SFy", "SFz", "SO")
STATE_VECS = ("u", "v", "w", "dxs", "ax", "ay", "az", "ax0", "ay0", "az0", "rhs", "p", "p0",
              "gpx", "gpy", "gpz", "temp", "mf", "cval")


class _Csr(C.Structure):
    _fields_ = [("nrows", C.c_int), ("ncols", C.c_int), ("nnz", C.c_int),
                ("rowptr", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p)]


class _Ops(C.Structure):
    _fields_ = [(n, _Csr) for n in OP_ORDER] + [
        ("n_inner", C.c_int), ("n_owned", C.c_int), ("n_faces", C.c_int)]


class _State(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in STATE_VECS] + [
        ("dt", C.c_double), ("sigma", C.c_double), ("time", C.c_double), ("started", C.c_int)]


class _Params(C.Structure):
    _fields_ = [("rho", C.c_double), ("gamma", C.c_double), ("cg_maxit", C.c_int),
                ("cg_mode", C.c_int), ("cg_tol", C.c_double)]


def build() -> None:
    """Compile the oracle library (and GIP's CPU build when the reference is present)."""
    subprocess.check_call(["make", "-s", "-C", _HERE, "oracle"])


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _lib.orc_dns_run.restype = C.c_int
        _lib.orc_pcg.restype = C.c_int
        _lib.orc_cfl.restype = C.c_double
        _lib.orc_dot.restype = C.c_double
        _lib.orc_norminf.restype = C.c_double
    return _lib


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def _csr_struct(m, keep: list) -> _Csr:
    rp = np.ascontiguousarray(m.rowptr, np.int32)
    col = np.ascontiguousarray(m.col, np.int32)
    val = np.ascontiguousarray(m.val, np.float64)
    keep += [rp, col, val]
    return _Csr(m.nrows, m.ncols, m.nnz, _ptr(rp), _ptr(col), _ptr(val))


def spmv(m, x: np.ndarray, y: np.ndarray, alpha: float = 0.0, beta: float = 0.0,
         mode: int = 0) -> np.ndarray:
    """GIP CPU SpMV semantics on a :class:`gip_b200.formats.Csr` (y updated in place)."""
    keep: list = []
    s = _csr_struct(m, keep)
    x = np.ascontiguousarray(x, np.float64)
    assert y.dtype == np.float64 and y.flags.c_contiguous
    lib().orc_spmv(C.byref(s), _ptr(x), _ptr(y), C.c_double(alpha), C.c_double(beta),
                   C.c_int(mode))
    return y


def pcg(L, b: np.ndarray, x0: np.ndarray, maxit: int = 100, mode: int = 0,
        tol: float = 0.0):
    """GIP_LinearSolver::solve restated; returns ``(x, iterations, r.r)``."""
    keep: list = []
    s = _csr_struct(L, keep)
    n_all = max(x0.shape[0], L.nrows)
    x0 = np.ascontiguousarray(x0, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    dinv = np.zeros(L.nrows)
    lib().orc_inverse_diagonal(C.byref(s), _ptr(dinv))
    x = np.zeros(n_all)
    work = np.zeros(4 * n_all)
    rr = C.c_double(0)
    it = lib().orc_pcg(C.byref(s), _ptr(dinv), _ptr(b), _ptr(x), _ptr(x0), C.c_int(n_all),
                       C.c_int(maxit), C.c_int(mode), C.c_double(tol), _ptr(work), C.byref(rr))
    return x, it, rr.value


class OracleDNS:
    """GIP_DNS<Multicore> restated: holds every GIP_DNS vector and advances timesteps."""

    def __init__(self, case, rho: float = 1.0, gamma: float = 1e-3, cg_maxit: int = 100,
                 cg_mode: int = 0, cg_tol: float = 0.0):
        self._keep: list = []
        self.ops = _Ops(**{n: _csr_struct(case.ops[n], self._keep) for n in OP_ORDER},
                        n_inner=case.n_inner, n_owned=case.n_owned, n_faces=case.n_faces)
        NO, NF = case.n_owned, case.n_faces
        self.vec: Dict[str, np.ndarray] = {}
        for n in STATE_VECS:
            size = NF if n == "mf" else (case.ops["D"].nnz if n == "cval" else NO)
            self.vec[n] = np.zeros(size)
        for n in ("u", "v", "w", "dxs"):
            self.vec[n][:] = case.fields[n]
        self.vec["cval"][:] = case.ops["D"].val   # C.postConstruct reads the D file
        self.state = _State(**{n: _ptr(self.vec[n]) for n in STATE_VECS}, dt=0.0, sigma=0.0,
                            time=0.0, started=0)
        self.params = _Params(rho, gamma, cg_maxit, cg_mode, cg_tol)

    def run(self, nsteps: int) -> Dict[str, np.ndarray]:
        out = {"time": np.zeros(nsteps), "dt": np.zeros(nsteps), "massr": np.zeros(nsteps),
               "iters": np.zeros(nsteps, np.int32), "rr": np.zeros(nsteps)}
        rc = lib().orc_dns_run(C.byref(self.ops), C.byref(self.params), C.byref(self.state),
                               C.c_int(nsteps), _ptr(out["time"]), _ptr(out["dt"]),
                               _ptr(out["massr"]), _ptr(out["iters"]), _ptr(out["rr"]))
        if rc != 0:
            raise RuntimeError("oracle: out of memory")
        return out

    @property
    def dt(self) -> float:
        return self.state.dt

    @property
    def time(self) -> float:
        return self.state.time


def format_line(time: float, dt: float, massr: float, it: int) -> str:
    """GIP's per-step line (GIP_DNS.h:403-404, std::scientific with 6 digits)."""
    return f"time {time:.6e} [dt::{dt:.6e}] massr {massr:.6e} ite {it}"
