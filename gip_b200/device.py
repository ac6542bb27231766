"""Python front end of the B200 library over its C ABI.

Device vectors are ``torch.float64`` CUDA tensors; the operators and solvers are
library handles.  Names follow GIP's Specification: ``DeviceMatrix.spmv`` is
``GIP_Matrix::spmv`` (y = A x, or y = alpha A x + beta y with mode 1, empty rows left
untouched), ``PcgSolver`` is ``GIP_LinearSolver`` and ``DnsEngine`` is ``GIP_DNS``.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional

import numpy as np
import torch

from . import _lib as L
from .formats import Csr, GipCase


def _stream(stream=None) -> C.c_void_p:
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


def _dptr(t: Optional[torch.Tensor]) -> C.c_void_p:
    if t is None:
        return C.c_void_p(0)
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    return C.c_void_p(t.data_ptr())


def _hptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def _host_csr(m: Csr, keep: list) -> L.HostCsr:
    rp = np.ascontiguousarray(m.rowptr, np.int32)
    col = np.ascontiguousarray(m.col, np.int32)
    val = np.ascontiguousarray(m.val, np.float64)
    keep += [rp, col, val]
    return L.HostCsr(m.nrows, m.ncols, m.nnz, _hptr(rp), _hptr(col), _hptr(val))


# ----------------------------------------------------------------------------- raw kernels
def spmv_raw(rowptr: torch.Tensor, col: torch.Tensor, val: torch.Tensor, x: torch.Tensor,
             y: torch.Tensor, alpha: float = 0.0, beta: float = 0.0, mode: int = 0,
             stream=None) -> torch.Tensor:
    L.call("gipb200_dcsr_spmv", rowptr.numel() - 1, _dptr(rowptr), _dptr(col), _dptr(val),
           _dptr(x), _dptr(y), alpha, beta, mode, _stream(stream))
    return y


def axpy(y: torch.Tensor, x: torch.Tensor, alpha: float, n: Optional[int] = None, stream=None):
    L.call("gipb200_daxpy", y.numel() if n is None else n, _dptr(y), _dptr(x), alpha,
           _stream(stream))
    return y


def axpby(y: torch.Tensor, x: torch.Tensor, alpha: float, beta: float, n: Optional[int] = None,
          stream=None):
    L.call("gipb200_daxpby", y.numel() if n is None else n, _dptr(y), _dptr(x), alpha, beta,
           _stream(stream))
    return y


def fill(y: torch.Tensor, value: float, stream=None):
    L.call("gipb200_dfill", y.numel(), _dptr(y), value, _stream(stream))
    return y


def dot(x: torch.Tensor, y: torch.Tensor, n: Optional[int] = None, stream=None) -> float:
    out = C.c_double()
    L.call("gipb200_ddot", x.numel() if n is None else n, _dptr(x), _dptr(y), C.byref(out),
           _stream(stream))
    return out.value


def norminf(x: torch.Tensor, n: Optional[int] = None, stream=None) -> float:
    out = C.c_double()
    L.call("gipb200_dnorminf", x.numel() if n is None else n, _dptr(x), C.byref(out),
           _stream(stream))
    return out.value


def cfl(u, v, w, dxs, n: int, gamma: float, rho: float, stream=None) -> float:
    out = C.c_double()
    L.call("gipb200_cfl", n, _dptr(u), _dptr(v), _dptr(w), _dptr(dxs), gamma, rho, C.byref(out),
           _stream(stream))
    return out.value


# ----------------------------------------------------------------------------- matrices
class DeviceMatrix:
    """A CSR operator resident on the device (``GIP_MatrixCuda`` counterpart)."""

    def __init__(self, m: Csr):
        lib = L.load()
        keep: list = []
        h = _host_csr(m, keep)
        handle = C.c_void_p()
        L.check(lib.gipb200_matrix_create(h.nrows, h.ncols, h.nnz, h.rowptr, h.col, h.val,
                                          C.byref(handle)), "gipb200_matrix_create")
        self.handle = handle
        self.nrows, self.ncols, self.nnz = m.nrows, m.ncols, m.nnz

    def info(self) -> dict:
        r, c, z = C.c_int(), C.c_int(), C.c_int()
        s = C.c_int64()
        L.call("gipb200_matrix_info", self.handle, C.byref(r), C.byref(c), C.byref(z), C.byref(s))
        return {"nrows": r.value, "ncols": c.value, "nnz": z.value, "padded_slots": s.value}

    def _check(self, x: torch.Tensor, ylen: int, y: torch.Tensor) -> None:
        if x.dtype != torch.float64 or y.dtype != torch.float64:
            raise TypeError("vectors must be float64")
        if x.numel() < self.ncols or y.numel() < ylen:
            raise ValueError(f"vector sizes ({x.numel()}, {y.numel()}) below operator "
                             f"({self.ncols}, {ylen})")

    def spmv(self, x: torch.Tensor, y: torch.Tensor, alpha: float = 0.0, beta: float = 0.0,
             mode: int = 0, stream=None) -> torch.Tensor:
        self._check(x, self.nrows, y)
        L.call("gipb200_matrix_spmv", self.handle, _dptr(x), _dptr(y), alpha, beta, mode,
               _stream(stream))
        return y

    def spmv_values(self, x: torch.Tensor, target: "DeviceMatrix", alpha: float = 0.0,
                    beta: float = 0.0, mode: int = 0, stream=None) -> None:
        if x.numel() < self.ncols:
            raise ValueError("x shorter than the operator's columns")
        L.call("gipb200_matrix_spmv_values", self.handle, _dptr(x), target.handle, alpha, beta,
               mode, _stream(stream))

    def values(self) -> np.ndarray:
        out = np.zeros(self.nnz)
        L.call("gipb200_matrix_get_values", self.handle, _hptr(out))
        return out

    def inverse_diagonal(self) -> tuple:
        d = torch.zeros(self.nrows, dtype=torch.float64, device="cuda")
        miss = C.c_int()
        L.call("gipb200_matrix_inverse_diagonal", self.handle, _dptr(d), C.byref(miss))
        return d, miss.value

    def spmv_dot(self, x: torch.Tensor, y: torch.Tensor, out: torch.Tensor, n_dot: int = None,
                 stream=None) -> torch.Tensor:
        """y = A x and out[0] = x[:n_dot].y[:n_dot] (device scalar, no host wait)."""
        self._check(x, self.nrows, y)
        L.call("gipb200_matrix_spmv_dot", self.handle, _dptr(x), _dptr(y),
               self.nrows if n_dot is None else n_dot, _dptr(out), _stream(stream))
        return out

    def close(self) -> None:
        if getattr(self, "handle", None):
            L.load().gipb200_matrix_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


MODES = {"fixed": L.PCG_FIXED, "tol": L.PCG_TOL, "mixed": L.PCG_MIXED}
PRECONDS = {"jacobi": 0, "amg": 1}


def pcg_params(mode: str = "fixed", maxit: int = 100, tol: float = 1e-6,
               inner_tol: float = 1e-3, inner_maxit: int = 2000, max_outer: int = 30,
               precond: str = "jacobi") -> L.PcgParams:
    """precond: "jacobi" (GIP's) or "amg" (tolerance and mixed modes: a smoothed-aggregation
    V-cycle, FP64 in the tolerance mode and FP32 in the mixed one, its hierarchy built on
    the host at create time; the fixed mode is GIP's and keeps Jacobi)."""
    return L.PcgParams(MODES[mode], maxit, tol, inner_tol, inner_maxit, max_outer,
                       PRECONDS[precond])


CYCLE_KINDS = ("jacobi0", "residual", "restrict", "dense", "prolong", "smooth", "tail")
# the kernel each product form runs as (GIPB200_FORM_*)
FORM_KERNELS = ("k_amgp_spmv", "k_amg_spmv", "k_amg_spmv_pf", "k_amg_csr", "k_amg_dense",
                "k_amg_jacobi0", "k_amg_tail", "k_amg_smooth_dot")


def _vcycle_profile(fn: str, handle, reps: int, stream) -> list:
    cap = 128
    nk = C.c_int()
    lvl = np.zeros(cap, np.int32)
    kind = np.zeros(cap, np.int32)
    ms = np.zeros(cap)
    by = np.zeros(cap)
    L.call(fn, handle, reps, _stream(stream), cap, C.byref(nk), _hptr(lvl), _hptr(kind),
           _hptr(ms), _hptr(by))
    form = np.zeros(cap, np.int32)
    nf = C.c_int()
    L.call(fn.replace("_profile", "_forms"), handle, cap, C.byref(nf), _hptr(form))
    return [{"level": int(lvl[k]), "kind": CYCLE_KINDS[kind[k]], "ms": float(ms[k]),
             "bytes": float(by[k]), "kernel": FORM_KERNELS[form[k]]}
            for k in range(min(nk.value, cap))]


class PcgSolver:
    """``GIP_LinearSolver`` on the device: Jacobi PCG, FP64 (fixed or tolerance) or
    mixed FP32-inner / FP64-refinement."""

    def __init__(self, A: DeviceMatrix, n_all: Optional[int] = None, **kw):
        self.A = A
        self.n_all = n_all or A.nrows
        self.params = pcg_params(**kw)
        handle = C.c_void_p()
        L.call("gipb200_pcg_create", A.handle, n_all or A.nrows, C.byref(self.params),
               C.byref(handle))
        self.handle = handle

    def solve(self, b: torch.Tensor, x: torch.Tensor, x0: torch.Tensor, stream=None) -> dict:
        n_all = max(self.n_all, self.A.nrows)
        if b.numel() < self.A.nrows or x.numel() < n_all or x0.numel() < n_all:
            raise ValueError("b needs the operator's rows, x and x0 need n_all entries")
        for t in (b, x, x0):
            if t.dtype != torch.float64:
                raise TypeError("vectors must be float64")
        res = L.PcgResult()
        L.call("gipb200_pcg_solve", self.handle, _dptr(b), _dptr(x), _dptr(x0), _stream(stream),
               C.byref(res))
        return {"iterations": res.iterations, "outer": res.outer, "status": res.status,
                "rr": res.rr, "bb": res.bb}

    def vcycle_profile(self, reps: int = 10, stream=None) -> list:
        """Per-kernel profile of the AMG V-cycle: [{level, kind, ms, bytes}] in launch order."""
        return _vcycle_profile("gipb200_pcg_vcycle_profile", self.handle, reps, stream)

    def kernel_time(self, reps: int = 20, stream=None) -> tuple:
        """(mean ms, streamed bytes) of the solver's SpMV-dot kernel over `reps` launches."""
        ms, nb = C.c_double(), C.c_double()
        L.call("gipb200_pcg_kernel_time", self.handle, reps, _stream(stream), C.byref(ms),
               C.byref(nb))
        return ms.value, nb.value

    def info(self) -> dict:
        i = L.PcgInfo()
        L.call("gipb200_pcg_get_info", self.handle, C.byref(i))
        return {k: getattr(i, k) for k, _ in L.PcgInfo._fields_}

    def close(self):
        if getattr(self, "handle", None):
            L.load().gipb200_pcg_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cg_update_dot(A: DeviceMatrix, n: int, x, r, z, p, q, dinv, sc: torch.Tensor, stream=None):
    """alpha = rz/pAp; x += alpha p; r -= alpha q; z = dinv r; rz, rr, beta into `sc`
    (a float64 device tensor laid out as gipb200_cg_scalars: rz, pAp, alpha, beta, rr)."""
    L.call("gipb200_cg_update_dot", A.handle, n, _dptr(x), _dptr(r), _dptr(z), _dptr(p),
           _dptr(q), _dptr(dinv), _dptr(sc), _stream(stream))


def cg_direction(n: int, p, z, sc: torch.Tensor, stream=None):
    """p = z + beta p, beta from `sc` on the device."""
    L.call("gipb200_cg_direction", n, _dptr(p), _dptr(z), _dptr(sc), _stream(stream))


def host_loop_pcg(A: DeviceMatrix, Dg: DeviceMatrix, dinv: torch.Tensor, b: torch.Tensor,
                  x: torch.Tensor, x0: torch.Tensor, maxit: int, stream=None) -> torch.Tensor:
    """GIP_LinearSolver::solve (GIP_LinearSolver.h:44-117) driven from the host over the fused
    entry points: the set-up with GIP's copies, SpMV and axpy, the Jacobi application as
    the diagonal operator `Dg`'s SpMV fused with r.z, then `maxit` iterations of
    spmv_dot / cg_update_dot / cg_direction with no host wait.  x (n_all) receives the
    solution; returns the device scalars (rz, pAp, alpha, beta, rr)."""
    n, n_all = A.nrows, x.numel()
    s = _stream(stream)
    sc = torch.zeros(5, dtype=torch.float64, device=x.device)
    p = x0.clone()                     # dp = x0 (ALL)
    Ax = x0.clone()                    # dAx = x0 (ALL)
    r = torch.empty(n_all, dtype=torch.float64, device=x.device)
    r[:n] = b[:n]                      # dr = b (INNER)
    z = torch.zeros(n_all, dtype=torch.float64, device=x.device)
    x.copy_(x0)                        # dx = x0 (ALL)
    A.spmv(x, Ax, stream=stream)       # dAx = A x
    L.call("gipb200_daxpy", n, _dptr(r), _dptr(Ax), -1.0, s)  # dr += -1 dAx
    Dg.spmv_dot(r, p, sc, n_dot=n, stream=stream)              # dp = D r; r1 = r.dp
    pAp = C.c_void_p(sc.data_ptr() + 8)
    for _ in range(maxit):
        L.call("gipb200_matrix_spmv_dot", A.handle, _dptr(p), _dptr(Ax), n, pAp, s)
        cg_update_dot(A, n, x, r, z, p, Ax, dinv, sc, stream)
        cg_direction(n, p, z, sc, stream)
    return sc


# ----------------------------------------------------------------------------- timestep
class DnsEngine:
    """``GIP_DNS`` on the device: ``advance(n)`` is ``integrate()`` for n timesteps."""

    def __init__(self, case: Optional[GipCase], rho: float = 1.0, gamma: float = 1e-3,
                 pcg_mode: str = "fixed", maxit: int = 100, tol: float = 1e-6,
                 inner_tol: float = 1e-3, inner_maxit: int = 2000, max_outer: int = 30,
                 use_graph: bool = True, reorder: bool = False, precond: str = "jacobi",
                 _handle=None, _sizes=None):
        self._owned = _handle is None
        if _handle is not None:  # a view of an engine owned elsewhere (a batch instance)
            self.handle = _handle
            self.n_inner, self.n_owned, self.n_faces = _sizes
            return
        lib = L.load()
        keep: list = []
        ops = L.DnsOps(**{n: _host_csr(case.ops[n], keep) for n in L.DNS_OPS},
                       n_inner=case.n_inner, n_owned=case.n_owned, n_faces=case.n_faces)
        f = {k: np.ascontiguousarray(case.fields[k], np.float64) for k in ("u", "v", "w", "dxs")}
        self.params = L.DnsParams(rho, gamma, pcg_params(pcg_mode, maxit, tol, inner_tol,
                                                         inner_maxit, max_outer, precond),
                                  int(use_graph), int(reorder))
        handle = C.c_void_p()
        L.check(lib.gipb200_dns_create(C.byref(ops), _hptr(f["u"]), _hptr(f["v"]), _hptr(f["w"]),
                                       _hptr(f["dxs"]), C.byref(self.params), C.byref(handle)),
                "gipb200_dns_create")
        self.handle = handle
        self.n_inner, self.n_owned, self.n_faces = case.n_inner, case.n_owned, case.n_faces

    def advance(self, nsteps: int, stream=None) -> None:
        L.call("gipb200_dns_advance", self.handle, nsteps, _stream(stream))

    def history(self) -> Dict[str, np.ndarray]:
        steps = C.c_int()
        L.call("gipb200_dns_history", self.handle, C.byref(steps), None, None, None, None, None,
               None, None)
        n = steps.value
        out = {"time": np.zeros(n), "dt": np.zeros(n), "massr": np.zeros(n),
               "iters": np.zeros(n, np.int32), "rr": np.zeros(n), "outer": np.zeros(n, np.int32),
               "kernels": np.zeros(n, np.int32)}
        L.call("gipb200_dns_history", self.handle, C.byref(steps), _hptr(out["time"]),
               _hptr(out["dt"]), _hptr(out["massr"]), _hptr(out["iters"]), _hptr(out["rr"]),
               _hptr(out["outer"]), _hptr(out["kernels"]))
        return out

    PHASES = ("predictor", "poisson_rhs", "pcg", "ghost_copy", "correction", "mass_fluxes",
              "cfl")

    def step_phases(self, stream=None) -> Dict[str, float]:
        """Advance one timestep (host-driven loops) and return each GIP_DNS phase's ms."""
        out = np.zeros(7)
        L.call("gipb200_dns_step_phases", self.handle, _stream(stream), _hptr(out))
        return dict(zip(self.PHASES, out.tolist()))

    def phase_stamps(self, on: bool = True) -> None:
        """Stamp the device clock at every step's phase boundaries (graph steps included)."""
        L.call("gipb200_dns_phase_stamps", self.handle, int(bool(on)))

    def phase_history(self) -> Dict[str, np.ndarray]:
        """Per-step phase durations in ms (NaN for steps taken with stamps off)."""
        steps = C.c_int()
        L.call("gipb200_dns_history", self.handle, C.byref(steps), None, None, None, None, None,
               None, None)
        out = np.zeros((steps.value, 7))
        got = C.c_int()
        L.call("gipb200_dns_phase_history", self.handle, steps.value, _hptr(out), C.byref(got))
        out = out[:got.value]
        return {name: out[:, k].copy() for k, name in enumerate(self.PHASES)}

    def field(self, name: str) -> np.ndarray:
        n = self.n_faces if name == "mf" else self.n_owned
        out = np.zeros(n)
        L.call("gipb200_dns_get_field", self.handle, name.encode(), _hptr(out), n)
        return out

    def field_ptr(self, name: str) -> tuple:
        p = C.c_void_p()
        n = C.c_int()
        L.call("gipb200_dns_field_ptr", self.handle, name.encode(), C.byref(p), C.byref(n))
        return p.value, n.value

    def copy_field(self, name: str, out: torch.Tensor, stream=None) -> torch.Tensor:
        """Device-to-device copy of a field in the caller's numbering into `out` (float64,
        at least the field's length), on `stream` with no host wait."""
        if out.dtype != torch.float64 or not out.is_cuda:
            raise TypeError("out must be a float64 device tensor")
        L.call("gipb200_dns_copy_field", self.handle, name.encode(), _dptr(out), out.numel(),
               _stream(stream))
        return out

    def set_time(self, time: float, stream=None) -> None:
        """Set the simulated time (GIP_DNS's `time` member)."""
        L.call("gipb200_dns_set_time", self.handle, float(time), _stream(stream))

    def set_field(self, name: str, values: np.ndarray, offset: int = 0, stream=None) -> None:
        """Asynchronous host->device copy into a field (keep `values` alive and, for a
        truly asynchronous copy, pinned, until the stream has passed it)."""
        if values.dtype != np.float64 or not values.flags.c_contiguous:
            raise TypeError("values must be a contiguous float64 array")
        L.call("gipb200_dns_set_field", self.handle, name.encode(), _hptr(values), offset,
               values.size, _stream(stream))

    def vcycle_profile(self, reps: int = 10, stream=None) -> list:
        """Per-kernel profile of the AMG V-cycle: [{level, kind, ms, bytes}] in launch order."""
        return _vcycle_profile("gipb200_dns_vcycle_profile", self.handle, reps, stream)

    def setup_profile(self) -> Dict[str, float]:
        """Host seconds of the engine's creation by stage."""
        out = np.zeros(4)
        L.call("gipb200_dns_setup_profile", self.handle, _hptr(out))
        return dict(zip(("renumbering", "operators", "solver", "total"), out.tolist()))

    def phase_bytes(self) -> Dict[str, float]:
        """Algorithmic bytes of each timestep phase (the PCG's is 0: see info())."""
        out = np.zeros(7)
        L.call("gipb200_dns_phase_bytes", self.handle, _hptr(out))
        return dict(zip(self.PHASES, out.tolist()))

    def kernel_time(self, kernel: str = "mixed", reps: int = 20, stream=None) -> tuple:
        """Mean CUDA-event time (ms) and compulsory bytes of one PCG SpMV+dot launch."""
        kid = {"fp64": 0, "mixed": 1, "mixed_update": 2}[kernel]
        ms, by = C.c_double(), C.c_double()
        L.call("gipb200_dns_kernel_time", self.handle, kid, reps, _stream(stream), C.byref(ms),
               C.byref(by))
        return ms.value, by.value

    def launch_count(self) -> int:
        c = C.c_longlong()
        L.call("gipb200_dns_launch_count", self.handle, C.byref(c))
        return c.value

    def scalars(self) -> dict:
        dt, sg, t = C.c_double(), C.c_double(), C.c_double()
        L.call("gipb200_dns_scalars", self.handle, C.byref(dt), C.byref(sg), C.byref(t))
        return {"dt": dt.value, "sigma": sg.value, "time": t.value}

    def info(self) -> dict:
        i = L.DnsInfo()
        L.call("gipb200_dns_get_info", self.handle, C.byref(i))
        return {k: getattr(i, k) for k, _ in L.DnsInfo._fields_}

    def snapshot(self, restore: bool = False, stream=None) -> None:
        """Save (or restore) the whole timestep state on the device."""
        L.call("gipb200_dns_snapshot", self.handle, int(restore), _stream(stream))

    def set_launch(self, spmv_blocks: int = 0, vec_blocks: int = 0) -> None:
        L.call("gipb200_dns_set_launch", self.handle, spmv_blocks, vec_blocks)

    def close(self):
        if getattr(self, "handle", None) and getattr(self, "_owned", True):
            L.load().gipb200_dns_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def dns_params(rho: float = 1.0, gamma: float = 1e-3, pcg_mode: str = "fixed", maxit: int = 100,
               tol: float = 1e-6, inner_tol: float = 1e-3, inner_maxit: int = 2000,
               max_outer: int = 30, use_graph: bool = True, reorder: bool = False,
               precond: str = "jacobi") -> L.DnsParams:
    return L.DnsParams(rho, gamma, pcg_params(pcg_mode, maxit, tol, inner_tol, inner_maxit,
                                              max_outer, precond), int(use_graph), int(reorder))


class DnsBatch:
    """Many independent cases advanced together: one graph launch per timestep whose
    parallel branches are the instances' steps (each with its own convergence loops)."""

    def __init__(self, cases, params):
        n = len(cases)
        keep: list = []
        ops = [L.DnsOps(**{k: _host_csr(c.ops[k], keep) for k in L.DNS_OPS},
                        n_inner=c.n_inner, n_owned=c.n_owned, n_faces=c.n_faces) for c in cases]
        fields = [{k: np.ascontiguousarray(c.fields[k], np.float64)
                   for k in ("u", "v", "w", "dxs")} for c in cases]
        keep += fields
        OpsArr = C.POINTER(L.DnsOps) * n
        PtrArr = C.c_void_p * n
        ops_p = OpsArr(*[C.pointer(o) for o in ops])
        arr = {k: PtrArr(*[f[k].ctypes.data for f in fields]) for k in ("u", "v", "w", "dxs")}
        prm = (L.DnsParams * n)(*params)
        h = C.c_void_p()
        L.call("gipb200_batch_create", n, C.cast(ops_p, C.c_void_p), C.cast(arr["u"], C.c_void_p),
               C.cast(arr["v"], C.c_void_p), C.cast(arr["w"], C.c_void_p),
               C.cast(arr["dxs"], C.c_void_p), prm, C.byref(h))
        self.handle = h
        self.instances = []
        for i, c in enumerate(cases):
            d = C.c_void_p()
            L.call("gipb200_batch_instance", h, i, C.byref(d))
            self.instances.append(DnsEngine(None, _handle=d, _sizes=(c.n_inner, c.n_owned,
                                                                      c.n_faces)))

    def advance(self, nsteps: int, stream=None) -> None:
        L.call("gipb200_batch_advance", self.handle, nsteps, _stream(stream))

    def set_solver(self, persistent: bool, block: int = 256, rows_per_warp: int = 32,
                   threads_per_sm: int = 1024) -> None:
        """Pressure solves in one persistent cooperative launch per step (every instance
        mixed with Jacobi) or, persistent=False, inside each instance's graph branch."""
        L.call("gipb200_batch_set_solver", self.handle, int(persistent), int(block),
               int(rows_per_warp), int(threads_per_sm))

    def balance(self, weights=None) -> None:
        """CTA shares of the persistent solve (None: rows x rows^(1/3))."""
        if weights is None:
            L.call("gipb200_batch_balance", self.handle, None)
            return
        w = np.ascontiguousarray(weights, np.float64)
        L.call("gipb200_batch_balance", self.handle, w.ctypes.data)

    def layout(self):
        """(grid, CTAs per instance) of the persistent solve; (0, zeros) when off."""
        g = C.c_int()
        n = np.zeros(len(self.instances), np.int32)
        L.call("gipb200_batch_layout", self.handle, C.byref(g), n.ctypes.data)
        return g.value, n

    def solver_status(self, stream=None) -> int:
        """Nonzero when a barrier of the persistent solve gave up since the last call."""
        e = C.c_int()
        L.call("gipb200_batch_solver_status", self.handle, _stream(stream), C.byref(e))
        return e.value

    def close(self):
        if getattr(self, "handle", None):
            for e in self.instances:
                e.handle = None
            L.load().gipb200_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
