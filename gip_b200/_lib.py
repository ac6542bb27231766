"""ctypes binding of ``libgipb200.so`` (the C ABI declared in ``include/gipb200.h``).

There is no CPU fallback: if the library cannot be loaded, importing the device API
raises.  Device memory and streams come from PyTorch; pointers cross the ABI as ints.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgipb200.so")


class GipB200Error(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        super().__init__(f"{where}: {message} (status {status})")
        self.status = status


class HostCsr(C.Structure):
    _fields_ = [("nrows", C.c_int), ("ncols", C.c_int), ("nnz", C.c_int),
                ("rowptr", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p)]


DNS_OPS = ("D", "Ec", "L", "Lb", "Mx", "My", "Mz", "Mres", "Gx", "Gy", "Gz",
           "SFx", "SFy", "SFz", "SO")


class DnsOps(C.Structure):
    _fields_ = [(n, HostCsr) for n in DNS_OPS] + [
        ("n_inner", C.c_int), ("n_owned", C.c_int), ("n_faces", C.c_int)]


class PcgParams(C.Structure):
    _fields_ = [("mode", C.c_int), ("maxit", C.c_int), ("tol", C.c_double),
                ("inner_tol", C.c_double), ("inner_maxit", C.c_int), ("max_outer", C.c_int),
                ("precond", C.c_int)]


class PcgResult(C.Structure):
    _fields_ = [("iterations", C.c_int), ("outer", C.c_int), ("status", C.c_int),
                ("rr", C.c_double), ("bb", C.c_double)]


class DnsParams(C.Structure):
    _fields_ = [("rho", C.c_double), ("gamma", C.c_double), ("pcg", PcgParams),
                ("use_graph", C.c_int), ("reorder", C.c_int)]


class PcgInfo(C.Structure):
    _fields_ = [("pin_row", C.c_int), ("compressed", C.c_int), ("value_table", C.c_int),
                ("compressed_fraction", C.c_double), ("amg_levels", C.c_int),
                ("amg_complexity", C.c_double), ("amg_setup_s", C.c_double),
                ("packed_residual", C.c_int)]


class DnsInfo(C.Structure):
    _fields_ = [("reordered", C.c_int), ("pin_row", C.c_int), ("compressed", C.c_int),
                ("value_table", C.c_int), ("compressed_fraction", C.c_double),
                ("slots_L", C.c_longlong), ("nnz_L", C.c_longlong), ("amg_levels", C.c_int),
                ("amg_complexity", C.c_double), ("amg_setup_s", C.c_double),
                ("iteration_bytes", C.c_double), ("replacement_bytes", C.c_double),
                ("packed_residual", C.c_int), ("value_tables", C.c_int)]


class CgScalars(C.Structure):
    _fields_ = [("rz", C.c_double), ("pAp", C.c_double), ("alpha", C.c_double),
                ("beta", C.c_double), ("rr", C.c_double)]


class AdjointParams(C.Structure):
    _fields_ = [("rho", C.c_double), ("gamma", C.c_double), ("nu0", C.c_double),
                ("tol", C.c_double), ("maxit", C.c_int), ("checkpoint_every", C.c_int),
                ("precond", C.c_int)]


PCG_FIXED, PCG_TOL, PCG_MIXED = 0, 1, 2
STATUS_OK, ERR_ARG, ERR_CUDA, ERR_BREAKDOWN, ERR_TIMEOUT, ERR_NOMEM, ERR_NOT_CONVERGED, \
    ERR_STATE = range(8)

_VP, _I, _D = C.c_void_p, C.c_int, C.c_double
_SIGNATURES = {
    "gipb200_version": (C.c_int, []),
    "gipb200_status_string": (C.c_char_p, [_I]),
    "gipb200_last_error": (C.c_char_p, []),
    "gipb200_set_device": (_I, [_I]),
    "gipb200_malloc": (_I, [C.POINTER(C.c_void_p), C.c_size_t]),
    "gipb200_free": (_I, [_VP]),
    "gipb200_memcpy_h2d": (_I, [_VP, _VP, C.c_size_t, _VP]),
    "gipb200_memcpy_d2h": (_I, [_VP, _VP, C.c_size_t, _VP]),
    "gipb200_memcpy_d2h_async": (_I, [_VP, _VP, C.c_size_t, _VP]),
    "gipb200_dcopy": (_I, [_I, _VP, _VP, _VP]),
    "gipb200_stream_sync": (_I, [_VP]),
    "gipb200_event_create": (_I, [C.POINTER(_VP)]),
    "gipb200_event_record": (_I, [_VP, _VP]),
    "gipb200_event_elapsed_ms": (_I, [_VP, _VP, C.POINTER(C.c_float)]),
    "gipb200_event_destroy": (_I, [_VP]),
    "gipb200_dcsr_spmv": (_I, [_I, _VP, _VP, _VP, _VP, _VP, _D, _D, _I, _VP]),
    "gipb200_daxpy": (_I, [_I, _VP, _VP, _D, _VP]),
    "gipb200_daxpby": (_I, [_I, _VP, _VP, _D, _D, _VP]),
    "gipb200_dfill": (_I, [_I, _VP, _D, _VP]),
    "gipb200_gather": (_I, [_I, _VP, _VP, _VP, _VP]),
    "gipb200_scatter": (_I, [_I, _VP, _VP, _VP, _VP]),
    "gipb200_ddot": (_I, [_I, _VP, _VP, C.POINTER(_D), _VP]),
    "gipb200_dnorminf": (_I, [_I, _VP, C.POINTER(_D), _VP]),
    "gipb200_cfl": (_I, [_I, _VP, _VP, _VP, _VP, _D, _D, C.POINTER(_D), _VP]),
    "gipb200_matrix_create": (_I, [_I, _I, _I, _VP, _VP, _VP, C.POINTER(_VP)]),
    "gipb200_matrix_destroy": (_I, [_VP]),
    "gipb200_matrix_info": (_I, [_VP, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I),
                                 C.POINTER(C.c_int64)]),
    "gipb200_matrix_spmv": (_I, [_VP, _VP, _VP, _D, _D, _I, _VP]),
    "gipb200_matrix_spmv_values": (_I, [_VP, _VP, _VP, _D, _D, _I, _VP]),
    "gipb200_matrix_get_values": (_I, [_VP, _VP]),
    "gipb200_matrix_inverse_diagonal": (_I, [_VP, _VP, C.POINTER(_I)]),
    "gipb200_matrix_spmv_dot": (_I, [_VP, _VP, _VP, _I, _VP, _VP]),
    "gipb200_cg_update_dot": (_I, [_VP, _I, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "gipb200_cg_direction": (_I, [_I, _VP, _VP, _VP, _VP]),
    "gipb200_pcg_create": (_I, [_VP, _I, C.POINTER(PcgParams), C.POINTER(_VP)]),
    "gipb200_pcg_destroy": (_I, [_VP]),
    "gipb200_pcg_get_info": (_I, [_VP, C.POINTER(PcgInfo)]),
    "gipb200_check_bounded_wait": (_I, [_VP, C.POINTER(_I)]),
    "gipb200_pcg_kernel_time": (_I, [_VP, _I, _VP, C.POINTER(_D), C.POINTER(_D)]),
    "gipb200_pcg_solve": (_I, [_VP, _VP, _VP, _VP, _VP, C.POINTER(PcgResult)]),
    "gipb200_pcg_solve_static": (_I, [_I, _I, _VP, _VP, _VP, _VP, _VP, _VP, _I, _I, _D, _VP,
                                      _VP]),
    "gipb200_adjoint_create": (_I, [C.POINTER(DnsOps), _VP, _VP, _VP, _VP, _VP, _VP, _I,
                                    C.POINTER(AdjointParams), C.POINTER(_VP)]),
    "gipb200_adjoint_destroy": (_I, [_VP]),
    "gipb200_adjoint_forward": (_I, [_VP, _VP, _D, _I, _VP, _I, C.POINTER(_D)]),
    "gipb200_adjoint_backward": (_I, [_VP, _VP, C.POINTER(_D)]),
    "gipb200_dns_set_launch": (_I, [_VP, _I, _I]),
    "gipb200_dns_snapshot": (_I, [_VP, _I, _VP]),
    "gipb200_dns_get_info": (_I, [_VP, C.POINTER(DnsInfo)]),
    "gipb200_batch_create": (_I, [_I, _VP, _VP, _VP, _VP, _VP, C.POINTER(DnsParams),
                                  C.POINTER(_VP)]),
    "gipb200_batch_destroy": (_I, [_VP]),
    "gipb200_batch_instance": (_I, [_VP, _I, C.POINTER(_VP)]),
    "gipb200_batch_advance": (_I, [_VP, _I, _VP]),
    "gipb200_batch_set_solver": (_I, [_VP, _I, _I, _I, _I]),
    "gipb200_batch_balance": (_I, [_VP, _VP]),
    "gipb200_batch_layout": (_I, [_VP, C.POINTER(_I), _VP]),
    "gipb200_batch_solver_status": (_I, [_VP, _VP, C.POINTER(_I)]),
    "gipb200_batch_check_bounded_wait": (_I, [_VP, C.POINTER(_I)]),
    "gipb200_dns_create": (_I, [C.POINTER(DnsOps), _VP, _VP, _VP, _VP, C.POINTER(DnsParams),
                                C.POINTER(_VP)]),
    "gipb200_dns_destroy": (_I, [_VP]),
    "gipb200_dns_advance": (_I, [_VP, _I, _VP]),
    "gipb200_dns_history": (_I, [_VP, C.POINTER(_I), _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "gipb200_dns_step_phases": (_I, [_VP, _VP, _VP]),
    "gipb200_dns_phase_stamps": (_I, [_VP, _I]),
    "gipb200_amg_host_levels": (_I, [_I, _VP, _VP, _VP, _VP, _I, C.c_double, _I, C.POINTER(_I),
                                     _VP, _VP, _VP]),
    "gipb200_dns_phase_history": (_I, [_VP, _I, _VP, C.POINTER(_I)]),
    "gipb200_dns_get_field": (_I, [_VP, C.c_char_p, _VP, _I]),
    "gipb200_dns_field_ptr": (_I, [_VP, C.c_char_p, C.POINTER(_VP), C.POINTER(_I)]),
    "gipb200_dns_copy_field": (_I, [_VP, C.c_char_p, _VP, _I, _VP]),
    "gipb200_dns_scalars": (_I, [_VP, C.POINTER(_D), C.POINTER(_D), C.POINTER(_D)]),
    "gipb200_dns_set_time": (_I, [_VP, _D, _VP]),
    "gipb200_dns_phase_bytes": (_I, [_VP, _VP]),
    "gipb200_dns_setup_profile": (_I, [_VP, _VP]),
    "gipb200_dns_vcycle_profile": (_I, [_VP, _I, _VP, _I, C.POINTER(_I), _VP, _VP, _VP, _VP]),
    "gipb200_pcg_vcycle_profile": (_I, [_VP, _I, _VP, _I, C.POINTER(_I), _VP, _VP, _VP, _VP]),
    "gipb200_dns_vcycle_forms": (_I, [_VP, _I, C.POINTER(_I), _VP]),
    "gipb200_pcg_vcycle_forms": (_I, [_VP, _I, C.POINTER(_I), _VP]),
    "gipb200_dns_set_field": (_I, [_VP, C.c_char_p, _VP, _I, _I, _VP]),
    "gipb200_dns_launch_count": (_I, [_VP, C.POINTER(C.c_longlong)]),
    "gipb200_dns_kernel_time": (_I, [_VP, _I, _I, _VP, C.POINTER(_D), C.POINTER(_D)]),
}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the library (building it first if the sources are present and it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        from . import build as _build
        _build.build()
    lib = C.CDLL(path)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, where: str) -> None:
    if status != STATUS_OK:
        lib = load()
        raise GipB200Error(status, where, lib.gipb200_last_error().decode(errors="replace"))


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args), name)


def declared_symbols(header: str = None) -> list:
    """Entry points declared in include/gipb200.h (for the export check)."""
    import re
    header = header or os.path.join(os.path.dirname(HERE), "include", "gipb200.h")
    txt = open(header).read()
    return sorted(set(re.findall(r"\b(gipb200_[a-z0-9_]+)\s*\(", txt)))
