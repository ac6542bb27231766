"""The ctypes binding agrees with include/gipb200.h: parameter counts of every bound entry
point, and the field names, order and kinds of every struct that crosses the ABI.  A
mismatch here is the kind that corrupts the stack at run time, so it is caught on the host."""
import ctypes as C
import os
import re

import pytest

from gip_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "gipb200.h")


def _source():
    s = open(HEADER).read()
    s = re.sub(r"/\*.*?\*/", " ", s, flags=re.S)
    return re.sub(r"//[^\n]*", " ", s)


def _functions():
    out = {}
    for m in re.finditer(r"\b(gipb200_\w+)\s*\(([^;{]*?)\)\s*;", _source(), flags=re.S):
        params = " ".join(m.group(2).split())
        out[m.group(1)] = [] if params in ("", "void") else [p.strip() for p in params.split(",")]
    return out


def _structs():
    out = {}
    for m in re.finditer(r"typedef\s+struct\s*\{(.*?)\}\s*(\w+)\s*;", _source(), flags=re.S):
        fields = []
        for decl in m.group(1).split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            first, *rest = [d.strip() for d in decl.split(",")]
            words = first.replace("*", " * ").split()
            ctype = " ".join(words[:-1])
            fields.append((words[-1], ctype))
            for name in rest:
                fields.append((name.replace("*", "").strip(), ctype))
        out[m.group(2)] = fields
    return out


def test_every_bound_function_has_the_declared_arity():
    decl = _functions()
    bound = _lib._SIGNATURES
    assert set(bound) <= set(decl), sorted(set(bound) - set(decl))
    wrong = {n: (len(args), len(decl[n])) for n, (_, args) in bound.items()
             if len(args) != len(decl[n])}
    assert wrong == {}


def _c_kind(param: str, handles) -> str:
    if "*" in param:
        return "ptr"
    words = param.replace("const ", "").split()
    base = " ".join(words[:-1]) if len(words) > 1 else words[0]
    if base in handles:
        return "ptr"
    return {"int": "int", "double": "double", "int64_t": "i64", "long long": "i64",
            "size_t": "size"}[base]


def _py_kind(t) -> str:
    if t in (C.c_void_p, C.c_char_p) or (isinstance(t, type) and issubclass(t, C._Pointer)):
        return "ptr"
    return {C.c_int: "int", C.c_double: "double", C.c_longlong: "i64", C.c_int64: "i64",
            C.c_size_t: "size"}[t]


def test_every_bound_function_has_the_declared_argument_kinds():
    handles = set(re.findall(r"typedef\s+struct\s+\w+\s*\*\s*(\w+)\s*;", _source()))
    decl = _functions()
    wrong = {}
    for name, (_, args) in _lib._SIGNATURES.items():
        ck = [_c_kind(p, handles) for p in decl[name]]
        pk = [_py_kind(t) for t in args]
        if ck != pk:
            wrong[name] = (ck, pk)
    assert wrong == {}


def test_entry_points_used_by_the_python_api_are_bound():
    # the Python layer calls these by name through _lib.call / attribute access
    for name in ("gipb200_dns_phase_stamps", "gipb200_dns_phase_history",
                 "gipb200_amg_host_levels", "gipb200_pcg_solve_static", "gipb200_dns_history"):
        assert name in _lib._SIGNATURES, name


KIND = {"int": C.c_int, "double": C.c_double, "long long": C.c_longlong}
STRUCTS = {"gipb200_host_csr": _lib.HostCsr, "gipb200_dns_ops": _lib.DnsOps,
           "gipb200_pcg_params": _lib.PcgParams, "gipb200_pcg_result": _lib.PcgResult,
           "gipb200_dns_params": _lib.DnsParams, "gipb200_pcg_info": _lib.PcgInfo,
           "gipb200_dns_info": _lib.DnsInfo, "gipb200_adjoint_params": _lib.AdjointParams,
           "gipb200_cg_scalars": _lib.CgScalars}


@pytest.mark.parametrize("cname", sorted(STRUCTS))
def test_struct_layout_matches_header(cname):
    fields = _structs()[cname]
    py = STRUCTS[cname]._fields_
    assert [n for n, _ in fields] == [n for n, _ in py]
    for (name, ctype), (_, pytype) in zip(fields, py):
        if "*" in ctype:
            assert pytype is C.c_void_p, name
        elif ctype.replace("const ", "") in STRUCTS:
            assert pytype is STRUCTS[ctype.replace("const ", "")], name
        else:
            assert pytype is KIND[ctype], (name, ctype)


def _enums():
    vals = {}
    for body in re.findall(r"enum\s*\{(.*?)\}", _source(), flags=re.S):
        nxt = 0
        for item in body.split(","):
            item = item.strip()
            if not item:
                continue
            name, _, v = item.partition("=")
            nxt = int(v) if v.strip() else nxt
            vals[name.strip()] = nxt
            nxt += 1
    return vals


def test_enum_values_match_header():
    from gip_b200 import device
    e = _enums()
    assert [e[f"GIPB200_PCG_{m.upper()}"] for m in ("fixed", "tol", "mixed")] == \
        [device.MODES[m] for m in ("fixed", "tol", "mixed")]
    assert {k: e[f"GIPB200_PRECOND_{k.upper()}"] for k in device.PRECONDS} == device.PRECONDS
    assert [e[n] for n in ("GIPB200_OK", "GIPB200_ERR_ARG", "GIPB200_ERR_CUDA",
                           "GIPB200_ERR_BREAKDOWN", "GIPB200_ERR_TIMEOUT", "GIPB200_ERR_NOMEM",
                           "GIPB200_ERR_NOT_CONVERGED", "GIPB200_ERR_STATE")] == \
        [_lib.STATUS_OK, _lib.ERR_ARG, _lib.ERR_CUDA, _lib.ERR_BREAKDOWN, _lib.ERR_TIMEOUT,
         _lib.ERR_NOMEM, _lib.ERR_NOT_CONVERGED, _lib.ERR_STATE]


def test_parameter_builders():
    from gip_b200 import device
    p = device.pcg_params("mixed", maxit=50, tol=1e-7, inner_tol=0.01, max_outer=9,
                          precond="amg")
    assert (p.mode, p.maxit, p.tol, p.inner_tol, p.max_outer, p.precond) == \
        (_lib.PCG_MIXED, 50, 1e-7, 0.01, 9, 1)
    d = device.dns_params(gamma=0.0025, pcg_mode="tol", tol=1e-9, use_graph=False,
                          reorder=True)
    assert (d.rho, d.gamma, d.pcg.mode, d.pcg.tol, d.pcg.precond, d.use_graph, d.reorder) == \
        (1.0, 0.0025, _lib.PCG_TOL, 1e-9, 0, 0, 1)
    with pytest.raises(KeyError):
        device.pcg_params("cg")
    with pytest.raises(KeyError):
        device.pcg_params("tol", precond="ilu")
