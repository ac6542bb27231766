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
           "gipb200_dns_info": _lib.DnsInfo, "gipb200_adjoint_params": _lib.AdjointParams}


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
