"""AMG setup on the host (no GPU): the library's hierarchy against the numpy restatement."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from amg_model import hierarchy
from gip_b200 import _lib, cavity


def _inner_operator(n: int):
    """The mixed form's inner system for the n^3 pressure operator: GIP's pinned diagonal
    removed (pure Neumann) and Jacobi-scaled, with its null vector."""
    L, _ = cavity.poisson_problem(n, seed=1)
    A = L.to_scipy().tocsr()
    d = A.diagonal()
    rs = np.asarray(A.sum(axis=1)).ravel()
    p = int(np.argmax(np.abs(rs)))
    A = A.tolil()
    A[p, p] -= rs[p]
    s = 1.0 / np.sqrt(d)
    Ah = (sp.diags(s) @ A.tocsr() @ sp.diags(s)).tocsr()
    return Ah, 1.0 / s


def _levels(A: sp.csr_matrix, z, singular: int, drop: float, max_levels: int = 16):
    lib = _lib.load()
    rp = np.ascontiguousarray(A.indptr, np.int32)
    ci = np.ascontiguousarray(A.indices, np.int32)
    v = np.ascontiguousarray(A.data, np.float64)
    z = np.ascontiguousarray(z, np.float64)
    lv = C.c_int()
    rows = np.zeros(max_levels, np.int32)
    nnz = np.zeros(max_levels, np.int64)
    checks = np.zeros(3 * max_levels)
    st = lib.gipb200_amg_host_levels(A.shape[0], rp.ctypes.data, ci.ctypes.data, v.ctypes.data,
                                     z.ctypes.data, singular, drop, max_levels, C.byref(lv),
                                     rows.ctypes.data, nnz.ctypes.data, checks.ctypes.data)
    _lib.check(st, "gipb200_amg_host_levels")
    k = lv.value
    return rows[:k].tolist(), nnz[:k].tolist(), checks[:3 * k].reshape(k, 3)


@pytest.mark.parametrize("n,drop", [(12, 0.0), (12, 0.02), (20, 0.0), (20, 0.02), (20, 0.1)])
def test_hierarchy_matches_model(n, drop):
    A, z = _inner_operator(n)
    rows, nnz, chk = _levels(A, z, 1, drop)
    ref = hierarchy(A, z, drop)
    assert list(zip(rows, nnz)) == ref
    assert rows[-1] <= 1024 and all(a > b for a, b in zip(rows, rows[1:]))
    # Galerkin and sparsified operators stay symmetric (exactly, once sparsified) and keep
    # annihilating the near-null vector; diagonals stay positive
    for l, (asym, null, dmin) in enumerate(chk):
        assert asym <= (0.0 if (drop > 0 and l > 0) else 1e-14), (l, asym)
        assert null <= 1e-12, (l, null)
        assert dmin > 0.0, (l, dmin)


def test_sparsification_lowers_coarse_nonzeros():
    A, z = _inner_operator(24)
    _, nnz0, _ = _levels(A, z, 1, 0.0)
    _, nnz2, _ = _levels(A, z, 1, 0.02)
    assert nnz2[0] == nnz0[0] and nnz2[1] < 0.8 * nnz0[1]
    assert sum(nnz2) / nnz2[0] < sum(nnz0) / nnz0[0]


def test_definite_operator_with_constant_vector():
    # the FP64 tolerance mode: GIP's pinned (definite) operator, constants as near-null vector
    L, _ = cavity.poisson_problem(16, seed=2)
    A = L.to_scipy().tocsr()
    rows, nnz, chk = _levels(A, np.ones(A.shape[0]), 0, 0.02)
    assert list(zip(rows, nnz)) == hierarchy(A, np.ones(A.shape[0]), 0.02)
    assert (chk[:, 2] > 0).all()


def test_max_levels_and_bad_arguments():
    A, z = _inner_operator(12)
    rows, _, _ = _levels(A, z, 1, 0.02, max_levels=1)
    assert rows == [A.shape[0]]
    lib = _lib.load()
    bad = np.ascontiguousarray(A.indices, np.int32).copy()
    bad[3] = A.shape[0] + 5  # a column past the operator
    rp = np.ascontiguousarray(A.indptr, np.int32)
    v = np.ascontiguousarray(A.data)
    lv = C.c_int()
    out = np.zeros(4, np.int32), np.zeros(4, np.int64), np.zeros(12)
    st = lib.gipb200_amg_host_levels(A.shape[0], rp.ctypes.data, bad.ctypes.data, v.ctypes.data,
                                     z.ctypes.data, 1, 0.02, 4, C.byref(lv), out[0].ctypes.data,
                                     out[1].ctypes.data, out[2].ctypes.data)
    assert st == _lib.ERR_ARG
    assert b"out of" in lib.gipb200_last_error()
    st = lib.gipb200_amg_host_levels(0, rp.ctypes.data, bad.ctypes.data, v.ctypes.data,
                                     z.ctypes.data, 1, 0.02, 4, C.byref(lv), out[0].ctypes.data,
                                     out[1].ctypes.data, out[2].ctypes.data)
    assert st == _lib.ERR_ARG
