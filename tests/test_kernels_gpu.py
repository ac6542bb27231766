"""Kernel parity on the device against the oracle (GIP's CPU semantics).

Element-wise results (SpMV rows, axpy, axpby, the CFL minimum and the infinity norm) are
compared bit for bit; dot products, whose summation order differs from GIP's sequential
loop, to 1e-13 relative."""
import numpy as np
import pytest
import torch

from gip_b200 import cavity, formats

pytestmark = pytest.mark.gpu


def _rand_csr(rng, nrows, ncols, maxlen, empty_frac=0.1):
    lens = rng.integers(0, maxlen + 1, nrows)
    lens[rng.random(nrows) < empty_frac] = 0
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    col = rng.integers(0, ncols, int(rp[-1])).astype(np.int32)  # unsorted, duplicates allowed
    val = rng.standard_normal(int(rp[-1]))
    return formats.Csr(nrows, ncols, rp, col, val)


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


CASES = [(1, 1, 1, 0.0), (5, 3, 0, 0.0), (37, 50, 9, 0.2), (1000, 1200, 13, 0.1),
         (70001, 70001, 7, 0.05)]


@pytest.mark.parametrize("nrows,ncols,maxlen,empty", CASES)
@pytest.mark.parametrize("mode", [0, 1])
def test_spmv_bitexact(gpu, oracle_mod, nrows, ncols, maxlen, empty, mode):
    from gip_b200 import device as dv
    rng = np.random.default_rng(nrows + 7 * mode)
    m = _rand_csr(rng, nrows, ncols, maxlen, empty)
    x = rng.standard_normal(ncols)
    y0 = rng.standard_normal(nrows)
    alpha, beta = 0.37, -1.25
    ref = oracle_mod.spmv(m, x, y0.copy(), alpha, beta, mode)
    # sliced handle
    A = dv.DeviceMatrix(m)
    y = _t(y0.copy())
    A.spmv(_t(x), y, alpha, beta, mode)
    assert np.array_equal(y.cpu().numpy(), ref)
    # raw CSR pointers (GIP_cudaDCsrSpMV counterpart)
    y2 = _t(y0.copy())
    dv.spmv_raw(_t(m.rowptr), _t(m.col) if m.nnz else _t(np.zeros(1, np.int32)),
                _t(m.val) if m.nnz else _t(np.zeros(1)), _t(x), y2, alpha, beta, mode)
    assert np.array_equal(y2.cpu().numpy(), ref)


def test_spmv_values_target(gpu, oracle_mod):
    from gip_b200 import device as dv
    case, _ = cavity.generate(5, re=100.0)
    D, Ec = case.ops["D"], case.ops["Ec"]
    mf = np.random.default_rng(3).standard_normal(case.n_faces)
    ref = oracle_mod.spmv(Ec, mf, D.val.copy())
    Cm = dv.DeviceMatrix(D)
    dv.DeviceMatrix(Ec).spmv_values(_t(mf), Cm)
    assert np.array_equal(Cm.values(), ref)
    # and the sliced copy follows: C u equals the oracle's
    u = np.random.default_rng(4).standard_normal(case.n_owned)
    Cref = formats.Csr(D.nrows, D.ncols, D.rowptr, D.col, ref)
    y = _t(np.zeros(D.nrows))
    Cm.spmv(_t(u), y)
    assert np.array_equal(y.cpu().numpy(), oracle_mod.spmv(Cref, u, np.zeros(D.nrows)))


@pytest.mark.parametrize("n", [1, 31, 4097, 1 << 20])
def test_vector_ops(gpu, oracle_mod, n):
    from gip_b200 import device as dv
    rng = np.random.default_rng(n)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    a, b = 0.3, -2.0
    ty = _t(y.copy())
    dv.axpy(ty, _t(x), a)
    yy = y.copy()
    for i in range(0, n, max(1, n // 4096)):
        pass
    ref = y + a * x  # numpy does not contract to FMA
    assert np.array_equal(ty.cpu().numpy(), ref)
    ty = _t(y.copy())
    dv.axpby(ty, _t(x), a, b)
    assert np.array_equal(ty.cpu().numpy(), a * x + b * y)
    d = dv.dot(_t(x), _t(y))
    r = oracle_mod.lib().orc_dot(n, x.ctypes.data_as(oracle_mod.C.c_void_p),
                                 y.ctypes.data_as(oracle_mod.C.c_void_p))
    assert abs(d - r) <= 1e-13 * max(1.0, np.abs(x * y).sum())
    assert dv.norminf(_t(x)) == np.abs(x).max()
    z = _t(np.zeros(n))
    dv.fill(z, 2.5)
    assert float(z.min()) == 2.5 == float(z.max())


def test_dot_deterministic(gpu):
    from gip_b200 import device as dv
    rng = np.random.default_rng(9)
    x, y = _t(rng.standard_normal(3_000_001)), _t(rng.standard_normal(3_000_001))
    vals = {dv.dot(x, y) for _ in range(5)}
    assert len(vals) == 1


@pytest.mark.parametrize("seed", [0, 1])
def test_cfl_bitexact(gpu, oracle_mod, seed):
    from gip_b200 import device as dv
    rng = np.random.default_rng(seed)
    n = 50_000
    u, v, w = (rng.standard_normal(n) * s for s in (1.0, 0.5, 2.0))
    u[:10] = 0.0
    v[:10] = 0.0
    w[:10] = 0.0  # zero velocity: only the diffusive limit applies
    dxs = rng.uniform(0.001, 0.02, n)
    C = oracle_mod.C
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    for gamma in (1e-3, 1e-2):
        ref = oracle_mod.lib().orc_cfl(n, P(u), P(v), P(w), P(dxs), C.c_double(gamma),
                                       C.c_double(1.0))
        got = dv.cfl(_t(u), _t(v), _t(w), _t(dxs), n, gamma, 1.0)
        assert got == ref


def test_inverse_diagonal(gpu, oracle_mod):
    from gip_b200 import device as dv
    case, _ = cavity.generate(6)
    L = case.ops["L"]
    d, miss = dv.DeviceMatrix(L).inverse_diagonal()
    assert miss == 0
    ref = np.zeros(L.nrows)
    lib, C = oracle_mod.lib(), oracle_mod.C
    keep = []
    s = oracle_mod._csr_struct(L, keep)
    lib.orc_inverse_diagonal(C.byref(s), ref.ctypes.data_as(C.c_void_p))
    assert np.array_equal(d.cpu().numpy(), ref)
