"""The standalone fused CG entry points (gipb200_matrix_spmv_dot, gipb200_cg_update_dot,
gipb200_cg_direction) against the oracle: GIP's per-iteration sequence
(GIP_LinearSolver.h:85-116) driven from the host over the three calls must give GIP's
iterates, and each call must keep GIP's element rounding."""
import numpy as np
import pytest
import torch

from gip_b200 import cavity, formats

pytestmark = pytest.mark.gpu


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("nrows,ncols,maxlen,empty", [(1, 1, 1, 0.0), (37, 50, 9, 0.3),
                                                      (20011, 20011, 8, 0.05)])
def test_spmv_dot_rows_bitexact_dot_close(gpu, oracle_mod, nrows, ncols, maxlen, empty):
    from gip_b200 import device as dv
    rng = np.random.default_rng(nrows)
    lens = rng.integers(0, maxlen + 1, nrows)
    lens[rng.random(nrows) < empty] = 0
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    col = rng.integers(0, ncols, int(rp[-1])).astype(np.int32)
    m = formats.Csr(nrows, ncols, rp, col, rng.standard_normal(int(rp[-1])))
    x = rng.standard_normal(max(ncols, nrows))
    y0 = rng.standard_normal(nrows)
    ref = oracle_mod.spmv(m, x[:ncols], y0.copy())          # empty rows keep y0
    A = dv.DeviceMatrix(m)
    y = _t(y0.copy())
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    n_dot = nrows - nrows // 3
    A.spmv_dot(_t(x), y, out, n_dot=n_dot)
    got = y.cpu().numpy()
    assert np.array_equal(got, ref)
    want = float(np.dot(x[:n_dot], ref[:n_dot]))
    assert abs(out.item() - want) <= 1e-13 * max(1.0, np.abs(x[:n_dot] * ref[:n_dot]).sum())


def test_cg_update_and_direction_match_gip_steps(gpu):
    from gip_b200 import device as dv
    rng = np.random.default_rng(4)
    n = 10007
    # any handle with >= n rows supplies the reduction scratch
    big = formats.Csr(n, 1, np.zeros(n + 1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    A = dv.DeviceMatrix(big)
    x, r, p, q = (rng.standard_normal(n) for _ in range(4))
    dinv = rng.uniform(0.5, 2.0, n)
    rz0, pAp = 3.25, 1.75
    sc = _t(np.array([rz0, pAp, 0.0, 0.0, 0.0]))
    dx, dr, dz = _t(x), _t(r), torch.zeros(n, dtype=torch.float64, device="cuda")
    dv.cg_update_dot(A, n, dx, dr, dz, _t(p), _t(q), _t(dinv), sc)
    alpha = rz0 / pAp
    xr = x + alpha * p
    rr_ = r + (-alpha) * q
    zr = 0.0 + rr_ * dinv
    assert np.array_equal(dx.cpu().numpy(), xr)
    assert np.array_equal(dr.cpu().numpy(), rr_)
    assert np.array_equal(dz.cpu().numpy(), zr)
    s = sc.cpu().numpy()
    assert s[2] == alpha
    assert abs(s[0] - np.dot(rr_, zr)) <= 1e-12 * np.abs(rr_ * zr).sum()
    assert abs(s[4] - np.dot(rr_, rr_)) <= 1e-12 * np.dot(rr_, rr_)
    assert s[3] == s[0] / rz0
    dp = _t(p)
    dv.cg_direction(n, dp, dz, sc)
    assert np.array_equal(dp.cpu().numpy(), 1.0 * zr + s[3] * p)


def _diag_csr(L, n_all):
    d = np.zeros(L.nrows)
    has = np.zeros(L.nrows, bool)
    for i in range(L.nrows):
        for k in range(L.rowptr[i], L.rowptr[i + 1]):
            if L.col[k] == i:
                d[i] = 1.0 / L.val[k]
                has[i] = True
    rows = np.nonzero(has)[0]
    rp = np.concatenate([[0], np.cumsum(has)]).astype(np.int32)
    return formats.Csr(L.nrows, n_all, rp, rows.astype(np.int32), d[rows]), d


@pytest.mark.parametrize("n,maxit", [(7, 100), (12, 37)])
def test_host_loop_pcg_matches_oracle_and_handle_pcg(gpu, oracle_mod, n, maxit):
    """GIP's solver loop on the host over the fused calls equals the oracle's fixed-count
    PCG (GIP_LinearSolver.h:44-117) and the device-resident handle PCG."""
    from gip_b200 import device as dv
    case, _ = cavity.generate(n, re=100.0)    # L with stored-zero ghost columns
    L = case.ops["L"]
    rng = np.random.default_rng(n)
    b = rng.standard_normal(L.nrows)
    x0 = rng.standard_normal(case.n_owned) * 0.1
    xr, it, rr = oracle_mod.pcg(L, b, x0, maxit=maxit, mode=0)
    A = dv.DeviceMatrix(L)
    Dm, dinv = _diag_csr(L, case.n_owned)
    Dg = dv.DeviceMatrix(Dm)
    x = torch.zeros(case.n_owned, dtype=torch.float64, device="cuda")
    sc = dv.host_loop_pcg(A, Dg, _t(dinv), _t(b), x, _t(x0), maxit)
    got = x.cpu().numpy()
    assert np.array_equal(got[L.nrows:], x0[L.nrows:])
    assert np.abs(got - xr).max() / np.abs(xr).max() < 1e-10
    # r.r of the last iteration: equal up to rounding relative to b.b (the solve may reach
    # machine precision, where r.r itself is noise)
    assert abs(sc[4].item() - rr) <= 1e-8 * rr + 1e-24 * float(np.dot(b, b))
    S = dv.PcgSolver(A, n_all=case.n_owned, mode="fixed", maxit=maxit)
    xh = torch.zeros_like(x)
    S.solve(_t(b), xh, _t(x0))
    assert np.abs(xh.cpu().numpy() - got).max() / np.abs(got).max() < 1e-12
