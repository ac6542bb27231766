"""The allocation-free PCG entry point (gipb200_pcg_solve_static) against the handle-based
one (gipb200_pcg_solve).  Callers that cannot allocate device memory at solve time use
the static variant; it must give the same solution.  Collected last on purpose: its
scratch array lives for the whole process, so it runs after every other test here and
also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest
import torch

from gip_b200 import _lib, cavity

pytestmark = pytest.mark.gpu


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _static_solve(L, b, x0, n_all, mode, maxit, tol):
    # every device buffer stays referenced until the stream has finished with it
    rp, col, val = _t(L.rowptr), _t(L.col), _t(L.val)
    db, dx0 = _t(b), _t(x0)
    x = torch.zeros(n_all, dtype=torch.float64, device="cuda")
    stats = torch.zeros(4, dtype=torch.float64, device="cuda")
    P = lambda t: C.c_void_p(t.data_ptr())
    _lib.call("gipb200_pcg_solve_static", L.nrows, n_all, P(rp), P(col), P(val), P(db), P(x),
              P(dx0), mode, maxit, tol, P(stats), None)
    torch.cuda.synchronize()
    return x.cpu().numpy(), stats.cpu().numpy()


@pytest.mark.parametrize("mode", ["fixed", "tol"])
def test_static_pcg_matches_handle_pcg_twice(gpu, mode):
    from gip_b200 import device as dv
    case, _ = cavity.generate(20, re=400.0)           # L with ghost columns, n_all > n
    L = case.ops["L"]
    rng = np.random.default_rng(11)
    b = rng.standard_normal(L.nrows)
    x0 = rng.standard_normal(case.n_owned) * 0.1
    kw = dict(mode=mode, maxit=100 if mode == "fixed" else 4000, tol=1e-9)
    S = dv.PcgSolver(dv.DeviceMatrix(L), n_all=case.n_owned, **kw)
    xr = torch.zeros(case.n_owned, dtype=torch.float64, device="cuda")
    db, dx0 = _t(b), _t(x0)
    res = S.solve(db, xr, dx0)
    xr = xr.cpu().numpy()
    m = _lib.PCG_FIXED if mode == "fixed" else _lib.PCG_TOL
    for _ in range(2):  # two calls in a row share and reuse the static scratch
        xs, st = _static_solve(L, b, x0, case.n_owned, m, kw["maxit"], kw["tol"])
        assert int(st[3]) == 0
        assert abs(int(st[0]) - res["iterations"]) <= 1
        assert np.abs(xs - xr).max() / np.abs(xr).max() < 1e-10
        assert np.array_equal(xs[L.nrows:], x0[L.nrows:])


def test_static_pcg_rejects_oversize(gpu):
    n = 262145
    z = torch.zeros(1, dtype=torch.float64, device="cuda")
    zi = torch.zeros(1, dtype=torch.int32, device="cuda")
    P = lambda t: C.c_void_p(t.data_ptr())
    st = _lib.load().gipb200_pcg_solve_static(n, n, P(zi), P(zi), P(z), P(z), P(z), P(z),
                                              _lib.PCG_FIXED, 1, 0.0, P(z), None)
    assert st == _lib.ERR_ARG
    assert b"static scratch limit" in _lib.load().gipb200_last_error()
