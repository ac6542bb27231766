"""The allocation-free PCG entry point (gipb200_pcg_solve_static) against the handle-based
one (gipb200_pcg_solve).  Callers that cannot allocate device memory at solve time use
the static variant; it must give the same solution and must not allocate.  Collected
last on purpose: its scratch array lives for the whole process, so it runs after every
other test here and also passes alone in a fresh process."""
import ctypes as C
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest
import torch

from gip_b200 import _lib, cavity

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _P(t):
    return C.c_void_p(t.data_ptr())


def _problem():
    case, _ = cavity.generate(20, re=400.0)           # L with ghost columns, n_all > n
    L = case.ops["L"]
    rng = np.random.default_rng(11)
    b = rng.standard_normal(L.nrows)
    x0 = rng.standard_normal(case.n_owned) * 0.1
    return case, L, b, x0


def _handle_solve(L, b, x0, n_all, kw):
    from gip_b200 import device as dv
    S = dv.PcgSolver(dv.DeviceMatrix(L), n_all=n_all, **kw)
    xr = torch.zeros(n_all, dtype=torch.float64, device="cuda")
    res = S.solve(_t(b), xr, _t(x0))
    return xr.cpu().numpy(), res


@pytest.mark.parametrize("mode", ["fixed", "tol"])
def test_static_pcg_matches_handle_pcg_twice_without_allocating(gpu, mode):
    case, L, b, x0 = _problem()
    n_all = case.n_owned
    kw = dict(mode=mode, maxit=100 if mode == "fixed" else 4000, tol=1e-9)
    xr, res = _handle_solve(L, b, x0, n_all, kw)
    m = _lib.PCG_FIXED if mode == "fixed" else _lib.PCG_TOL
    # every device buffer exists before the first measurement and stays referenced
    rp, col, val, db, dx0 = _t(L.rowptr), _t(L.col), _t(L.val), _t(b), _t(x0)
    x = torch.zeros(n_all, dtype=torch.float64, device="cuda")
    stats = torch.zeros(4, dtype=torch.float64, device="cuda")
    args = lambda: (L.nrows, n_all, _P(rp), _P(col), _P(val), _P(db), _P(x), _P(dx0), m,
                    kw["maxit"], kw["tol"], _P(stats), None)
    _lib.call("gipb200_pcg_solve_static", *args())   # first call: symbol address, modules
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    torch0 = torch.cuda.memory_allocated()
    for _ in range(2):  # two calls in a row share and reuse the static scratch
        x.zero_()
        _lib.call("gipb200_pcg_solve_static", *args())
        torch.cuda.synchronize()
        st = stats.cpu().numpy()
        xs = x.cpu().numpy()
        assert int(st[3]) == 0
        assert abs(int(st[0]) - res["iterations"]) <= 1
        assert np.abs(xs - xr).max() / np.abs(xr).max() < 1e-10
        assert np.array_equal(xs[L.nrows:], x0[L.nrows:])
    assert torch.cuda.mem_get_info()[0] == free0      # no device allocation by the calls
    assert torch.cuda.memory_allocated() == torch0


def test_static_pcg_rejects_oversize(gpu):
    n = 262145
    z = torch.zeros(1, dtype=torch.float64, device="cuda")
    zi = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = _lib.load().gipb200_pcg_solve_static(n, n, _P(zi), _P(zi), _P(z), _P(z), _P(z), _P(z),
                                              _lib.PCG_FIXED, 1, 0.0, _P(z), None)
    assert st == _lib.ERR_ARG
    assert b"static scratch limit" in _lib.load().gipb200_last_error()


def test_static_pcg_first_call_on_a_nonblocking_stream_in_a_fresh_process(gpu):
    # the first call of a process resolves the array's address; its counter clear and
    # the solve must be ordered on the caller's stream even when that stream does not
    # synchronise with the legacy default stream
    code = textwrap.dedent("""
        import ctypes as C, sys
        import numpy as np, torch
        sys.path.insert(0, %r)
        sys.path.insert(0, %r)
        from test_zz_no_alloc import _problem, _handle_solve, _t, _P
        from gip_b200 import _lib
        torch.cuda.set_device(0)
        case, L, b, x0 = _problem()
        n_all = case.n_owned
        s = torch.cuda.Stream()          # created non-blocking by torch
        with torch.cuda.stream(s):
            rp, col, val, db, dx0 = _t(L.rowptr), _t(L.col), _t(L.val), _t(b), _t(x0)
            x = torch.full((n_all,), 7.0, dtype=torch.float64, device="cuda")
            stats = torch.zeros(4, dtype=torch.float64, device="cuda")
        _lib.call("gipb200_pcg_solve_static", L.nrows, n_all, _P(rp), _P(col), _P(val),
                  _P(db), _P(x), _P(dx0), _lib.PCG_TOL, 4000, 1e-9, _P(stats),
                  C.c_void_p(s.cuda_stream))
        s.synchronize()
        xs, st = x.cpu().numpy(), stats.cpu().numpy()
        xr, res = _handle_solve(L, b, x0, n_all, dict(mode="tol", maxit=4000, tol=1e-9))
        assert int(st[3]) == 0, st
        assert abs(int(st[0]) - res["iterations"]) <= 1, (st, res)
        err = np.abs(xs - xr).max() / np.abs(xr).max()
        assert err < 1e-10, err
        print("fresh-process static solve ok", int(st[0]), err)
    """) % (REPO, os.path.join(REPO, "tests"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-3000:]
    assert "fresh-process static solve ok" in r.stdout
