"""PCG parity: fixed iterations (GIP's solver), tolerance mode, mixed precision."""
import numpy as np
import pytest
import torch

from gip_b200 import cavity

pytestmark = pytest.mark.gpu


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("n,maxit", [(6, 5), (10, 100), (16, 37)])
def test_pcg_fixed_matches_oracle(gpu, oracle_mod, n, maxit):
    from gip_b200 import device as dv
    L, b = cavity.poisson_problem(n, seed=n)
    x0 = np.random.default_rng(1).standard_normal(L.nrows) * 0.1
    xr, it, rr = oracle_mod.pcg(L, b, x0, maxit=maxit, mode=0)
    S = dv.PcgSolver(dv.DeviceMatrix(L), mode="fixed", maxit=maxit)
    x = _t(np.zeros(L.nrows))
    res = S.solve(_t(b), x, _t(x0))
    assert res["iterations"] == it == maxit
    err = np.abs(x.cpu().numpy() - xr).max() / np.abs(xr).max()
    assert err < 1e-10, err


def test_pcg_fixed_with_ghost_columns(gpu, oracle_mod):
    # the cavity's L carries stored-zero ghost columns and warm-starts from an n_all x0
    from gip_b200 import device as dv
    case, _ = cavity.generate(7, re=100.0)
    L = case.ops["L"]
    rng = np.random.default_rng(5)
    b = rng.standard_normal(L.nrows)
    x0 = rng.standard_normal(case.n_owned)
    xr, it, rr = oracle_mod.pcg(L, b, x0, maxit=100, mode=0)
    S = dv.PcgSolver(dv.DeviceMatrix(L), n_all=case.n_owned, mode="fixed", maxit=100)
    x = _t(np.zeros(case.n_owned))
    S.solve(_t(b), x, _t(x0))
    got = x.cpu().numpy()
    assert np.array_equal(got[L.nrows:], x0[L.nrows:])  # ghosts keep x0 (GIP_LinearSolver.h:67)
    assert np.abs(got - xr).max() / np.abs(xr).max() < 1e-10


@pytest.mark.parametrize("n,tol", [(12, 1e-6), (20, 1e-8)])
def test_pcg_tol_iterations_within_one(gpu, oracle_mod, n, tol):
    from gip_b200 import device as dv
    L, b = cavity.poisson_problem(n, seed=3)
    x0 = np.zeros(L.nrows)
    xr, it, rr = oracle_mod.pcg(L, b, x0, maxit=5000, mode=1, tol=tol)
    S = dv.PcgSolver(dv.DeviceMatrix(L), mode="tol", maxit=5000, tol=tol)
    x = _t(np.zeros(L.nrows))
    res = S.solve(_t(b), x, _t(x0))
    assert res["status"] == 0
    assert abs(res["iterations"] - it) <= 1, (res["iterations"], it)
    r = b - L.to_scipy() @ x.cpu().numpy()
    assert np.linalg.norm(r) <= 1.5 * tol * np.linalg.norm(b)


@pytest.mark.parametrize("n,tol", [(16, 1e-6), (24, 1e-8)])
def test_pcg_mixed_reaches_fp64_tolerance(gpu, oracle_mod, n, tol):
    from gip_b200 import device as dv
    L, b = cavity.poisson_problem(n, seed=4)
    S = dv.PcgSolver(dv.DeviceMatrix(L), mode="mixed", maxit=5000, tol=tol, inner_tol=1e-3,
                     inner_maxit=2000, max_outer=40)
    x = _t(np.zeros(L.nrows))
    res = S.solve(_t(b), x, _t(np.zeros(L.nrows)))
    assert res["status"] == 0, res
    xs = x.cpu().numpy()
    r = b - L.to_scipy() @ xs
    assert np.linalg.norm(r) <= tol * np.linalg.norm(b) * 1.0001
    # against the FP64 oracle solved tighter: solution error is bounded by conditioning
    xr, _, _ = oracle_mod.pcg(L, b, np.zeros(L.nrows), maxit=20000, mode=1, tol=1e-13)
    assert np.abs(xs - xr).max() / np.abs(xr).max() < 1e4 * tol


def _anisotropic_pinned(nx, ny, nz, w=(1.0, 2.5, 0.6), extra=30, seed=0):
    """Pinned-Neumann graph Laplacian of an nx*ny*nz grid with direction weights w, plus
    `extra` rows coupled to three random far cells (rows of 9-10 nonzeros), pinned as GIP
    pins its pressure operator (L_00 += L_00 / 101)."""
    import scipy.sparse as sp
    from gip_b200.formats import Csr
    N = nx * ny * nz
    idx = np.arange(N).reshape(nz, ny, nx)
    rows, cols, vals = [], [], []
    for ax, ww in zip((2, 1, 0), w):
        a = np.take(idx, range(0, idx.shape[ax] - 1), axis=ax).ravel()
        b = np.take(idx, range(1, idx.shape[ax]), axis=ax).ravel()
        rows += [a, b]
        cols += [b, a]
        vals += [np.full(a.size, -ww)] * 2
    rng = np.random.default_rng(seed)
    for h in rng.choice(N, extra, replace=False):
        o = rng.choice(N, 3, replace=False)
        o = o[o != h]
        rows += [np.full(o.size, h), o]
        cols += [o, np.full(o.size, h)]
        vals += [np.full(o.size, -0.3)] * 2
    A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(N, N)).tocsr()
    A.sum_duplicates()
    A = (A + sp.diags(-np.asarray(A.sum(axis=1)).ravel())).tolil()
    A[0, 0] += A[0, 0] / 101.0
    A = A.tocsr()
    A.sort_indices()
    return Csr(N, N, A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.copy())


def test_mixed_packed_operator_8bit_table_and_plain_slices(gpu, monkeypatch):
    # ~100 distinct FP32 values (8-bit table) and rows longer than 8 slots (plain slices):
    # the packed kernel, its plain fallback and the unpacked kernel give identical solves
    from gip_b200 import device as dv
    L = _anisotropic_pinned(20, 18, 16)
    rng = np.random.default_rng(9)
    b = rng.standard_normal(L.nrows)
    kw = dict(mode="mixed", maxit=5000, tol=1e-9, inner_tol=0.1, max_outer=100)
    S = dv.PcgSolver(dv.DeviceMatrix(L), **kw)
    info = S.info()
    assert info["compressed"] == 1 and info["value_table"] == 8 and info["pin_row"] == 0
    assert 0.5 < info["compressed_fraction"] < 1.0
    monkeypatch.setenv("GIPB200_NO_COMPRESS", "1")
    P = dv.PcgSolver(dv.DeviceMatrix(L), **kw)
    assert P.info()["compressed"] == 0
    xs, xp = _t(np.zeros(L.nrows)), _t(np.zeros(L.nrows))
    rs = S.solve(_t(b), xs, _t(np.zeros(L.nrows)))
    rp = P.solve(_t(b), xp, _t(np.zeros(L.nrows)))
    assert rs["status"] == 0 and (rs["iterations"], rs["outer"]) == (rp["iterations"], rp["outer"])
    assert torch.equal(xs, xp)
    r = b - L.to_scipy() @ xs.cpu().numpy()
    assert np.linalg.norm(r) <= 1e-9 * np.linalg.norm(b) * 1.0001


@pytest.mark.parametrize("mode", ["tol", "mixed"])
def test_pcg_reports_breakdown_and_nonconvergence(gpu, mode):
    # failures come back as statuses (no device trap): a non-finite right-hand side is a
    # breakdown, an iteration cap below what the tolerance needs is non-convergence
    from gip_b200 import device as dv
    L, b = cavity.poisson_problem(10, seed=2)
    A = dv.DeviceMatrix(L)
    kw = dict(inner_tol=0.3, max_outer=50) if mode == "mixed" else {}
    S = dv.PcgSolver(A, mode=mode, maxit=3, tol=1e-12, **kw)
    x = _t(np.zeros(L.nrows))
    assert S.solve(_t(b), x, _t(np.zeros(L.nrows)))["status"] == 6  # NOT_CONVERGED
    bad = b.copy()
    bad[17] = np.nan
    S2 = dv.PcgSolver(A, mode=mode, maxit=500, tol=1e-8, **kw)
    assert S2.solve(_t(bad), x, _t(np.zeros(L.nrows)))["status"] == 3  # BREAKDOWN
    res = S2.solve(_t(b), x, _t(np.zeros(L.nrows)))  # the solver is still usable
    assert res["status"] == 0


def test_bounded_wait_gives_up_with_status(gpu):
    # a barrier wait that nothing completes times out and reports; the context stays usable
    import ctypes as C
    from gip_b200 import _lib
    from gip_b200 import device as dv
    st = C.c_int(-1)
    _lib.call("gipb200_check_bounded_wait", None, C.byref(st))
    assert st.value == 4  # GIPB200_ERR_TIMEOUT
    L, b = cavity.poisson_problem(6, seed=1)
    S = dv.PcgSolver(dv.DeviceMatrix(L), mode="tol", maxit=500, tol=1e-8)
    assert S.solve(_t(b), _t(np.zeros(L.nrows)), _t(np.zeros(L.nrows)))["status"] == 0


@pytest.mark.parametrize("n,tol", [(20, 1e-8), (33, 1e-6)])
def test_mixed_amg_preconditioner(gpu, oracle_mod, n, tol):
    # the AMG V-cycle (FP32) inside the mixed form: the FP64 true residual meets the
    # tolerance in a few dozen iterations where Jacobi-scaled CG needs hundreds, and the
    # solution agrees with the FP64 oracle solved tighter
    from gip_b200 import device as dv
    L, b = cavity.poisson_problem(n, seed=4)
    A = dv.DeviceMatrix(L)
    S = dv.PcgSolver(A, mode="mixed", maxit=2000, tol=tol, inner_tol=1e-3, max_outer=100,
                     precond="amg")
    info = S.info()
    assert info["amg_levels"] >= 2 and info["pin_row"] >= 0
    x = _t(np.zeros(L.nrows))
    res = S.solve(_t(b), x, _t(np.zeros(L.nrows)))
    J = dv.PcgSolver(A, mode="mixed", maxit=20000, tol=tol, inner_tol=0.3, max_outer=400)
    rj = J.solve(_t(b), _t(np.zeros(L.nrows)), _t(np.zeros(L.nrows)))
    assert res["status"] == 0, res
    assert res["iterations"] < 60 and res["iterations"] * 5 < rj["iterations"], (res, rj)
    xs = x.cpu().numpy()
    assert np.linalg.norm(b - L.to_scipy() @ xs) <= tol * np.linalg.norm(b) * 1.0001
    xr, _, _ = oracle_mod.pcg(L, b, np.zeros(L.nrows), maxit=20000, mode=1, tol=1e-13)
    assert np.abs(xs - xr).max() / np.abs(xr).max() < 1e4 * tol


def test_amg_coarse_sparsification_thresholds(gpu, monkeypatch):
    # coarse operators lose their weak couplings (lumped onto the diagonal): fewer stored
    # nonzeros at the default threshold, and a large threshold still builds (rows whose
    # diagonal would lose more than half keep their couplings) and converges (its sparser
    # level 1 aggregates into more, denser levels below, so complexity is not monotone)
    from gip_b200 import device as dv
    L, b = cavity.poisson_problem(40, seed=7)
    A = dv.DeviceMatrix(L)
    cx = {}
    for th in ("0", "0.02", "0.1"):
        monkeypatch.setenv("GIPB200_AMG_DROP", th)
        S = dv.PcgSolver(A, mode="mixed", maxit=2000, tol=1e-8, inner_tol=1e-3, max_outer=100,
                         precond="amg")
        cx[th] = S.info()["amg_complexity"]
        x = _t(np.zeros(L.nrows))
        res = S.solve(_t(b), x, _t(np.zeros(L.nrows)))
        assert res["status"] == 0 and res["iterations"] < 200, (th, res)
        xs = x.cpu().numpy()
        assert np.linalg.norm(b - L.to_scipy() @ xs) <= 1e-8 * np.linalg.norm(b) * 1.0001, th
    assert cx["0.02"] < cx["0"], cx


def test_fp64_amg_preconditioner_and_fixed_mode_refusal(gpu, oracle_mod):
    # FP64 tolerance mode with the FP64 V-cycle; FIXED mode (GIP's) keeps GIP's Jacobi
    from gip_b200 import _lib
    from gip_b200 import device as dv
    L, b = cavity.poisson_problem(24, seed=5)
    A = dv.DeviceMatrix(L)
    with pytest.raises(_lib.GipB200Error):
        dv.PcgSolver(A, mode="fixed", maxit=10, precond="amg")
    S = dv.PcgSolver(A, mode="tol", maxit=2000, tol=1e-10, precond="amg")
    x = _t(np.zeros(L.nrows))
    res = S.solve(_t(b), x, _t(np.zeros(L.nrows)))
    xr, it, _ = oracle_mod.pcg(L, b, np.zeros(L.nrows), maxit=20000, mode=1, tol=1e-10)
    assert res["status"] == 0 and res["iterations"] * 5 < it, (res, it)
    xs = x.cpu().numpy()
    assert np.linalg.norm(b - L.to_scipy() @ xs) <= 1.5e-10 * np.linalg.norm(b)
    assert np.abs(xs - xr).max() / np.abs(xr).max() < 1e-6


@pytest.mark.parametrize("coarse_half", [False, True])
def test_amg_compact_coarse_operators(gpu, monkeypatch, coarse_half):
    # the FP32 cycle's long-row operators stored with 16-bit column offsets from each row's
    # base column (exact), optionally with FP16 coarse values (a slightly different, still
    # symmetric preconditioner): the solve meets the same tolerance on the FP64 true
    # residual in about the same number of iterations as with 32-bit columns
    from gip_b200 import device as dv
    L, b = cavity.poisson_problem(48, seed=9)
    A = dv.DeviceMatrix(L)
    its = {}
    for wide in ("1", "0"):
        if wide == "0":  # the compact forms (opt-in)
            monkeypatch.setenv("GIPB200_AMG_COMPACT", "1")
            if coarse_half:
                monkeypatch.setenv("GIPB200_AMG_COARSE_HALF", "1")
        S = dv.PcgSolver(A, mode="mixed", maxit=2000, tol=1e-8, inner_tol=1e-2, max_outer=100,
                         precond="amg")
        x = _t(np.zeros(L.nrows))
        res = S.solve(_t(b), x, _t(np.zeros(L.nrows)))
        assert res["status"] == 0, (wide, res)
        xs = x.cpu().numpy()
        assert np.linalg.norm(b - L.to_scipy() @ xs) <= 1.0001e-8 * np.linalg.norm(b), wide
        its[wide] = res["iterations"]
    if coarse_half:
        assert abs(its["0"] - its["1"]) <= max(2, its["1"] // 10), its
    else:  # 16-bit columns alone change nothing
        assert its["0"] == its["1"], its


def test_amg_coarse_tail_is_exact(gpu, monkeypatch):
    # the small levels run as one cooperative launch: every row is still summed by one warp
    # with the separate kernels' row functions, so the solve is identical, bit for bit
    from gip_b200 import device as dv
    L, b = cavity.poisson_problem(48, seed=4)
    A = dv.DeviceMatrix(L)
    out = {}
    for tail in (True, False):
        if tail:
            monkeypatch.setenv("GIPB200_AMG_TAIL", "2")
        else:
            monkeypatch.delenv("GIPB200_AMG_TAIL", raising=False)
        S = dv.PcgSolver(A, mode="mixed", maxit=2000, tol=1e-9, inner_tol=1e-2, max_outer=100,
                         precond="amg")
        x = _t(np.zeros(L.nrows))
        res = S.solve(_t(b), x, _t(np.zeros(L.nrows)))
        assert res["status"] == 0, (tail, res)
        prof = S.vcycle_profile(reps=2)
        out[tail] = (x.cpu().numpy(), res["iterations"], [c["kind"] for c in prof])
        # each kernel names the form it ran in: the tail launch, the packed level 0
        kern = [c["kernel"] for c in prof]
        assert ("k_amg_tail" in kern) == tail, kern
        assert prof[0]["kernel"] == "k_amgp_spmv" and prof[-1]["kernel"] == "k_amgp_spmv", kern
    assert "tail" in out[True][2] and "tail" not in out[False][2]
    assert out[True][1] == out[False][1]
    assert np.array_equal(out[True][0], out[False][0])
