"""Parity at the benchmark definition's own sizes: the 128^3 pressure-Poisson solve
(FP64 and mixed forms at tol 1e-8) and the 32 uneven batched cavities (10 mixed steps).
The oracle restates GIP_LinearSolver::solve (GIP_LinearSolver.h:44-117) and GIP_DNS
(GIP_DNS.h:99-414) with a tolerance stopping rule."""
import numpy as np
import pytest
import torch

from gip_b200 import cavity

pytestmark = pytest.mark.gpu


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_config2_poisson_128_fp64_and_mixed(gpu, oracle_mod):
    """128^3 Neumann Laplacian with one pinned cell (2,097,152 rows), seeded RHS U[-1,1]
    minus its mean, tol 1e-8: the FP64 form takes the oracle's iteration count within one
    and meets the tolerance on the true residual; both mixed forms (Jacobi and AMG) meet it
    on the FP64 true residual and agree with the FP64 solution."""
    from gip_b200 import device as dv
    L, b = cavity.poisson_problem(128, seed=1234)
    assert L.nrows == 128 ** 3 and L.nnz == 14581760
    Ls = L.to_scipy()
    nb = np.linalg.norm(b)
    A = dv.DeviceMatrix(L)
    x0 = np.zeros(L.nrows)
    xr, it, _ = oracle_mod.pcg(L, b, x0, maxit=5000, mode=1, tol=1e-8)
    S = dv.PcgSolver(A, mode="tol", maxit=5000, tol=1e-8)
    x = _t(x0)
    res = S.solve(_t(b), x, _t(x0))
    assert res["status"] == 0
    assert abs(res["iterations"] - it) <= 1, (res["iterations"], it)
    xf = x.cpu().numpy()
    assert np.linalg.norm(b - Ls @ xf) <= 1.5e-8 * nb
    assert np.abs(xf - xr).max() / np.abs(xr).max() < 1e-6
    for kw in (dict(inner_tol=0.3, max_outer=400),
               dict(inner_tol=0.01, max_outer=400, precond="amg")):
        M = dv.PcgSolver(A, mode="mixed", maxit=20000, tol=1e-8, **kw)
        xm = _t(x0)
        rm = M.solve(_t(b), xm, _t(x0))
        assert rm["status"] == 0, (kw, rm)
        xm = xm.cpu().numpy()
        assert np.linalg.norm(b - Ls @ xm) <= 1.0001e-8 * nb, kw
        # both solutions are within the tolerance times the conditioning of each other
        assert np.linalg.norm(xm - xf) / np.linalg.norm(xf) < 1e-4, kw


def _batch_set(seed=1234):
    rng = np.random.default_rng(seed)
    edges = rng.choice([24, 32, 48, 64, 80, 96], size=32)
    res = np.exp(rng.uniform(np.log(100.0), np.log(1000.0), size=32))
    return [int(n) for n in edges], [float(r) for r in res]


@pytest.mark.slow
def test_config5_batch_32_uneven_cavities(gpu, oracle_mod):
    """The 32 seeded cavities (edges from {24..96}, Re log-uniform on [100, 1000]) advance 10
    mixed steps (tol 1e-8) in one batch, with AMG in the graph branches and with GIP's
    Jacobi in one persistent launch: every instance keeps massr < 1e-6 and its velocity
    within 1e-6 (of its velocity scale) of the FP64 form solved to 1e-10; the instances of
    edge <= 32 are checked against the FP64 oracle directly as well."""
    from gip_b200.device import DnsBatch, DnsEngine, dns_params
    edges, res = _batch_set()
    assert sorted(set(edges)) <= [24, 32, 48, 64, 80, 96] and len(edges) == 32
    cases = [cavity.generate(n, re=r)[0] for n, r in zip(edges, res)]
    kw = dict(maxit=20000, tol=1e-8, inner_tol=0.01, max_outer=400, reorder=True)
    params = [dns_params(gamma=1.0 / r, pcg_mode="mixed", precond="amg", **kw) for r in res]
    B = DnsBatch(cases, params)
    steps = 10
    B.advance(steps)
    # the same batch with GIP's Jacobi, every pressure solve in one persistent launch
    pj = [dns_params(gamma=1.0 / r, pcg_mode="mixed", precond="jacobi",
                     **dict(kw, inner_tol=0.3)) for r in res]
    P = DnsBatch(cases, pj)
    P.set_solver(True, 256, 64, 1536)
    P.advance(steps)
    torch.cuda.synchronize()
    assert P.solver_status() == 0
    checked_oracle = 0
    for c, n, r, e, ep in zip(cases, edges, res, B.instances, P.instances):
        h = e.history()
        assert len(h["massr"]) == steps and np.all(h["massr"] < 1e-6), (n, r, h["massr"])
        hp = ep.history()
        assert len(hp["massr"]) == steps and np.all(hp["massr"] < 1e-6), (n, r, hp["massr"])
        F = DnsEngine(c, gamma=1.0 / r, pcg_mode="tol", precond="amg",
                      **dict(kw, tol=1e-10))
        F.advance(steps)
        scale = np.abs(F.field("u")).max()
        for k in ("u", "v", "w"):
            err = np.abs(e.field(k) - F.field(k)).max() / scale
            assert err < 1e-6, (n, r, k, err)
            err = np.abs(ep.field(k) - F.field(k)).max() / scale
            assert err < 1e-6, ("persistent", n, r, k, err)
        del F
        if n <= 32:
            d = oracle_mod.OracleDNS(c, gamma=1.0 / r, cg_maxit=20000, cg_mode=1, cg_tol=1e-10)
            d.run(steps)
            for k in ("u", "v", "w"):
                err = np.abs(e.field(k) - d.vec[k]).max() / scale
                assert err < 1e-6, ("oracle", n, r, k, err)
            checked_oracle += 1
    assert checked_oracle >= 1
