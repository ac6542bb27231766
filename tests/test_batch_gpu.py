"""Batched uneven cavities: one graph launch per step, instances converge independently;
every instance equals the same case run alone (same kernels, same launch shapes)."""
import numpy as np
import pytest

from gip_b200 import cavity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["tol", "mixed"])
def test_batch_equals_single_runs(gpu, mode):
    from gip_b200.device import DnsBatch, DnsEngine, dns_params
    specs = [(6, 100.0), (10, 400.0), (8, 1000.0)]
    cases = [cavity.generate(n, re=re)[0] for n, re in specs]
    kw = dict(pcg_mode=mode, maxit=4000, tol=1e-8, inner_tol=0.1, max_outer=200)
    params = [dns_params(gamma=1.0 / re, **kw) for _, re in specs]
    B = DnsBatch(cases, params)
    B.advance(4)
    for c, (n, re), e in zip(cases, specs, B.instances):
        single = DnsEngine(c, gamma=1.0 / re, **kw)
        single.advance(4)
        hb, hs = e.history(), single.history()
        assert hb["iters"].tolist() == hs["iters"].tolist()
        for k in ("u", "v", "w", "p", "mf"):
            assert np.array_equal(e.field(k), single.field(k)), (n, k)


def test_autotune_picks_a_grid(gpu):
    from gip_b200 import autotune
    from gip_b200.device import DnsEngine
    case, _ = cavity.generate(24, re=400.0)
    E = DnsEngine(case, gamma=1.0 / 400, pcg_mode="mixed", maxit=4000, tol=1e-6, inner_tol=0.1,
                  max_outer=200)
    E.advance(1)
    r = autotune.tune(E, "mixed", rows=case.n_inner, nnz=case.ops["L"].nnz)
    assert r["blocks"] > 0
    E.advance(2)  # the re-captured step still converges
    assert np.all(E.history()["massr"] < 1e-4)


@pytest.mark.parametrize("block,rows_per_warp,occ", [(256, 32, 1024), (128, 64, 1024),
                                                     (512, 32, 1536), (128, 64, 1536)])
def test_persistent_solve_matches_branch_solves(gpu, block, rows_per_warp, occ):
    """The persistent launch (one CTA group per instance, the group's own convergence loop)
    against the same batch solving inside its graph branches: same algorithm (mixed
    Jacobi-PCG with reliable updates), so the steps agree to the solve's tolerance; every
    group barrier completed."""
    from gip_b200.device import DnsBatch, dns_params
    specs = [(6, 100.0), (10, 400.0), (8, 1000.0), (12, 250.0)]
    cases = [cavity.generate(n, re=re, permute_seed=7)[0] for n, re in specs]
    kw = dict(pcg_mode="mixed", maxit=4000, tol=1e-10, inner_tol=0.3, max_outer=200)
    params = [dns_params(gamma=1.0 / re, **kw) for _, re in specs]
    A = DnsBatch(cases, params)
    A.advance(5)
    B = DnsBatch(cases, params)
    B.set_solver(True, block, rows_per_warp, occ)
    grid, ncta = B.layout()
    assert grid > 0 and ncta.min() >= 1 and ncta.sum() <= grid
    B.advance(5)
    assert B.solver_status() == 0
    for (n, re), ea, eb in zip(specs, A.instances, B.instances):
        ha, hb = ea.history(), eb.history()
        assert np.all(hb["massr"] < 1e-6), (n, hb["massr"])
        assert np.all(np.abs(hb["iters"] - ha["iters"]) <= 0.1 * ha["iters"] + 3), (n, ha, hb)
        assert np.allclose(hb["time"], ha["time"], rtol=1e-7, atol=0)
        scale = np.abs(ea.field("u")).max()
        for k in ("u", "v", "w"):
            err = np.abs(eb.field(k) - ea.field(k)).max() / scale
            assert err < 1e-8, (n, k, err)
    # one launch for the whole batch's solves, counted on the first instance
    k0 = B.instances[0].history()["kernels"]
    k1 = B.instances[1].history()["kernels"]
    assert np.all(k0 == 11) and np.all(k1 == 10)


def test_persistent_balance_keeps_graph(gpu):
    """New CTA shares take effect in the already-captured step graph."""
    from gip_b200.device import DnsBatch, dns_params
    specs = [(8, 100.0), (14, 1000.0)]
    cases = [cavity.generate(n, re=re)[0] for n, re in specs]
    kw = dict(pcg_mode="mixed", maxit=4000, tol=1e-8, inner_tol=0.3, max_outer=200)
    B = DnsBatch(cases, [dns_params(gamma=1.0 / re, **kw) for _, re in specs])
    B.set_solver(True, 256, 32)
    B.advance(2)
    g0, n0 = B.layout()
    B.balance([1.0, 0.0])  # the second instance gets the minimum share
    g1, n1 = B.layout()
    assert g1 == g0 and n1[1] == 1 and n1[0] > n0[0] - 1
    B.advance(2)
    assert B.solver_status() == 0
    for e in B.instances:
        assert np.all(e.history()["massr"] < 1e-6)


def test_persistent_barrier_wait_is_bounded(gpu):
    """A group barrier that can never complete (the group claims a CTA that does not
    exist) gives up after its bounded spin, records the timeout and returns; the context
    stays usable."""
    import ctypes as C

    import torch

    from gip_b200 import _lib
    st = C.c_int(-1)
    _lib.call("gipb200_batch_check_bounded_wait", None, C.byref(st))
    assert st.value == _lib.ERR_TIMEOUT
    x = torch.ones(1024, device="cuda")
    assert float(x.sum()) == 1024.0
