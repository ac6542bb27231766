"""Timestep parity: the device engine against the oracle and GIP's own goldens."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_lines, have_c100k, rel_err
from gip_b200 import cavity

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "p", "p0", "mf", "ax0")


def _lines(oracle, h):
    return [oracle.format_line(h["time"][i], h["dt"][i], h["massr"][i], i + 1)
            for i in range(len(h["time"]))]


@pytest.mark.skipif(not have_c100k(), reason="merged C100K set not built")
@pytest.mark.parametrize("graph,reorder", [(True, False), (False, False), (True, True)])
def test_c100k_readme_golden(gpu, oracle_mod, c100k_case, graph, reorder):
    from gip_b200.device import DnsEngine
    E = DnsEngine(c100k_case, gamma=1e-3, pcg_mode="fixed", maxit=100, use_graph=graph,
                  reorder=reorder)
    E.advance(10)
    h = E.history()
    assert _lines(oracle_mod, h) == golden_lines("c100k_readme.txt")
    d = oracle_mod.OracleDNS(c100k_case, gamma=1e-3)
    d.run(10)
    for k in FIELDS:
        assert rel_err(E.field(k), d.vec[k]) < 1e-10, k


@pytest.mark.parametrize("n", [8, 12])
def test_fields_match_reference_goldens(gpu, n):
    from gip_b200.device import DnsEngine
    g = np.load(os.path.join(GOLDEN, f"cavity{n}_ref.npz"))
    case, _ = cavity.generate(n, re=float(g["re"]))
    E = DnsEngine(case, gamma=1.0 / float(g["re"]))
    E.advance(int(g["steps"]))
    h = E.history()
    assert h["iters"].tolist() == [100] * int(g["steps"])
    ref_dt = [float(l.split("[dt::")[1].split("]")[0]) for l in g["lines"]]
    assert np.allclose(h["dt"], ref_dt, rtol=1e-6)
    for k in FIELDS:
        assert rel_err(E.field(k)[: g[k].size], g[k]) < 1e-10, k


@pytest.mark.parametrize("n,re,seed,reorder", [(10, 100.0, None, False), (9, 1000.0, 11, False),
                                               (9, 1000.0, 11, True), (12, 400.0, None, True)])
def test_engine_matches_oracle_stepwise(gpu, oracle_mod, n, re, seed, reorder):
    from gip_b200.device import DnsEngine
    case, _ = cavity.generate(n, re=re, permute_seed=seed)
    E = DnsEngine(case, gamma=1.0 / re, reorder=reorder)
    d = oracle_mod.OracleDNS(case, gamma=1.0 / re)
    for chunk in (3, 4):
        E.advance(chunk)
        d.run(chunk)
        for k in FIELDS:
            assert rel_err(E.field(k), d.vec[k]) < 1e-10, k
    h = E.history()
    assert len(h["time"]) == 7
    assert E.scalars()["time"] == pytest.approx(d.time, rel=1e-12)


@pytest.mark.parametrize("graph,reorder", [(True, False), (False, False), (True, True)])
def test_engine_tol_mode_iterations(gpu, oracle_mod, graph, reorder):
    from gip_b200.device import DnsEngine
    case, _ = cavity.generate(16, re=400.0)
    E = DnsEngine(case, gamma=1.0 / 400, pcg_mode="tol", maxit=3000, tol=1e-8, use_graph=graph,
                  reorder=reorder)
    E.advance(5)
    d = oracle_mod.OracleDNS(case, gamma=1.0 / 400, cg_maxit=3000, cg_mode=1, cg_tol=1e-8)
    hr = d.run(5)
    h = E.history()
    assert np.all(np.abs(h["iters"] - hr["iters"]) <= 1), (h["iters"], hr["iters"])
    for k in ("u", "p"):
        assert rel_err(E.field(k), d.vec[k]) < 1e-7, k


@pytest.mark.parametrize("graph,reorder", [(True, False), (False, False), (True, True)])
def test_engine_mixed_close_to_fp64(gpu, oracle_mod, graph, reorder):
    from gip_b200.device import DnsEngine
    case, _ = cavity.generate(16, re=400.0)
    E = DnsEngine(case, gamma=1.0 / 400, pcg_mode="mixed", maxit=3000, tol=1e-8,
                  inner_tol=1e-3, use_graph=graph, reorder=reorder)
    E.advance(5)
    d = oracle_mod.OracleDNS(case, gamma=1.0 / 400, cg_maxit=3000, cg_mode=1, cg_tol=1e-10)
    d.run(5)
    h = E.history()
    assert np.all(h["massr"] < 1e-6)
    for k in ("u", "v", "w"):
        assert rel_err(E.field(k), d.vec[k]) < 1e-6, k
    # recorded launches: 10 phase kernels, the first residual, then per FP32 iteration
    # SpMV + update (graph: apply + residual only per replacement; host loop: every
    # iteration), plus a few that found the solve done (graph: at most one body of 4
    # kernels and its 2 replacement bodies; host loop: up to 15 iterations before the
    # next poll)
    if graph:
        base, slack = 11 + 2 * h["iters"] + 2 * h["outer"], 8
    else:
        base, slack = 11 + 4 * h["iters"], 60
    assert np.all(h["kernels"] >= base) and np.all(h["kernels"] <= base + slack), h["kernels"]


def test_set_and_copy_field_roundtrip_reordered(gpu):
    import torch
    from gip_b200.device import DnsEngine
    case, meta = cavity.generate(6, re=100.0, permute_seed=2)
    E = DnsEngine(case, gamma=1e-2, reorder=True)
    u = E.field("u")
    assert np.array_equal(u, case.fields["u"])
    lid = np.full(36, 0.5)
    off = case.n_inner + 5 * 36
    E.set_field("u", lid, offset=off)
    torch.cuda.synchronize()
    u2 = E.field("u")
    assert np.array_equal(u2[off:off + 36], lid) and np.array_equal(u2[:off], u[:off])
    d = torch.zeros(case.n_owned, dtype=torch.float64, device="cuda")
    from gip_b200 import _lib
    import ctypes
    _lib.call("gipb200_dns_copy_field", E.handle, b"u", ctypes.c_void_p(d.data_ptr()),
              case.n_owned, None)
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy(), u2)


def test_compressed_fp32_operator_is_exact(gpu, monkeypatch):
    # the compressed layout streams fewer bytes but computes the same products (both
    # engines take the FP64 residual from L's sliced layout: the packed FP64 residual sums
    # in another order and has its own test)
    from gip_b200.device import DnsEngine
    case, _ = cavity.generate(20, re=400.0, permute_seed=4)
    kw = dict(gamma=1.0 / 400, pcg_mode="mixed", maxit=5000, tol=1e-8, inner_tol=0.1,
              max_outer=200, reorder=True)
    monkeypatch.setenv("GIPB200_NO_PACKED_RESIDUAL", "1")
    E = DnsEngine(case, **kw)
    info = E.info()
    assert info["compressed"] == 1 and info["value_table"] == 4 and info["pin_row"] >= 0
    assert info["compressed_fraction"] == 1.0 and info["packed_residual"] == 0
    monkeypatch.setenv("GIPB200_NO_COMPRESS", "1")
    P = DnsEngine(case, **kw)
    assert P.info()["compressed"] == 0
    for X in (E, P):
        X.advance(3)
    assert E.history()["iters"].tolist() == P.history()["iters"].tolist()
    for k in ("u", "v", "w", "p", "mf"):
        assert np.array_equal(E.field(k), P.field(k)), k


@pytest.mark.parametrize("mode", ["fixed", "mixed"])
def test_snapshot_restore_replays_exactly(gpu, mode):
    from gip_b200.device import DnsEngine
    case, _ = cavity.generate(12, re=400.0)
    E = DnsEngine(case, gamma=1.0 / 400, pcg_mode=mode, maxit=100 if mode == "fixed" else 4000,
                  tol=1e-8, inner_tol=0.1, max_outer=200)
    E.advance(2)
    E.snapshot()
    E.advance(3)
    first = {k: E.field(k) for k in ("u", "p", "mf")}
    h1 = E.history()
    E.snapshot(restore=True)
    E.advance(3)
    h2 = E.history()
    assert len(h2["time"]) == 5 and np.array_equal(h1["massr"], h2["massr"])
    for k, v in first.items():
        assert np.array_equal(E.field(k), v), k


@pytest.mark.parametrize("graph", [True, False])
def test_engine_mixed_amg_close_to_fp64(gpu, oracle_mod, graph):
    from gip_b200.device import DnsEngine
    case, _ = cavity.generate(16, re=400.0, permute_seed=7)
    E = DnsEngine(case, gamma=1.0 / 400, pcg_mode="mixed", maxit=3000, tol=1e-8,
                  inner_tol=1e-3, max_outer=100, use_graph=graph, reorder=True, precond="amg")
    assert E.info()["amg_levels"] >= 2
    E.advance(5)
    d = oracle_mod.OracleDNS(case, gamma=1.0 / 400, cg_maxit=3000, cg_mode=1, cg_tol=1e-10)
    hr = d.run(5)
    h = E.history()
    assert np.all(h["massr"] < 1e-6)
    assert np.all(h["iters"] * 4 < hr["iters"]), (h["iters"], hr["iters"])
    for k in ("u", "v", "w"):
        assert rel_err(E.field(k), d.vec[k]) < 1e-6, k


def test_engine_fp64_amg_matches_oracle(gpu, oracle_mod):
    from gip_b200.device import DnsEngine
    case, _ = cavity.generate(14, re=400.0)
    E = DnsEngine(case, gamma=1.0 / 400, pcg_mode="tol", maxit=3000, tol=1e-10, precond="amg")
    E.advance(4)
    d = oracle_mod.OracleDNS(case, gamma=1.0 / 400, cg_maxit=3000, cg_mode=1, cg_tol=1e-12)
    hr = d.run(4)
    h = E.history()
    assert np.all(h["iters"] * 4 < hr["iters"]), (h["iters"], hr["iters"])
    for k in ("u", "v", "w"):
        assert rel_err(E.field(k), d.vec[k]) < 1e-8, k
    # device-counted launches: per step 10 + init + 2 per iteration + the V-cycles' kernels
    assert np.all(h["kernels"] > 11 + 2 * h["iters"])


def test_amg_packed_level0_is_exact(gpu, monkeypatch):
    # the V-cycle's level-0 products from the packed operator equal the plain layout's
    from gip_b200.device import DnsEngine
    case, _ = cavity.generate(18, re=400.0, permute_seed=3)
    kw = dict(gamma=1.0 / 400, pcg_mode="mixed", maxit=3000, tol=1e-8, inner_tol=1e-2,
              max_outer=100, reorder=True, precond="amg")
    monkeypatch.setenv("GIPB200_NO_PACKED_RESIDUAL", "1")  # the same FP64 residual in both
    E = DnsEngine(case, **kw)
    assert E.info()["compressed"] == 1
    monkeypatch.setenv("GIPB200_NO_COMPRESS", "1")
    P = DnsEngine(case, **kw)
    assert P.info()["compressed"] == 0
    E.advance(3)
    P.advance(3)
    assert E.history()["iters"].tolist() == P.history()["iters"].tolist()
    for k in ("u", "v", "w", "p"):
        assert np.array_equal(E.field(k), P.field(k)), k


@pytest.mark.parametrize("mode", ["fixed", "mixed"])
def test_value_tables_are_exact(gpu, monkeypatch, mode):
    """The phase kernels reading their operators' values through 8-bit value tables produce
    the same doubles as reading them directly: identical steps, every field equal."""
    from gip_b200.device import DnsEngine
    case, _ = cavity.generate(24, re=400.0, permute_seed=5)
    kw = dict(gamma=1.0 / 400, pcg_mode=mode, maxit=400 if mode == "fixed" else 3000, tol=1e-8,
              inner_tol=0.1, max_outer=100, reorder=True)
    E = DnsEngine(case, **kw)
    assert E.info()["value_tables"] == 4
    monkeypatch.setenv("GIPB200_NO_VALUE_TABLE", "1")
    P = DnsEngine(case, **kw)
    assert P.info()["value_tables"] == 0
    E.advance(4)
    P.advance(4)
    assert E.history()["iters"].tolist() == P.history()["iters"].tolist()
    assert np.array_equal(E.history()["massr"], P.history()["massr"])
    for k in ("u", "v", "w", "p", "mf", "ax0", "rhs", "gpx", "gpy", "gpz", "temp"):
        assert np.array_equal(E.field(k), P.field(k)), k


@pytest.mark.parametrize("pipe", ["0", "1"])
def test_amg_pipelined_products_are_exact(gpu, monkeypatch, pipe):
    """The software-pipelined sliced V-cycle products (next batch loaded before the current
    one's gathers) compute the same sums in the same order: identical steps whether no
    sliced operator (0), the long-row ones (default) or all of them (1) run pipelined.
    64^3 has more slices than warps at level 0, so warps walk several slices and batches."""
    from gip_b200.device import DnsEngine
    case, _ = cavity.generate(64, re=400.0, permute_seed=3)
    kw = dict(gamma=1.0 / 400, pcg_mode="mixed", maxit=3000, tol=1e-8, inner_tol=1e-2,
              max_outer=100, reorder=True, precond="amg")
    E = DnsEngine(case, **kw)
    monkeypatch.setenv("GIPB200_AMG_PIPE", pipe)
    P = DnsEngine(case, **kw)
    E.advance(2)
    P.advance(2)
    assert E.history()["iters"].tolist() == P.history()["iters"].tolist()
    for k in ("u", "v", "w", "p"):
        assert np.array_equal(E.field(k), P.field(k)), k


def test_step_phases_report_and_advance_like_a_step(gpu):
    # the per-phase report times a real step: same state as a graph-launched step
    from gip_b200.device import DnsEngine
    case, _ = cavity.generate(10, re=400.0)
    E = DnsEngine(case, gamma=1.0 / 400, pcg_mode="tol", maxit=2000, tol=1e-9)
    G = DnsEngine(case, gamma=1.0 / 400, pcg_mode="tol", maxit=2000, tol=1e-9)
    E.advance(2)
    G.advance(2)
    ph = E.step_phases()
    G.advance(1)
    assert list(ph) == list(DnsEngine.PHASES) and all(v >= 0.0 for v in ph.values())
    assert ph["pcg"] > 0.0
    assert len(E.history()["time"]) == 3
    for k in ("u", "v", "w", "p", "mf"):
        assert np.array_equal(E.field(k), G.field(k)), k


@pytest.mark.parametrize("mode", ["fixed", "mixed"])
def test_phase_stamps_time_graph_steps_without_changing_them(gpu, mode):
    # device clock stamps at the phase boundaries of graph-launched steps: 8 more kernels
    # per step, identical fields, and one finite duration per phase for stamped steps only
    from gip_b200.device import DnsEngine
    case, _ = cavity.generate(10, re=400.0)
    # FIXED runs exactly maxit iterations: GIP's 100 (far more would run past convergence)
    kw = dict(gamma=1.0 / 400, pcg_mode=mode, maxit=100 if mode == "fixed" else 2000, tol=1e-9,
              inner_tol=0.01, max_outer=50, use_graph=True)
    E = DnsEngine(case, **kw)
    G = DnsEngine(case, **kw)
    E.advance(2)
    G.advance(2)
    E.phase_stamps(True)
    E.advance(3)
    G.advance(3)
    hE, hG = E.history(), G.history()
    assert hE["iters"].tolist() == hG["iters"].tolist()
    assert (hE["kernels"][2:] - hG["kernels"][2:]).tolist() == [8, 8, 8]
    assert hE["kernels"][:2].tolist() == hG["kernels"][:2].tolist()
    for k in ("u", "v", "w", "p", "mf"):
        assert np.isfinite(G.field(k)).all() and np.array_equal(E.field(k), G.field(k)), k
    ph = E.phase_history()
    assert list(ph) == list(DnsEngine.PHASES)
    for name, v in ph.items():
        assert v.shape == (5,), name
        assert np.isnan(v[:2]).all(), name
        assert np.isfinite(v[2:]).all() and (v[2:] >= 0).all(), name
    assert (ph["pcg"][2:] > 0).all()
    E.phase_stamps(False)
    E.advance(1)
    G.advance(1)
    ph = E.phase_history()
    assert np.isnan(ph["pcg"][5]) and E.history()["kernels"][5] == G.history()["kernels"][5]


@pytest.mark.parametrize("general", [False, True])
def test_merged_face_operators_are_exact(gpu, monkeypatch, general):
    # the mass-flux kernel over SFx/SFy/SFz merged per face (its one-operator-per-face form
    # by default, its general form with GIPB200_NO_FACE1) gives the same fields, bit for
    # bit, as the kernel walking the three operators separately
    from gip_b200.device import DnsEngine
    case, _ = cavity.generate(12, re=400.0, permute_seed=5)
    kw = dict(gamma=1.0 / 400, pcg_mode="fixed", maxit=100, reorder=True)
    if general:
        monkeypatch.setenv("GIPB200_NO_FACE1", "1")
    E = DnsEngine(case, **kw)
    monkeypatch.setenv("GIPB200_NO_FACE3", "1")
    P = DnsEngine(case, **kw)
    E.advance(3)
    P.advance(3)
    for k in ("u", "v", "w", "p", "mf"):
        assert np.array_equal(E.field(k), P.field(k)), k


@pytest.mark.parametrize("precond", ["amg", "jacobi"])
def test_packed_fp64_residual_matches_sliced(gpu, monkeypatch, precond):
    # the mixed form's FP64 residual from the packed operator's columns (L's values from a
    # table, the ghost part of b - L x formed once per solve) against the sliced FP64 L: the
    # same solve to rounding, the same iteration counts to within one
    from gip_b200.device import DnsEngine
    case, _ = cavity.generate(20, re=400.0, permute_seed=3)
    kw = dict(gamma=1.0 / 400, pcg_mode="mixed", maxit=4000, tol=1e-9,
              inner_tol=0.01 if precond == "amg" else 0.3, max_outer=200, reorder=True,
              precond=precond)
    E = DnsEngine(case, **kw)
    monkeypatch.setenv("GIPB200_NO_PACKED_RESIDUAL", "1")
    F = DnsEngine(case, **kw)
    assert E.info()["packed_residual"] == 1 and F.info()["packed_residual"] == 0
    E.advance(4)
    F.advance(4)
    he, hf = E.history(), F.history()
    assert np.all(np.abs(he["iters"] - hf["iters"]) <= 1), (he["iters"], hf["iters"])
    assert np.all(he["massr"] < 1e-8)
    scale = np.abs(F.field("u")).max()
    for k in ("u", "v", "w"):
        assert np.abs(E.field(k) - F.field(k)).max() / scale < 1e-8, k
    assert np.abs(E.field("p") - F.field("p")).max() / np.abs(F.field("p")).max() < 1e-7
