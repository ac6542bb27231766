"""The oracle is pinned against GIP's own goldens before anything is compared with it."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, REF_BIN, golden_lines, have_c100k
from gip_b200 import cavity, formats


def _oracle_lines(oracle, hist):
    return [oracle.format_line(hist["time"][i], hist["dt"][i], hist["massr"][i], i + 1)
            for i in range(len(hist["time"]))]


def test_readme_golden_matches_reference_runs():
    # GIP's README block, its CPU build at 4 ranks and at 1 rank (merged) agree exactly
    readme = golden_lines("c100k_readme.txt")
    assert len(readme) == 10
    assert golden_lines("c100k_np4.txt") == readme
    assert golden_lines("c100k_np1.txt") == readme


@pytest.mark.skipif(not have_c100k(), reason="merged C100K set not built")
def test_oracle_prints_readme_on_c100k(oracle_mod, c100k_case):
    d = oracle_mod.OracleDNS(c100k_case, gamma=1e-3)
    hist = d.run(10)
    assert _oracle_lines(oracle_mod, hist) == golden_lines("c100k_readme.txt")


@pytest.mark.parametrize("n", [8, 12])
def test_oracle_bitexact_vs_reference_fields(oracle_mod, n):
    g = np.load(os.path.join(GOLDEN, f"cavity{n}_ref.npz"))
    case, _ = cavity.generate(n, re=float(g["re"]))
    d = oracle_mod.OracleDNS(case, gamma=1.0 / float(g["re"]))
    hist = d.run(int(g["steps"]))
    assert _oracle_lines(oracle_mod, hist) == list(g["lines"])
    for k in ("u", "v", "w", "p", "p0", "mf", "ax0"):
        assert np.array_equal(d.vec[k][: g[k].size], g[k]), k


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="GIP CPU build absent")
def test_oracle_bitexact_vs_reference_binary_live(oracle_mod):
    # a case the fixtures do not hold: permuted 6^3 cavity, 4 steps
    case, meta = cavity.generate(6, re=250.0, permute_seed=3)
    with tempfile.TemporaryDirectory() as td:
        formats.write_case(td, "P6", [case])
        env = dict(os.environ, GIPSHIM_NP="1")
        subprocess.run([REF_BIN, "P6", "4", os.path.join(td, "d"), "250.0"], cwd=td, env=env,
                       check=True, capture_output=True)
        ref = {k: np.fromfile(os.path.join(td, f"d.{k}.0.f64")) for k in ("u", "p", "mf")}
    d = oracle_mod.OracleDNS(case, gamma=1.0 / 250.0)
    d.run(4)
    for k, v in ref.items():
        assert np.array_equal(d.vec[k][: v.size], v), k


def test_oracle_pcg_tolerance_mode(oracle_mod):
    L, b = cavity.poisson_problem(8, seed=1)
    x, it, rr = oracle_mod.pcg(L, b, np.zeros(L.nrows), maxit=1000, mode=1, tol=1e-8)
    assert 0 < it < 1000
    assert np.sqrt(rr) <= 1e-8 * np.linalg.norm(b)
    r = b - L.to_scipy() @ x
    assert np.linalg.norm(r) <= 2e-8 * np.linalg.norm(b)


def test_oracle_pcg_fixed_equals_reference_formula(oracle_mod):
    # fixed mode runs exactly maxit iterations, as GIP_LinearSolver does
    L, b = cavity.poisson_problem(6, seed=2)
    _, it, _ = oracle_mod.pcg(L, b, np.zeros(L.nrows), maxit=17, mode=0)
    assert it == 17


def test_torch_adjoint_reference_forward_matches_oracle(oracle_mod):
    # the torch timestep used as the gradient reference reproduces the oracle's state
    import torch
    from adjoint_reference import kinetic_energy
    case, meta = cavity.generate(6, re=100.0)
    d = oracle_mod.OracleDNS(case, gamma=1e-2, cg_maxit=5000, cg_mode=1, cg_tol=1e-14)
    h = d.run(4)
    N = case.n_inner
    vol = np.full(N, meta.h ** 3)
    J_or = 0.5 * (vol * (d.vec["u"][:N] ** 2 + d.vec["v"][:N] ** 2 + d.vec["w"][:N] ** 2)).sum()
    lid = case.fields["u"][meta.lid_ghosts]
    J = kinetic_energy(case, meta.lid_ghosts, torch.tensor(lid), torch.tensor(1.0), h["dt"], vol)
    assert abs(J.item() - J_or) <= 1e-9 * abs(J_or)
