"""The first configuration: 48^3 lid-driven cavity, Re 100, 10 steps, against GIP's own
CPU build (1 rank and 4 slab ranks, committed fixture) and, in the tolerance mode the
configuration adds, against the oracle's iteration counts."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err
from gip_b200 import cavity

pytestmark = pytest.mark.gpu


def _parse(line):
    f = line.split()
    return float(f[1]), float(f[2].split("::")[1].rstrip("]")), float(f[4])


@pytest.fixture(scope="module")
def case48():
    return cavity.generate(48, re=100.0)[0]


@pytest.mark.parametrize("reorder", [False, True])
def test_fixed100_matches_gip_cpu(gpu, oracle_mod, case48, reorder):
    from gip_b200.device import DnsEngine
    g = json.load(open(os.path.join(GOLDEN, "cavity48_ref.json")))
    E = DnsEngine(case48, gamma=1.0 / 100, pcg_mode="fixed", maxit=100, reorder=reorder)
    E.advance(10)
    h = E.history()
    for k, (l1, l4) in enumerate(zip(g["lines_np1"], g["lines_np4"])):
        t, dt, m = _parse(l1)
        assert oracle_mod.format_line(h["time"][k], h["dt"][k], h["massr"][k], k + 1).split()[:3] \
            == l1.split()[:3]
        assert abs(h["massr"][k] - m) <= 1e-5 * m + 1e-14
        assert _parse(l4)[:2] == (t, dt)  # GIP at 4 ranks: same times and steps
    N = case48.n_inner
    for k, cs in g["checksums_np1"].items():
        x = E.field(k)[:N]
        assert abs(np.sqrt((x * x).sum()) - cs["l2"]) <= 1e-10 * cs["l2"], k
        assert abs(np.abs(x).max() - cs["max"]) <= 1e-10 * cs["max"], k


def test_tol_mode_iterations_match_oracle(gpu, oracle_mod, case48):
    from gip_b200.device import DnsEngine
    E = DnsEngine(case48, gamma=1.0 / 100, pcg_mode="tol", maxit=5000, tol=1e-6)
    E.advance(10)
    d = oracle_mod.OracleDNS(case48, gamma=1.0 / 100, cg_maxit=5000, cg_mode=1, cg_tol=1e-6)
    hr = d.run(10)
    h = E.history()
    assert np.all(np.abs(h["iters"] - hr["iters"]) <= 1), (h["iters"], hr["iters"])
    for k in ("u", "v", "w", "p"):
        assert rel_err(E.field(k), d.vec[k]) < 1e-6, k
