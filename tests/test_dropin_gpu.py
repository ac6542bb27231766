"""The B200 Specification dropped into GIP's own driver and templates (GIP_DNS,
GIP_LinearSolver) prints GIP's README golden on C100K in every build variant, and two
integrate() calls of 5 steps continue exactly like one call of 10 (GIP_DNS.h:99-113: each
call starts from the members the previous one left)."""
import json
import os
import re
import subprocess

import pytest

from conftest import C100K_1P, REPO, golden_lines, have_c100k

pytestmark = pytest.mark.gpu

BUILD = os.path.join(REPO, "gip_b200", "spec", "_build")
VARIANTS = ["DrivenCavityB200", "DrivenCavityB200_pcg", "DrivenCavityB200_ops",
            "DrivenCavityB200_dns"]


def _run(variant, *args):
    exe = os.path.join(BUILD, variant)
    if not os.path.exists(exe):
        pytest.skip("drop-in driver not built (gip_b200/spec/Makefile needs the GIP checkout)")
    r = subprocess.run([exe, "C100K", *args], cwd=C100K_1P, capture_output=True, text=True,
                       timeout=600, env=dict(os.environ, GIPSHIM_NP="1"))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("time ")]
    info = json.loads([ln for ln in r.stderr.splitlines() if ln.startswith("{")][-1])
    return lines, info


@pytest.mark.skipif(not have_c100k(), reason="merged C100K set not built")
@pytest.mark.parametrize("variant", VARIANTS)
def test_dropin_prints_readme_golden(gpu, variant):
    lines, _ = _run(variant)
    assert lines == golden_lines("c100k_readme.txt")


@pytest.mark.skipif(not have_c100k(), reason="merged C100K set not built")
@pytest.mark.parametrize("variant", VARIANTS)
def test_dropin_integrate_twice_continues(gpu, variant):
    ten, i10 = _run(variant, "10", "1")
    five, i55 = _run(variant, "5", "2")
    strip = lambda ls: [re.sub(r" ite \d+$", "", ln) for ln in ls]
    assert strip(five) == strip(ten)
    assert [ln.rsplit(" ", 1)[1] for ln in five] == [str(k) for k in list(range(1, 6)) * 2]
    assert i55["fields"] == i10["fields"]
    assert i55["time"] == i10["time"]
