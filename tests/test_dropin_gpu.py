"""The B200 Specification dropped into GIP's own driver and templates (GIP_DNS,
GIP_LinearSolver) prints GIP's README golden on C100K, in all three build variants."""
import os
import subprocess

import pytest

from conftest import C100K_1P, REPO, golden_lines, have_c100k

pytestmark = pytest.mark.gpu

BUILD = os.path.join(REPO, "gip_b200", "spec", "_build")
VARIANTS = ["DrivenCavityB200", "DrivenCavityB200_pcg", "DrivenCavityB200_dns"]


@pytest.mark.skipif(not have_c100k(), reason="merged C100K set not built")
@pytest.mark.parametrize("variant", VARIANTS)
def test_dropin_prints_readme_golden(gpu, variant):
    exe = os.path.join(BUILD, variant)
    if not os.path.exists(exe):
        pytest.skip("drop-in driver not built (gip_b200/spec/Makefile needs the GIP checkout)")
    r = subprocess.run([exe, "C100K"], cwd=C100K_1P, capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, GIPSHIM_NP="1"))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("time ")]
    assert lines == golden_lines("c100k_readme.txt")
