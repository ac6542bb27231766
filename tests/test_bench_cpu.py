"""bench.py's reference arm and JSON contract, on the host (GIP's own CPU build)."""
import json
import os
import subprocess
import sys

import pytest

from conftest import REF_BIN, REPO


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="GIP CPU build not built")
def test_reference_arm_line():
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference",
                        "--n", "12", "--steps", "2", "--warmup", "1"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "ms/timestep"
    assert d["higher_is_better"] is False and d["value"] > 0
    assert d["steps"] == 2 and d["warmup"] == 1
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["config"]["cells"] == 12 ** 3
    # the headline is GIP's stock step, measured as it ships (100 PCG iterations), and the
    # config says what ran: FP64, GIP's Jacobi, GIP's own decomposition
    assert d["pcg_iterations_per_step"] == 100 and "fixed 100" in d["config"]["pcg"]
    assert d["config"]["precond"] == "jacobi" and d["config"]["form"].startswith("FP64")
    assert d["value"] == d["samples"]["100"]["ms_per_step"]
    # GIP's own per-step line after the untimed and the timed steps (3 timesteps of dt 0.1)
    for s in d["samples"].values():
        assert s["last_line"].startswith("time 3.000000e-01")


def test_clock_sampler_parses_samples_and_reasons():
    sys.path.insert(0, REPO)
    import bench

    class Done:
        def terminate(self):
            pass

        def wait(self, timeout=None):
            return 0

    cs = bench.ClockSampler(0)
    cs.proc = Done()
    rows = ["0, 1965, 1965, 512.30, 0x0, Not Active, Not Active, Not Active, Not Active",
            "0, 1950, 1965, 990.10, 0x4, Not Active, Not Active, Not Active, Active",
            "0, 1965, 1965, [N/A], 0x0, Not Active, Not Active, Not Active, Not Active",
            "garbage line"]
    cs.out.write(("\n".join(rows) + "\n").encode())
    cs.out.flush()
    r = cs.stop()
    assert r["samples"] == 3 and r["sm_mhz"] == 1965.0 and r["sm_max_mhz"] == 1965.0
    assert r["power_w_max"] == 990.1 and r["reasons"] == ["sw_power_cap"]


def test_peaks_and_traffic_helpers(tmp_path, monkeypatch):
    sys.path.insert(0, REPO)
    import bench
    p = bench.peaks()
    assert p["hbm_gbs"] > 0 and p["source"] in ("measured", "fallback")
    t = bench.ncu_traffic("k_mxp_spmv_dot", 1000)
    assert t is None or t > 0
    monkeypatch.setattr(bench, "REPO", str(tmp_path))
    assert bench.peaks() == {"hbm_gbs": 6650.0, "source": "fallback"}
    assert bench.ncu_traffic("k_mxp_spmv_dot", 1000) is None


def test_other_configs_record_errors_and_keep_the_line(monkeypatch):
    """A configuration that fails records its error under other_configs; the others still
    run and the cavity line is still printed (each entry also carries its wall time)."""
    import argparse

    sys.path.insert(0, REPO)
    import torch

    import bench
    monkeypatch.setattr(torch.cuda, "synchronize", lambda: None)

    def boom(*a, **k):
        raise RuntimeError("no device")

    monkeypatch.setattr(bench, "poisson_results", boom)
    monkeypatch.setattr(bench, "adjoint_results",
                        lambda a, n, nd: {"results": {"n": n, "dirs": nd}})
    monkeypatch.setattr(bench, "batch_results", lambda a, full: {"results": {"full": full}})
    out = bench.other_configs(argparse.Namespace())
    assert out["poisson_128"]["error"] == "RuntimeError: no device"
    assert out["adjoint_64"]["results"] == {"n": 64, "dirs": 4}
    assert out["batch_32"]["results"] == {"full": False}
    assert all("wall_s" in v for v in out.values())
