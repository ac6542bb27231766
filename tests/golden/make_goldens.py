"""Regenerates the committed golden fixtures from GIP itself (run where the reference
checkout exists; the fixtures then travel with the repository).

* ``c100k_readme.txt``  -- the expected-output block of GIP's README.md (lines 73-82).
* ``c100k_np4.txt``     -- stdout of GIP's CPU build at 4 ranks on the shipped C100K set.
* ``c100k_np1.txt``     -- stdout of GIP's CPU build at 1 rank on C100K merged to one rank.
* ``cavity<n>_ref.npz`` -- GIP's CPU build (1 rank) on generated n^3 cavities: the per-step
  lines and the final fields u, v, w, p, p0, mf, ax0.

It also writes the merged C100K single-rank set to ``oracle/_ref/c100k`` (git-ignored;
it travels with the tree for the GPU known-answer test).

Usage: python tests/golden/make_goldens.py --reference <GIP checkout>
(or with the checkout's path in the GIP_REFERENCE environment variable)
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from gip_b200 import cavity, formats  # noqa: E402

REF_BIN = os.path.join(REPO, "oracle", "_ref", "gip_ref_cpu")
C100K_1P = os.path.join(REPO, "oracle", "_ref", "c100k")

# generated cavities pinned against GIP's own CPU build: (n, Re, steps)
CAVITIES = [(8, 100.0, 10), (12, 400.0, 10)]


def run_ref(cwd: str, case: str, nranks: int, steps: int = 10, dump: str = "-", re_: float = None):
    args = [REF_BIN, case, str(steps), dump]
    if re_ is not None:
        args.append(repr(re_))
    env = dict(os.environ, GIPSHIM_NP=str(nranks))
    r = subprocess.run(args, cwd=cwd, env=env, capture_output=True, text=True, check=True)
    return [ln for ln in r.stdout.splitlines() if ln.startswith("time ")]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("GIP_REFERENCE"),
                    help="the GIP checkout (default: $GIP_REFERENCE)")
    a = ap.parse_args()
    if not a.reference:
        ap.error("--reference <GIP checkout> (or GIP_REFERENCE) is required")
    subprocess.check_call(["make", "-s", "-C", os.path.join(REPO, "oracle"), "all",
                           f"REF={a.reference}"])
    readme = open(os.path.join(a.reference, "README.md")).read().splitlines()
    lines = [ln.strip() for ln in readme if re.match(r"^\s*time \S+ \[dt::", ln)]
    open(os.path.join(HERE, "c100k_readme.txt"), "w").write("\n".join(lines) + "\n")

    with tempfile.TemporaryDirectory() as td:
        os.symlink(os.path.join(a.reference, "InputFiles"), os.path.join(td, "InputFiles"))
        out = run_ref(td, "C100K", 4)
    open(os.path.join(HERE, "c100k_np4.txt"), "w").write("\n".join(out) + "\n")

    merged = formats.merge_ranks(a.reference, "C100K", 4)
    formats.check_case(merged)
    formats.write_case(C100K_1P, "C100K", [merged])
    out = run_ref(C100K_1P, "C100K", 1)
    open(os.path.join(HERE, "c100k_np1.txt"), "w").write("\n".join(out) + "\n")

    for n, re_, steps in CAVITIES:
        case, meta = cavity.generate(n, re=re_)
        with tempfile.TemporaryDirectory() as td:
            formats.write_case(td, "CAV", [case])
            dump = os.path.join(td, "dump")
            lines = run_ref(td, "CAV", 1, steps, dump, re_)
            fields = {k: np.fromfile(f"{dump}.{k}.0.f64")
                      for k in ("u", "v", "w", "p", "p0", "mf", "ax0")}
            parts = formats.split_ranks(case, cavity.slab_partition(meta, 2), 2)
            formats.write_case(td, "CAV", parts)
            lines2 = run_ref(td, "CAV", 2, steps, "-", re_)
        np.savez_compressed(os.path.join(HERE, f"cavity{n}_ref.npz"), lines=np.array(lines),
                            lines_np2=np.array(lines2), re=re_, steps=steps, **fields)

    # the first configuration: 48^3, Re 100, 10 steps; GIP at 4 slab ranks and at 1 rank.
    # Only per-step lines and field checksums are kept (the fields are 110k cells each).
    import json
    case, meta = cavity.generate(48, re=100.0)
    out = {"n": 48, "re": 100.0, "steps": 10}
    with tempfile.TemporaryDirectory() as td:
        formats.write_case(td, "CAV48", [case])
        dump = os.path.join(td, "dump")
        out["lines_np1"] = run_ref(td, "CAV48", 1, 10, dump, 100.0)
        out["checksums_np1"] = {k: _checksums(np.fromfile(f"{dump}.{k}.0.f64"), case.n_inner)
                                for k in ("u", "v", "w", "p", "mf")}
        parts = formats.split_ranks(case, cavity.slab_partition(meta, 4), 4)
        formats.write_case(td, "CAV48", parts)
        out["lines_np4"] = run_ref(td, "CAV48", 4, 10, "-", 100.0)
    with open(os.path.join(HERE, "cavity48_ref.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("goldens written to", HERE)


def _checksums(x: np.ndarray, n_inner: int) -> dict:
    """Order-free summaries of a field: L1, L2 and max norms of the inner part."""
    xi = x[:n_inner]
    return {"l1": float(np.abs(xi).sum()), "l2": float(np.sqrt((xi * xi).sum())),
            "max": float(np.abs(xi).max())}


if __name__ == "__main__":
    main()
