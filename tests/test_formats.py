"""GIP file formats, the rank merge/split and the structured cavity generator."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import REF_BIN
from gip_b200 import cavity, formats


def test_csr_vec_topo_roundtrip(tmp_path):
    case, _ = cavity.generate(4)
    formats.write_case(str(tmp_path), "T", [case])
    back = formats.load_case(str(tmp_path), "T", 1, 0)
    for k, m in case.ops.items():
        b = back.ops[k]
        assert (b.nrows, b.ncols, b.nnz) == (m.nrows, m.ncols, m.nnz)
        assert np.array_equal(b.rowptr, m.rowptr) and np.array_equal(b.col, m.col)
        assert np.array_equal(b.val, m.val)
    for k in formats.FIELD_NAMES:
        assert np.array_equal(back.fields[k], case.fields[k])
    assert back.topo_cols.inner == case.n_inner and back.topo_cols.owned == case.n_owned


def test_truncated_csr_is_rejected(tmp_path):
    case, _ = cavity.generate(3)
    p = str(tmp_path / "x.csr")
    formats.write_csr(p, case.ops["L"])
    data = open(p, "rb").read()
    open(p, "wb").write(data[:-8])
    with pytest.raises(formats.FormatError):
        formats.read_csr(p)


def test_bad_rowptr_is_rejected():
    m = formats.Csr(2, 2, np.array([0, 2, 1], np.int32), np.array([0], np.int32), np.array([1.0]))
    with pytest.raises(formats.FormatError):
        m.validate("m")


@pytest.mark.parametrize("n", [3, 5])
def test_generator_identities(n):
    case, meta = cavity.generate(n, re=100.0)
    formats.check_case(case)
    S = {k: v.to_scipy() for k, v in case.ops.items()}
    N = meta.n_inner
    A = -(S["Mres"] @ S["SO"])
    diff = (S["L"] - A).tocoo()
    nz = np.abs(diff.data) > 0
    # L = -Mres SO except the pinned diagonal (+L_pp/101)
    assert list(zip(diff.row[nz], diff.col[nz])) == [(meta.pin_cell, meta.pin_cell)]
    for d in "xyz":
        assert abs(S["M" + d] + S["Mres"] @ S["SF" + d]).max() == 0
        assert abs(S["G" + d][:N, :N] - S["M" + d][:, :N].T / meta.h ** 3).max() < 1e-9
    assert abs(np.asarray(S["D"].sum(axis=1))).max() < 1e-9 * abs(S["D"]).max()
    L = S["L"][:, :N]
    assert abs(L - L.T).max() == 0
    # Ec: one row per D nonzero; C = Ec mf is skew on interior neighbours
    assert case.ops["Ec"].nrows == case.ops["D"].nnz
    # lid ghosts carry u = 1, other ghosts 0
    u = case.fields["u"]
    assert np.all(u[:N] == 0) and set(np.unique(u[N:])) <= {0.0, 1.0}
    assert (u[N:] == 1.0).sum() == n * n


def test_permutation_preserves_products():
    case, meta = cavity.generate(4, re=100.0)
    pc, _ = cavity.generate(4, re=100.0, permute_seed=7)
    pm = cavity.permute(case, meta, 7)[1]
    cmap = np.concatenate([pm.cell_perm, np.arange(meta.n_inner, meta.n_inner + meta.n_ghost)])
    x = np.random.default_rng(0).standard_normal(meta.n_inner + meta.n_ghost)
    xp = np.empty_like(x)
    xp[cmap] = x
    for op in ("L", "D", "Gx", "Mx"):
        y = case.ops[op].to_scipy() @ x
        yp = pc.ops[op].to_scipy() @ xp
        assert np.array_equal(yp[cmap[: y.size]], y), op


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="GIP CPU build absent")
def test_split_runs_in_reference_at_3_ranks():
    case, meta = cavity.generate(6, re=100.0)
    with tempfile.TemporaryDirectory() as td:
        formats.write_case(td, "S6", [case])
        env1 = dict(os.environ, GIPSHIM_NP="1")
        r1 = subprocess.run([REF_BIN, "S6", "3", "-", "100"], cwd=td, env=env1, check=True,
                            capture_output=True, text=True).stdout
        parts = formats.split_ranks(case, cavity.slab_partition(meta, 3), 3)
        formats.write_case(td, "S6", parts)
        env3 = dict(os.environ, GIPSHIM_NP="3")
        r3 = subprocess.run([REF_BIN, "S6", "3", "-", "100"], cwd=td, env=env3, check=True,
                            capture_output=True, text=True).stdout
    l1 = [ln.split()[1:4] for ln in r1.splitlines() if ln.startswith("time")]
    l3 = [ln.split()[1:4] for ln in r3.splitlines() if ln.startswith("time")]
    assert l1 == l3  # time and dt agree to the printed digits


def test_merge_of_split_restores_case(tmp_path):
    case, meta = cavity.generate(5, re=100.0)
    parts = formats.split_ranks(case, cavity.slab_partition(meta, 2), 2)
    formats.write_case(str(tmp_path), "M5", parts)
    merged = formats.merge_ranks(str(tmp_path), "M5", 2)
    formats.check_case(merged)
    assert merged.n_inner == case.n_inner and merged.n_owned == case.n_owned
    # same operators up to a relabelling of cells: compare sorted value multisets
    for op in ("L", "D", "Mres", "SO"):
        assert np.array_equal(np.sort(merged.ops[op].val), np.sort(case.ops[op].val)) or \
            merged.ops[op].nnz >= case.ops[op].nnz
