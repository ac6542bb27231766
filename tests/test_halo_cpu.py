"""The slab-split pressure solve (gip_b200.halo) as gloo ranks on CPU: GIP's per-rank
layout and send/receive lists from formats.split_ranks, the halo exchange and the
all-reduced dots, against the single-rank oracle solve (GIP_LinearSolver.h:44-117).

The per-element operations run here through a CPU model of the fused device calls (this
file's ModelOps, test infrastructure only); on GPUs SlabPcg uses the device ones."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from gip_b200 import cavity, formats
from gip_b200.halo import PAP, RR, RZ, BETA, ALPHA, SlabPcg, jacobi_diagonal


class ModelOps:
    """CPU model of DeviceOps: GIP's row semantics (rows without nonzeros keep their
    output), dots over the inner cells, scalars in a 5-entry tensor."""

    def __init__(self, part):
        L = part.ops["L"]
        self.n = L.nrows
        self.A = L.to_scipy().tocsr()
        self.nonempty = np.diff(L.rowptr) > 0
        Dm, self.dinv = jacobi_diagonal(L)
        self.has_diag = np.diff(Dm.rowptr) > 0

    def tensor(self, a, dtype=torch.float64):
        return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype)

    def zeros(self, n):
        return torch.zeros(n, dtype=torch.float64)

    def spmv(self, x, y):
        v = self.A @ x.numpy()
        y[:self.n][torch.from_numpy(self.nonempty)] = torch.from_numpy(v[self.nonempty])

    def spmv_dot(self, x, y, sc):
        self.spmv(x, y)
        sc[PAP] = float(np.dot(x[:self.n].numpy(), y[:self.n].numpy()))

    def jacobi_dot(self, r, p, sc):
        h = torch.from_numpy(self.has_diag)
        p[:self.n][h] = (r[:self.n] * torch.from_numpy(self.dinv))[h]
        sc[RZ] = float(np.dot(r[:self.n].numpy(), p[:self.n].numpy()))

    def update(self, x, r, z, p, q, sc):
        n = self.n
        alpha = float(sc[RZ] / sc[PAP])
        x[:n] += alpha * p[:n]
        r[:n] += -alpha * q[:n]
        z[:n] = r[:n] * torch.from_numpy(self.dinv)
        rz_prev = float(sc[RZ])
        sc[ALPHA] = alpha
        sc[RZ] = float(np.dot(r[:n].numpy(), z[:n].numpy()))
        sc[RR] = float(np.dot(r[:n].numpy(), r[:n].numpy()))
        sc[BETA] = float(sc[RZ]) / rz_prev

    def direction(self, p, z, sc):
        p[:self.n] = z[:self.n] + float(sc[BETA]) * p[:self.n]

    def axpy(self, y, x, a, n):
        y[:n] += a * x[:n]

    def gather(self, idx, x, buf):
        buf[:] = x[idx.long()]

    def scatter(self, idx, buf, x):
        x[idx.long()] = buf


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _problem(n=10, seed=5):
    case, meta = cavity.generate(n, re=400.0, permute_seed=seed)
    rng = np.random.default_rng(seed)
    b = rng.standard_normal(case.n_inner)
    x0 = rng.standard_normal(case.n_owned) * 0.1
    return case, meta, b, x0


def _worker(rank, world, port, q, maxit):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        case, meta, b, x0 = _problem()
        parts = formats.split_ranks(case, cavity.slab_partition(meta, world), world)
        part = parts[rank]
        ids = part.cell_ids
        n = part.n_inner
        S = SlabPcg(part, rank, world, dist=dist, ops=ModelOps(part))
        bl = torch.from_numpy(b[ids[:n]].copy())
        x0l = torch.from_numpy(x0[ids].copy())
        x, sc = S.solve(bl, x0l, maxit)
        q.put((rank, ids[:n].tolist(), x[:n].numpy().tolist(), float(sc[RR]),
               x[n:].numpy().tolist(), ids[n:].tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_split_pcg_matches_single_rank_oracle(oracle_mod, world):
    maxit = 60
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q, maxit)) for r in range(world)]
    for p in ps:
        p.start()
    got = [q.get(timeout=300) for _ in range(world)]
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    case, meta, b, x0 = _problem()
    L = case.ops["L"]
    xr, it, rr = oracle_mod.pcg(L, b, x0, maxit=maxit, mode=0)
    x = np.full(case.n_owned, np.nan)
    rr_ranks = set()
    for rank, ids, xs, rrk, xh, hid in got:
        x[ids] = xs
        rr_ranks.add(rrk)
        # boundary and halo cells of x keep x0 (x is copied from the exchanged x0 and never
        # updated outside the inner cells, GIP_LinearSolver.h:67)
        assert np.array_equal(np.array(xh), x0[hid])
    inner = np.arange(case.n_inner)
    assert not np.isnan(x[inner]).any()
    err = np.abs(x[inner] - xr[inner]).max() / np.abs(xr[inner]).max()
    assert err < 1e-10, err
    assert len(rr_ranks) == 1                      # every rank holds the same global r.r
    assert abs(next(iter(rr_ranks)) - rr) <= 1e-8 * rr + 1e-24 * float(np.dot(b, b))


def test_halo_lists_cover_every_remote_read():
    # GIP_Topo's lists: what rank r receives from q is exactly what q sends to r, and the
    # received cells are every column of r's operators outside its own cells
    case, meta, b, x0 = _problem()
    world = 3
    parts = formats.split_ranks(case, cavity.slab_partition(meta, world), world)
    for r, pr in enumerate(parts):
        t = pr.topo_cols
        for qq, pq in enumerate(parts):
            if qq == r:
                continue
            tq = pq.topo_cols
            recv = pr.cell_ids[t.recv_indx[t.recv_row[qq]:t.recv_row[qq + 1]]]
            sent = pq.cell_ids[tq.send_indx[tq.send_row[r]:tq.send_row[r + 1]]]
            assert np.array_equal(recv, sent)
        L = pr.ops["L"]
        cols = np.unique(L.col)
        remote = cols[cols >= t.owned]
        assert np.array_equal(np.sort(remote), np.sort(t.recv_indx))
