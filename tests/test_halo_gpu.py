"""Device side of the slab-split solve: GIP_Topo's pack/unpack kernels (gipb200_gather /
gipb200_scatter) and SlabPcg over the device operations at one rank, against the oracle.
(The exchange between ranks runs as gloo ranks in test_halo_cpu.py; a GPU call here has
one GPU.)"""
import numpy as np
import pytest
import torch

from gip_b200 import cavity

pytestmark = pytest.mark.gpu


def test_pack_unpack_kernels(gpu):
    from gip_b200 import halo
    rng = np.random.default_rng(2)
    x = rng.standard_normal(5000)
    idx = rng.permutation(5000)[:1234].astype(np.int32)
    case, _ = cavity.generate(6, re=100.0)
    ops = halo.DeviceOps(case, torch.device("cuda"))
    dx, di = ops.tensor(x), ops.tensor(idx, torch.int32)
    buf = ops.zeros(idx.size)
    ops.gather(di, dx, buf)
    assert np.array_equal(buf.cpu().numpy(), x[idx])
    y = ops.zeros(5000)
    ops.scatter(di, buf, y)
    want = np.zeros(5000)
    want[idx] = x[idx]
    assert np.array_equal(y.cpu().numpy(), want)


@pytest.mark.parametrize("n,maxit", [(10, 60), (14, 100)])
def test_slab_pcg_one_rank_on_device_matches_oracle(gpu, oracle_mod, n, maxit):
    from gip_b200 import formats, halo
    case, meta = cavity.generate(n, re=400.0, permute_seed=n)
    part = formats.split_ranks(case, cavity.slab_partition(meta, 1), 1)[0]
    rng = np.random.default_rng(n)
    b = rng.standard_normal(case.n_inner)
    x0 = rng.standard_normal(case.n_owned) * 0.1
    S = halo.SlabPcg(part, 0, 1, device=torch.device("cuda"))
    ids = part.cell_ids
    k = part.n_inner
    x, sc = S.solve(S.ops.tensor(b[ids[:k]]), S.ops.tensor(x0[ids]), maxit)
    xr, it, rr = oracle_mod.pcg(case.ops["L"], b, x0, maxit=maxit, mode=0)
    got = np.empty(case.n_owned)
    got[ids] = x.cpu().numpy()
    assert np.abs(got[:k] - xr[:k]).max() / np.abs(xr[:k]).max() < 1e-10
    assert np.array_equal(got[k:], x0[k:])


def _device_rank(rank, world, port, q, maxit):
    # one rank of the slab-split solve on the device (ranks share the GPU here: gloo moves
    # the halos and the dot partials through host memory, no kernel waits on another rank)
    import datetime
    import os

    import torch.distributed as dist

    from gip_b200 import formats, halo
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        case, meta = cavity.generate(10, re=400.0, permute_seed=5)
        rng = np.random.default_rng(5)
        b = rng.standard_normal(case.n_inner)
        x0 = rng.standard_normal(case.n_owned) * 0.1
        part = formats.split_ranks(case, cavity.slab_partition(meta, world), world)[rank]
        ids, k = part.cell_ids, part.n_inner
        S = halo.SlabPcg(part, rank, world, dist=dist, device=torch.device("cuda"))
        x, sc = S.solve(S.ops.tensor(b[ids[:k]]), S.ops.tensor(x0[ids]), maxit)
        q.put((rank, ids[:k].tolist(), x[:k].cpu().numpy().tolist()))
    finally:
        dist.destroy_process_group()


def test_slab_pcg_two_ranks_on_device_matches_oracle(gpu, oracle_mod):
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    world, maxit = 2, 60
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_device_rank, args=(r, world, port, q, maxit)) for r in range(world)]
    for p in ps:
        p.start()
    got = [q.get(timeout=300) for _ in range(world)]
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    case, meta = cavity.generate(10, re=400.0, permute_seed=5)
    rng = np.random.default_rng(5)
    b = rng.standard_normal(case.n_inner)
    x0 = rng.standard_normal(case.n_owned) * 0.1
    xr, it, rr = oracle_mod.pcg(case.ops["L"], b, x0, maxit=maxit, mode=0)
    x = np.full(case.n_owned, np.nan)
    for _, ids, xs in got:
        x[ids] = xs
    k = case.n_inner
    assert not np.isnan(x[:k]).any()
    assert np.abs(x[:k] - xr[:k]).max() / np.abs(xr[:k]).max() < 1e-10
