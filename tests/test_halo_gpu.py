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
