"""The device FP64 discrete adjoint against torch autograd on the same operators and
against central finite differences (frozen CFL steps)."""
import numpy as np
import pytest
import torch

from adjoint_reference import kinetic_energy
from gip_b200 import cavity

pytestmark = pytest.mark.gpu


def _setup(n, re, seed=5):
    case, meta = cavity.generate(n, re=re)
    lid_cells = meta.lid_ghosts
    rng = np.random.default_rng(seed)
    lid = 1.0 + rng.normal(0.0, 0.01, lid_cells.size)
    vol = np.full(case.n_inner, meta.h ** 3)
    return case, meta, lid_cells, lid, vol


@pytest.mark.parametrize("n,re,steps,every,precond", [(6, 100.0, 5, 2, "jacobi"),
                                                      (8, 400.0, 6, 4, "jacobi"),
                                                      (10, 400.0, 5, 3, "amg")])
def test_adjoint_matches_torch_autograd(gpu, n, re, steps, every, precond):
    from gip_b200.adjoint import CavityAdjoint
    case, meta, lid_cells, lid, vol = _setup(n, re)
    nu0 = 1.0 / re
    A = CavityAdjoint(case, lid_cells, vol, nu0=nu0, gamma=1.0 / re, tol=1e-13,
                      checkpoint_every=every, precond=precond)
    J = A.forward(lid, nu0, steps)
    g_lid, g_nu = A.backward()
    # reference: torch autograd through the same step with the same frozen steps
    tl = torch.tensor(lid, dtype=torch.float64, requires_grad=True)
    ts = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    Jr = kinetic_energy(case, lid_cells, tl, ts, A.dt, vol)
    Jr.backward()
    assert abs(J - Jr.item()) <= 1e-10 * abs(Jr.item())
    ref_lid = tl.grad.numpy()
    ref_nu = ts.grad.item() / nu0
    assert np.abs(g_lid - ref_lid).max() <= 1e-6 * np.abs(ref_lid).max()
    assert abs(g_nu - ref_nu) <= 1e-6 * abs(ref_nu)


def test_autograd_function_and_finite_differences(gpu):
    from gip_b200.adjoint import CavityAdjoint
    case, meta, lid_cells, lid, vol = _setup(8, 400.0, seed=7)
    nu0 = 1.0 / 400
    A = CavityAdjoint(case, lid_cells, vol, nu0=nu0, gamma=1.0 / 400, tol=1e-13,
                      checkpoint_every=3)
    steps = 7
    tl = torch.tensor(lid, dtype=torch.float64, device="cuda", requires_grad=True)
    tn = torch.tensor(nu0, dtype=torch.float64, device="cuda", requires_grad=True)
    J = A.energy(tl, tn, steps)
    J.backward()
    g = np.concatenate([tl.grad.cpu().numpy(), [tn.grad.item()]])
    rng = np.random.default_rng(3)
    eps = 1e-6
    for _ in range(4):
        d = rng.standard_normal(lid.size + 1)
        d /= np.linalg.norm(d)
        Jp = A.forward(lid + eps * d[:-1], nu0 + eps * d[-1], steps)
        Jm = A.forward(lid - eps * d[:-1], nu0 - eps * d[-1], steps)
        fd = (Jp - Jm) / (2 * eps)
        assert abs(fd - g @ d) <= 1e-6 * max(abs(fd), np.abs(g).max()), (fd, g @ d)


@pytest.mark.slow
def test_adjoint_config_64cube_50_steps(gpu):
    """The adjoint-sensitivity configuration: 64^3 cavity, Re 400, 50 steps, checkpoints
    every 10, lid 1 + N(0, 0.01); central differences (eps 1e-6) on 16 random directions."""
    from gip_b200.adjoint import CavityAdjoint
    case, meta, lid_cells, lid, vol = _setup(64, 400.0, seed=64)
    nu0 = 1.0 / 400
    A = CavityAdjoint(case, lid_cells, vol, nu0=nu0, gamma=1.0 / 400, tol=1e-12,
                      checkpoint_every=10)
    steps = 50
    A.forward(lid, nu0, steps)
    g_lid, g_nu = A.backward()
    g = np.concatenate([g_lid, [g_nu]])
    rng = np.random.default_rng(16)
    eps = 1e-6
    errs = []
    for _ in range(16):
        d = rng.standard_normal(lid.size + 1)
        d /= np.linalg.norm(d)
        fd = (A.forward(lid + eps * d[:-1], nu0 + eps * d[-1], steps) -
              A.forward(lid - eps * d[:-1], nu0 - eps * d[-1], steps)) / (2 * eps)
        errs.append(abs(fd - g @ d) / max(abs(fd), 1e-300))
    assert max(errs) < 1e-6, errs
