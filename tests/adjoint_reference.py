"""Test helper: the timestep in plain torch float64 (sparse products as gather /
index_add, the Poisson solve as an exact sparse LU with its own autograd node), so
torch autograd gives an independent reference gradient of the kinetic energy.  It takes
the same operators and the same frozen dt sequence as the device adjoint."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl
import torch


class _Spmv:
    def __init__(self, m, device):
        rp = np.asarray(m.rowptr, np.int64)
        self.rows = torch.from_numpy(np.repeat(np.arange(m.nrows), np.diff(rp))).to(device)
        self.col = torch.from_numpy(np.asarray(m.col, np.int64)).to(device)
        self.val = torch.from_numpy(np.asarray(m.val, np.float64)).to(device)
        self.nrows = m.nrows
        self.nonempty = torch.from_numpy(np.diff(rp) > 0).to(device)

    def __call__(self, x, vals=None):
        v = self.val if vals is None else vals
        y = torch.zeros(self.nrows, dtype=torch.float64, device=x.device)
        return y.index_add(0, self.rows, v * x[self.col])


class _Solve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, b, lu):
        ctx.lu = lu
        x = lu.solve(b.detach().cpu().numpy())
        return torch.from_numpy(x).to(b.device)

    @staticmethod
    def backward(ctx, g):
        y = ctx.lu.solve(g.detach().cpu().numpy(), trans="T")
        return torch.from_numpy(y).to(g.device), None


def kinetic_energy(case, lid_cells, lid, nu_scale, dts, volume, rho=1.0, device="cpu"):
    """J after len(dts) steps; lid and nu_scale are torch scalars/vectors (requires_grad)."""
    N, NO = case.n_inner, case.n_owned
    op = {k: _Spmv(case.ops[k], device) for k in case.ops}
    L = case.ops["L"].to_scipy()[:, :N].tocsc()
    lu = spl.splu(L)
    u = torch.from_numpy(case.fields["u"].copy()).to(device)
    lid_idx = torch.from_numpy(np.asarray(lid_cells, np.int64)).to(device)
    u = u.index_put((lid_idx,), lid)
    v = torch.from_numpy(case.fields["v"].copy()).to(device)
    w = torch.from_numpy(case.fields["w"].copy()).to(device)
    vel = [u, v, w]
    a0 = [torch.zeros(N, dtype=torch.float64, device=device) for _ in range(3)]
    mf = torch.zeros(case.n_faces, dtype=torch.float64, device=device)
    cval = torch.from_numpy(case.ops["D"].val.copy()).to(device)
    so_empty = ~op["SO"].nonempty
    vol = torch.from_numpy(np.asarray(volume, np.float64)).to(device)
    ec_nonempty = op["Ec"].nonempty
    for dt in dts:
        sigma = 1.0 / dt
        cval = torch.where(ec_nonempty, op["Ec"](mf), cval)
        a = [nu_scale * op["D"](x) - op["D"](x, cval) for x in vel]
        star = []
        for d in range(3):
            inner = vel[d][:N] + 1.5 * dt * a[d] + (-0.5 * dt) * a0[d]
            star.append(torch.cat([inner, vel[d][N:]]))
        a0 = a
        rhs = sigma * (op["Mx"](star[0]) + op["My"](star[1]) + op["Mz"](star[2]))
        p = _Solve.apply(rhs, lu)
        pfull = torch.cat([p, torch.zeros(NO - N, dtype=torch.float64, device=device)])
        ghost = op["Lb"](pfull)
        pfull = torch.cat([p, ghost[N:]])
        gp = [op["G" + ax](pfull) for ax in "xyz"]
        fact = -1.0 / (rho * sigma)
        vel = [torch.cat([star[d][:N] + fact * gp[d][:N], star[d][N:]]) for d in range(3)]
        new = (-1.0 / sigma) * op["SO"](pfull)
        for d, ax in enumerate("xyz"):
            new = new + (1.0 / sigma) * op["SF" + ax](gp[d]) + rho * op["SF" + ax](vel[d])
        mf = torch.where(so_empty, mf + new, new)
    return 0.5 * (vol * (vel[0][:N] ** 2 + vel[1][:N] ** 2 + vel[2][:N] ** 2)).sum()
