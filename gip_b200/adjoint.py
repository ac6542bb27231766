"""FP64 discrete adjoint of the timestep behind a ``torch.autograd.Function``.

``CavityAdjoint`` holds a device engine (``gipb200_adjoint_*``) for one case; ``energy(lid,
nu)`` returns the kinetic energy after ``nsteps`` timesteps as a differentiable torch
scalar whose gradient with respect to the lid's ghost velocities and the viscosity comes
from the hand-written adjoint (transposed SpMVs, adjoint Poisson solve, convective
adjoint), not from taping.  The CFL steps of the first forward are frozen and reused.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import _lib as L
from .device import _host_csr, _hptr
from .formats import GipCase


class CavityAdjoint:
    def __init__(self, case: GipCase, lid_cells: np.ndarray, volume: np.ndarray, nu0: float,
                 rho: float = 1.0, gamma: float = 1e-3, tol: float = 1e-12, maxit: int = 20000,
                 checkpoint_every: int = 10, precond: str = "jacobi"):
        keep: list = []
        self._ops = L.DnsOps(**{n: _host_csr(case.ops[n], keep) for n in L.DNS_OPS},
                             n_inner=case.n_inner, n_owned=case.n_owned, n_faces=case.n_faces)
        self._keep = keep
        f = {k: np.ascontiguousarray(case.fields[k], np.float64) for k in ("u", "v", "w", "dxs")}
        self.lid_cells = np.ascontiguousarray(lid_cells, np.int32)
        vol = np.ascontiguousarray(volume, np.float64)
        self.nu0 = nu0
        from .device import PRECONDS
        prm = L.AdjointParams(rho, gamma, nu0, tol, maxit, checkpoint_every, PRECONDS[precond])
        h = C.c_void_p()
        L.call("gipb200_adjoint_create", C.byref(self._ops), _hptr(f["u"]), _hptr(f["v"]),
               _hptr(f["w"]), _hptr(f["dxs"]), _hptr(vol), _hptr(self.lid_cells),
               self.lid_cells.size, C.byref(prm), C.byref(h))
        self.handle = h
        self.dt: Optional[np.ndarray] = None

    def forward(self, lid: np.ndarray, nu: float, nsteps: int, freeze_dt: bool = True) -> float:
        """J after nsteps; the first call records the CFL steps, later calls reuse them."""
        lid = np.ascontiguousarray(lid, np.float64)
        J = C.c_double()
        given = int(freeze_dt and self.dt is not None and self.dt.size == nsteps)
        dt = self.dt if given else np.zeros(nsteps)
        L.call("gipb200_adjoint_forward", self.handle, _hptr(lid), nu / self.nu0, nsteps,
               _hptr(dt), given, C.byref(J))
        if not given:
            self.dt = dt
        return J.value

    def backward(self) -> tuple:
        g = np.zeros(self.lid_cells.size)
        gn = C.c_double()
        L.call("gipb200_adjoint_backward", self.handle, _hptr(g), C.byref(gn))
        return g, gn.value

    def energy(self, lid: torch.Tensor, nu: torch.Tensor, nsteps: int) -> torch.Tensor:
        return _KineticEnergy.apply(lid, nu, self, nsteps)

    def close(self):
        if getattr(self, "handle", None):
            L.load().gipb200_adjoint_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _KineticEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, lid, nu, adj: CavityAdjoint, nsteps: int):
        J = adj.forward(lid.detach().cpu().double().numpy(), float(nu), nsteps)
        ctx.adj = adj
        ctx.dev = lid.device
        return torch.tensor(J, dtype=torch.float64, device=lid.device)

    @staticmethod
    def backward(ctx, gJ):
        g, gn = ctx.adj.backward()
        s = gJ.detach().to(torch.float64)
        gl = torch.from_numpy(g).to(ctx.dev) * s
        gnu = torch.tensor(gn, dtype=torch.float64, device=ctx.dev) * s
        return gl, gnu, None, None
