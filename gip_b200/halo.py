"""GIP's pressure solve split over several GPUs, one rank per GPU, with GIP_Topo's halo
exchange kept in device memory.

GIP parallelises by domain decomposition: every rank owns a slab of cells laid out
``[interiors | interfaces | boundaries | halos]`` (GIP_Topo.h:8-18), and before each
product that reads neighbours' cells, ``Vector::update`` packs the interface cells other
ranks read, exchanges them with MPI_Isend/Irecv and unpacks the halo cells it receives
(GIP_Topo.cpp:109-181, GIP_VectorMulticore.cpp:197-216).  Its Cuda Specification stages
that exchange through host memory (GIP_VectorCuda.cpp:224-247) and sums every dot product
with MPI_Allreduce (GIP_VectorCuda.cpp:158).

Here the same algorithm (GIP_LinearSolver::solve, GIP_LinearSolver.h:44-117, run for a
fixed count like GIP's) runs on each rank's part of the case as ``gip_b200.formats.
split_ranks`` writes it, in GIP's own per-rank layout and send/receive lists:

* pack and unpack are device kernels (``gipb200_gather`` / ``gipb200_scatter``); the
  exchange is torch.distributed point-to-point (NCCL between GPUs: each halo crosses
  NVLink once into this GPU's own buffer, no peer pointer is ever read by a kernel);
* the product, the update and the direction are the fused entry points
  (``gipb200_matrix_spmv_dot``, ``gipb200_cg_update_dot``, ``gipb200_cg_direction``), whose
  partial dots stay in device memory until one all-reduce per dot sums them;
* every rank takes the same collective steps in the same order.

The arithmetic per element is GIP's, so the split solve differs from the single-rank
solve only in the order of the dot products' sums.

``SlabPcg`` takes the per-element operations as an object so the exchange and reduction
logic can be exercised on CPU ranks (gloo) with a model of those operations; the device
operations (``DeviceOps``) are the product and need the CUDA library.
"""
from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from .formats import GipCase

# layout of the device scalars (gipb200_cg_scalars)
RZ, PAP, ALPHA, BETA, RR = range(5)


def jacobi_diagonal(L) -> "Csr":
    """GIP's Jacobi operator (GIP_MatrixMulticore::setUpDiagonal, GIP_MatrixMulticore.cpp:
    177-210): one entry 1/A_ii per row, the last diagonal entry of a row winning; a row
    without a diagonal stays empty (its output keeps its value)."""
    from .formats import Csr
    d = np.zeros(L.nrows)
    has = np.zeros(L.nrows, bool)
    rows = np.repeat(np.arange(L.nrows), np.diff(L.rowptr))
    on = np.nonzero(L.col == rows)[0]          # diagonal nonzeros in stored order
    d[rows[on]] = 1.0 / L.val[on]              # later entries overwrite earlier ones
    has[rows[on]] = True
    keep = np.nonzero(has)[0]
    rp = np.concatenate([[0], np.cumsum(has)]).astype(np.int32)
    return Csr(L.nrows, max(L.ncols, L.nrows), rp, keep.astype(np.int32), d[keep]), d


class DeviceOps:
    """The per-rank operations on the device, through the C ABI."""

    def __init__(self, part: GipCase, device: torch.device):
        from . import device as dv
        if device.type != "cuda":
            raise RuntimeError("DeviceOps runs on a CUDA device")
        self.dv = dv
        self.device = device
        L = part.ops["L"]
        self.n = L.nrows
        self.A = dv.DeviceMatrix(L)               # rows: inner cells, columns: all local
        Dm, d = jacobi_diagonal(L)
        self.D = dv.DeviceMatrix(Dm)
        self.dinv = self.tensor(d)

    def tensor(self, a: np.ndarray, dtype=torch.float64) -> torch.Tensor:
        return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=self.device)

    def zeros(self, n: int) -> torch.Tensor:
        return torch.zeros(n, dtype=torch.float64, device=self.device)

    def _dot_out(self, sc: torch.Tensor, k: int):
        import ctypes as C
        return C.c_void_p(sc.data_ptr() + 8 * k)

    def spmv(self, x, y):                          # y = A x (rows without nonzeros keep y)
        self.A.spmv(x, y)

    def spmv_dot(self, x, y, sc):                  # y = A x, sc[PAP] = local x.y
        from . import _lib as L
        L.call("gipb200_matrix_spmv_dot", self.A.handle, self.dv._dptr(x), self.dv._dptr(y),
               self.n, self._dot_out(sc, PAP), self.dv._stream(None))

    def jacobi_dot(self, r, p, sc):                # p = D r (GIP's diagonal SpMV), sc[RZ] = r.p
        from . import _lib as L
        L.call("gipb200_matrix_spmv_dot", self.D.handle, self.dv._dptr(r), self.dv._dptr(p),
               self.n, self._dot_out(sc, RZ), self.dv._stream(None))

    def update(self, x, r, z, p, q, sc):           # GIP_LinearSolver.h:93-111, local sums
        self.dv.cg_update_dot(self.A, self.n, x, r, z, p, q, self.dinv, sc)

    def direction(self, p, z, sc):                 # p = z + beta p
        self.dv.cg_direction(self.n, p, z, sc)

    def axpy(self, y, x, a, n):
        self.dv.axpy(y, x, a, n=n)

    def gather(self, idx, x, buf):
        from . import _lib as L
        L.call("gipb200_gather", idx.numel(), self.dv._dptr(idx), self.dv._dptr(x),
               self.dv._dptr(buf), self.dv._stream(None))

    def scatter(self, idx, buf, x):
        from . import _lib as L
        L.call("gipb200_scatter", idx.numel(), self.dv._dptr(idx), self.dv._dptr(buf),
               self.dv._dptr(x), self.dv._stream(None))


def _stage_on_host(dist, t: torch.Tensor) -> bool:
    """gloo moves host tensors only: device buffers are staged through host memory."""
    return t.is_cuda and dist is not None and dist.get_backend() == "gloo"


class HaloExchange:
    """GIP_Topo::update for one rank (GIP_Topo.cpp:176-181): pack the interface cells each
    neighbour reads, exchange them point to point, unpack the halo cells received.  With
    NCCL the device buffers go straight over NVLink; with gloo (tests of several ranks
    sharing a GPU, or CPU ranks) device buffers are staged through host memory, as GIP's
    own Cuda Specification stages every exchange (GIP_VectorCuda.cpp:224-247)."""

    def __init__(self, part: GipCase, rank: int, world: int, dist, ops):
        t = part.topo_cols
        self.rank, self.world, self.dist, self.ops = rank, world, dist, ops
        self.sends, self.recvs = [], []
        for q in range(world):
            s0, s1 = int(t.send_row[q]), int(t.send_row[q + 1])
            r0, r1 = int(t.recv_row[q]), int(t.recv_row[q + 1])
            if s1 > s0:
                idx = ops.tensor(t.send_indx[s0:s1], torch.int32)
                self.sends.append((q, idx, ops.zeros(s1 - s0)))
            if r1 > r0:
                idx = ops.tensor(t.recv_indx[r0:r1], torch.int32)
                self.recvs.append((q, idx, ops.zeros(r1 - r0)))

    def update(self, x: torch.Tensor) -> None:
        if self.world == 1:
            return
        for q, idx, buf in self.sends:
            self.ops.gather(idx, x, buf)
        host = _stage_on_host(self.dist, x)
        sb = [(q, buf.cpu() if host else buf) for q, _, buf in self.sends]
        rb = [(q, torch.empty(buf.shape, dtype=buf.dtype) if host else buf)
              for q, _, buf in self.recvs]
        P2P = self.dist.P2POp
        reqs = [P2P(self.dist.isend, b, q) for q, b in sb]
        reqs += [P2P(self.dist.irecv, b, q) for q, b in rb]
        if reqs:
            for w in self.dist.batch_isend_irecv(reqs):
                w.wait()
        for (q, idx, buf), (_, b) in zip(self.recvs, rb):
            if host:
                buf.copy_(b)
            self.ops.scatter(idx, buf, x)


class SlabPcg:
    """GIP_LinearSolver::solve on one rank's part (FIXED: exactly `maxit` iterations)."""

    def __init__(self, part: GipCase, rank: int, world: int, dist=None, ops=None,
                 device: Optional[torch.device] = None):
        self.part = part
        self.ops = ops if ops is not None else DeviceOps(part, device or torch.device("cuda"))
        self.dist = dist
        self.world = world
        self.halo = HaloExchange(part, rank, world, dist, self.ops)
        self.n = part.ops["L"].nrows                  # inner cells
        self.n_all = part.topo_cols.all         # with boundary and halo cells

    def _allreduce(self, sc: torch.Tensor, k: int) -> None:
        if self.world > 1:
            v = sc[k:k + 1].cpu() if _stage_on_host(self.dist, sc) else sc[k:k + 1].clone()
            self.dist.all_reduce(v)
            sc[k:k + 1] = v.to(sc.device)

    def solve(self, b: torch.Tensor, x0: torch.Tensor, maxit: int) -> tuple:
        """x (n_all, halos as exchanged) and the scalars (rz, pAp, alpha, beta, rr)."""
        ops, n, n_all = self.ops, self.n, self.n_all
        sc = ops.zeros(5)
        self.halo.update(x0)                          # dx0->update()        (:55)
        p = x0.clone()                                # dx0->copyTo(&dp)     (:56)
        Ax = x0.clone()                               # dx0->copyTo(&dAx)    (:66)
        x = x0.clone()                                # dx0->copyTo(dx)      (:67)
        r = ops.zeros(n_all)
        r[:n] = b[:n]                                 # db->copyTo(&dr)      (:64)
        z = ops.zeros(n_all)
        ops.spmv(x, Ax)                               # dA->spmv(dx,&dAx)    (:69)
        ops.axpy(r, Ax, -1.0, n)                      # dr.axpy(&dAx,-1.0)   (:70)
        ops.jacobi_dot(r, p, sc)                      # dp = D dr; r1 = dr.dp (:72-80)
        self._allreduce(sc, RZ)
        for _ in range(maxit):                        # :85-116
            self.halo.update(p)                       # dp.update()
            ops.spmv_dot(p, Ax, sc)                   # dAx = A dp; dn = dp.dAx
            self._allreduce(sc, PAP)
            rz_prev = sc[RZ].clone()
            ops.update(x, r, z, p, Ax, sc)            # alpha; x, r; z = D r; r.z, r.r
            self._allreduce(sc, RZ)
            self._allreduce(sc, RR)
            sc[BETA] = sc[RZ] / rz_prev               # beta = r1 / r0 over all ranks
            ops.direction(p, z, sc)                   # dp = 1.0 ds + beta dp
        return x, sc
