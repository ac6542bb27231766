"""Structured lid-driven-cavity operators in GIP's algebraic form.

GIP ships operators for one tetrahedral cavity (C100K) and no generator.  This module
emits the same fifteen operators for a uniform ``n^3`` hexahedral grid of the unit
cube, following the conventions the shipped operators obey (checked on C100K merged
to one rank):

* ``Mres`` -- face/cell incidence (N x F), +1 where the face normal points out of the
  cell.  Boundary faces point out of the domain.
* ``SO`` -- ``A/delta * (p_nb - p_own)`` per interior face (own = the +1 cell); rows of
  boundary faces are empty, so no mass crosses a wall.
* ``SF{x,y,z}`` -- ``A n_d / 2`` on both cells of an interior face.
* ``L = -Mres SO`` on the inner block, plus one pinned diagonal ``L_pp += L_pp / 101``
  (homogeneous Neumann made SPD), with stored zeros at ghost columns.
* ``D_ij = nu (-L_ij) / Omega_i``; a wall face adds ``nu A / (delta_b Omega_i)`` at the
  ghost column with delta_b the centre-to-face distance; ``D_ii = -sum_j D_ij``.
* ``M_d = -Mres SF_d``; ``G_d = Omega^-1 M_d^T`` on inner rows, ghost rows empty.
* ``Ec`` -- one row per nonzero of D (the product ``Ec.mf`` is C's value array,
  GIP_DNS.h:312): neighbour slot ``Mres/(2 Omega)`` on the shared face, ghost slot
  ``Mres/Omega`` on the wall face, diagonal slot ``Mres/(2 Omega)`` on the interior faces
  of wall-adjacent cells and 0 elsewhere.
* ``Lb`` -- ghost row -> adjacent inner cell, weight 1 (Neumann ghost copy of p).
* fields: u = lid velocity on the lid's ghost cells (top face z=1, along +x), zero
  elsewhere; ``dxs = h`` on inner cells.

Cells are numbered ``i + n*j + n*n*k`` (x fastest); ghost cells follow the inner ones
in the order of their wall faces.  Faces are numbered x-faces, then y-, then z-faces.
Every row lists its nonzeros in ascending column order.  An optional seeded random
permutation renumbers inner cells and faces (rows keep their nonzero order).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Optional

import numpy as np

from .formats import Csr, GipCase, Topo


@dataclasses.dataclass
class CavityMeta:
    n: int
    re: float
    h: float
    n_inner: int
    n_ghost: int
    n_faces: int
    pin_cell: int
    cell_perm: Optional[np.ndarray]   # new id of natural inner cell i (None = identity)
    face_perm: Optional[np.ndarray]   # new id of natural face f
    lid_ghosts: np.ndarray            # ghost ids (global) of the lid cells, lid (i,j) order
    cell_k: np.ndarray                # z index of every owned cell (inner + ghost), new order


class _CsrOut(C.Structure):
    _fields_ = [("rp", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p)]


class _CavityOut(C.Structure):
    _fields_ = [("L", _CsrOut), ("D", _CsrOut), ("Mres", _CsrOut), ("SO", _CsrOut),
                ("SF", _CsrOut * 3), ("M", _CsrOut * 3), ("G", _CsrOut * 3), ("Lb", _CsrOut),
                ("Ec", _CsrOut), ("u", C.c_void_p), ("v", C.c_void_p), ("w", C.c_void_p),
                ("dxs", C.c_void_p), ("lid_ghost", C.c_void_p), ("cell_k", C.c_void_p),
                ("ghost_cell", C.c_void_p)]


_host = None


def _hostlib():
    global _host
    if _host is None:
        from . import build
        path = build.build_host()
        _host = C.CDLL(path)
        _host.gip_cavity_fill.restype = C.c_int
        _host.gip_cavity_fill.argtypes = [C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_int,
                                          C.POINTER(_CavityOut)]
        _host.gip_permute_rows.restype = None
        _host.gip_permute_rows.argtypes = [C.c_int64] + [C.c_void_p] * 8
    return _host


def _p(a: Optional[np.ndarray]) -> C.c_void_p:
    return C.c_void_p(0 if a is None else a.ctypes.data)


def _alloc(nrows: int, ncols: int, nnz: int) -> tuple:
    m = Csr(nrows, ncols, np.zeros(nrows + 1, np.int32), np.zeros(nnz, np.int32),
            np.zeros(nnz, np.float64))
    return m, _CsrOut(_p(m.rowptr), _p(m.col), _p(m.val))


def generate(n: int, re: float = 100.0, lid: float = 1.0,
             lid_profile: Optional[np.ndarray] = None, permute_seed: Optional[int] = None,
             ghost_cols: bool = True) -> tuple:
    """Return ``(GipCase, CavityMeta)`` for an ``n^3`` cavity at Reynolds number ``re``
    (``nu = 1/re`` is baked into D).  ``lid_profile`` (n x n, indexed [i, j]) overrides
    the uniform lid velocity on the top face."""
    if n < 2:
        raise ValueError("n must be >= 2")
    N = n ** 3
    G = 6 * n * n
    NO = N + G
    F = 3 * (n + 1) * n * n
    h = 1.0 / n
    prof = None
    if lid_profile is not None:
        prof = np.ascontiguousarray(lid_profile, np.float64)
        if prof.shape != (n, n):
            raise ValueError("lid_profile must be n x n")
    out = _CavityOut()
    ops = {}
    if ghost_cols:
        ops["L"], out.L = _alloc(N, NO, 7 * N)
        ops["D"], out.D = _alloc(N, NO, 7 * N)
        ops["Mres"], out.Mres = _alloc(N, F, 6 * N)
        ops["SO"], out.SO = _alloc(F, NO, 6 * n * n * (n - 1))
        for d, ax in enumerate("xyz"):
            ops["SF" + ax], out.SF[d] = _alloc(F, NO, 2 * n * n * (n - 1))
            ops["M" + ax], out.M[d] = _alloc(N, NO, 2 * N)
            ops["G" + ax], out.G[d] = _alloc(NO, NO, 2 * N)
        ops["Lb"], out.Lb = _alloc(NO, NO, G)
        ops["Ec"], out.Ec = _alloc(7 * N, F, 12 * N)
    else:
        idx = np.arange(N, dtype=np.int64)
        walls = sum(((idx // s) % n == 0).astype(np.int64) + ((idx // s) % n == n - 1)
                    for s in (1, n, n * n))
        L = Csr(N, NO, np.zeros(N + 1, np.int32), None, None)
        L.rowptr[1:] = np.cumsum(7 - walls)
        L.col = np.zeros(int(L.rowptr[-1]), np.int32)
        L.val = np.zeros(int(L.rowptr[-1]))
        ops["L"] = L
        out.L = _CsrOut(_p(L.rowptr), _p(L.col), _p(L.val))
    fields = {k: np.zeros(NO) for k in ("u", "v", "w", "dxs")}
    lid_g = np.zeros(n * n, np.int32)
    cell_k = np.zeros(NO, np.int32)
    ghost_cell = np.zeros(G, np.int32)
    out.u, out.v, out.w, out.dxs = (_p(fields[k]) for k in ("u", "v", "w", "dxs"))
    out.lid_ghost, out.cell_k, out.ghost_cell = _p(lid_g), _p(cell_k), _p(ghost_cell)
    rc = _hostlib().gip_cavity_fill(n, float(re), float(lid), _p(prof), int(ghost_cols),
                                    C.byref(out))
    if rc != 0:
        raise RuntimeError("gip_cavity_fill failed")
    pin = int((n // 2) + n * (n // 2) + n * n * (n // 2))
    meta = CavityMeta(n, re, h, N, G, F, pin, None, None, lid_g.astype(np.int64),
                      cell_k.astype(np.int64))
    case = GipCase(ops, fields, Topo.single_rank(NO, N, G), Topo.single_rank(F, N, G))
    if permute_seed is not None:
        case, meta = permute(case, meta, permute_seed)
    return case, meta


def _permute_csr(m: Csr, order: np.ndarray, colmap: Optional[np.ndarray]) -> Csr:
    rp = m.rowptr.astype(np.int64)
    lens = rp[order + 1] - rp[order]
    out_rp = np.zeros(m.nrows + 1, np.int64)
    np.cumsum(lens, out=out_rp[1:])
    out_rp = out_rp.astype(np.int32)
    col = np.zeros(m.nnz, np.int32)
    val = np.zeros(m.nnz)
    cm = None if colmap is None else np.ascontiguousarray(colmap, np.int32)
    _hostlib().gip_permute_rows(m.nrows, _p(m.rowptr), _p(m.col), _p(m.val),
                                _p(np.ascontiguousarray(order, np.int64)), _p(cm), _p(out_rp),
                                _p(col), _p(val))
    return Csr(m.nrows, m.ncols, out_rp, col, val)


def permute(case: GipCase, meta: CavityMeta, seed: int) -> tuple:
    """Renumber inner cells and faces with seeded random permutations.  Ghost cells
    keep their ids; every row keeps its nonzero order (so each product sums in the
    same order as before the renumbering)."""
    from .formats import OPERATOR_SPACES, _row_nnz_index
    rng = np.random.default_rng(seed)
    N, NO, F = meta.n_inner, meta.n_inner + meta.n_ghost, meta.n_faces
    pc = rng.permutation(N)                    # natural cell i -> new id pc[i]
    pf = rng.permutation(F)
    cmap = np.concatenate([pc, np.arange(N, NO)])
    inv_c = np.empty(NO, np.int64)
    inv_c[cmap] = np.arange(NO)
    inv_f = np.empty(F, np.int64)
    inv_f[pf] = np.arange(F)
    ops = {}
    for name, m in case.ops.items():
        if name == "Ec":
            continue
        rk, ck = OPERATOR_SPACES[name]
        order = inv_f if rk == "face" else inv_c[:m.nrows]
        ops[name] = _permute_csr(m, order, cmap if ck == "cell" else pf)
    if "Ec" in case.ops:
        ec_rows = _row_nnz_index(case.ops["D"].rowptr, inv_c[:N])
        ops["Ec"] = _permute_csr(case.ops["Ec"], ec_rows, pf)
    fields = {k: x[inv_c] for k, x in case.fields.items()}
    meta2 = dataclasses.replace(meta, pin_cell=int(pc[meta.pin_cell]), cell_perm=pc,
                                face_perm=pf, cell_k=meta.cell_k[inv_c],
                                lid_ghosts=meta.lid_ghosts)
    return GipCase(ops, fields, case.topo_cols, case.topo_faces), meta2


def slab_partition(meta: CavityMeta, nparts: int) -> np.ndarray:
    """Rank of every owned cell for a split into ``nparts`` z-slabs (ghosts follow their
    adjacent cell)."""
    if nparts < 1 or nparts > meta.n:
        raise ValueError("nparts must be in [1, n]")
    return (meta.cell_k * nparts) // meta.n


def poisson_problem(n: int, seed: int = 0) -> tuple:
    """The pressure-Poisson benchmark: the cavity's L on an ``n^3`` grid without ghost
    columns (homogeneous Neumann, one pinned cell) and a seeded right-hand side
    ``U[-1,1]`` with its mean removed.  Returns ``(Csr, rhs)``."""
    case, _ = generate(n, ghost_cols=False)
    L = case.ops["L"]
    L = Csr(L.nrows, L.nrows, L.rowptr, L.col, L.val)
    rng = np.random.default_rng(seed)
    b = rng.uniform(-1.0, 1.0, n ** 3)
    b -= b.mean()
    return L, b
