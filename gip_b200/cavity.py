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


def _compress(rows_cols: np.ndarray, rows_vals: np.ndarray, valid: np.ndarray, ncols: int) -> Csr:
    """Rows given as fixed-width slot arrays (nrows x K) with a validity mask; the slot
    order is the nonzero order."""
    nrows = rows_cols.shape[0]
    counts = valid.sum(axis=1).astype(np.int64)
    rowptr = np.zeros(nrows + 1, np.int64)
    np.cumsum(counts, out=rowptr[1:])
    col = rows_cols[valid].astype(np.int32)
    val = rows_vals[valid].astype(np.float64)
    return Csr(nrows, ncols, rowptr.astype(np.int32), col, val)


def generate(n: int, re: float = 100.0, lid: float = 1.0,
             lid_profile: Optional[np.ndarray] = None, permute_seed: Optional[int] = None,
             ghost_cols: bool = True) -> tuple:
    """Return ``(GipCase, CavityMeta)`` for an ``n^3`` cavity at Reynolds number ``re``
    (``nu = 1/re`` is baked into D).  ``lid_profile`` (n x n, indexed [i, j]) overrides
    the uniform lid velocity on the top face."""
    if n < 2:
        raise ValueError("n must be >= 2")
    h = 1.0 / n
    N = n ** 3
    A = h * h
    vol = h ** 3
    nu = 1.0 / re
    Fx = (n + 1) * n * n
    F = 3 * Fx
    idx = np.arange(N, dtype=np.int64)
    ci = idx % n
    cj = (idx // n) % n
    ck = idx // (n * n)

    # ---- faces of every cell, ascending id: xm, xp, ym, yp, zm, zp
    fxm = ci + (n + 1) * (cj + n * ck)
    fym = Fx + ci + n * (cj + (n + 1) * ck)
    fzm = 2 * Fx + ci + n * (cj + n * ck)
    cell_faces = np.stack([fxm, fxm + 1, fym, fym + n, fzm, fzm + n * n], axis=1)
    lo_bnd = np.stack([ci == 0, cj == 0, ck == 0], axis=1)          # xm/ym/zm are walls
    hi_bnd = np.stack([ci == n - 1, cj == n - 1, ck == n - 1], axis=1)
    face_is_bnd = np.empty((N, 6), bool)
    face_is_bnd[:, 0::2] = lo_bnd
    face_is_bnd[:, 1::2] = hi_bnd
    # Mres: +1 where the normal points out of the cell (the high face, or a wall face)
    mres_sign = np.empty((N, 6))
    mres_sign[:, 1::2] = 1.0
    mres_sign[:, 0::2] = np.where(lo_bnd, 1.0, -1.0)

    # ---- wall faces -> ghost cells, in wall-face id order
    bface_ids = np.sort(cell_faces[face_is_bnd])
    G = bface_ids.shape[0]
    ghost_of_face = np.full(F, -1, np.int64)
    ghost_of_face[bface_ids] = N + np.arange(G)
    ghost_slot = np.where(face_is_bnd, ghost_of_face[cell_faces], -1)   # N x 6
    # adjacent inner cell of every ghost
    ghost_cell = np.empty(G, np.int64)
    rr, ss = np.nonzero(face_is_bnd)
    ghost_cell[ghost_slot[rr, ss] - N] = rr
    NO = N + G

    strides = np.array([1, n, n * n], np.int64)
    lo_nb = idx[:, None] - strides[None, :]   # x-1, y-1, z-1
    hi_nb = idx[:, None] + strides[None, :]

    # ---- L and D share one sparsity: [zm, ym, xm, diag, xp, yp, zp, ghosts(6)]
    nb_cols = np.stack([lo_nb[:, 2], lo_nb[:, 1], lo_nb[:, 0], idx,
                        hi_nb[:, 0], hi_nb[:, 1], hi_nb[:, 2]], axis=1)
    nb_valid = np.stack([~lo_bnd[:, 2], ~lo_bnd[:, 1], ~lo_bnd[:, 0], np.ones(N, bool),
                         ~hi_bnd[:, 0], ~hi_bnd[:, 1], ~hi_bnd[:, 2]], axis=1)
    # interior faces of each neighbour slot, with the cell's Mres sign on that face
    nb_face = np.stack([cell_faces[:, 4], cell_faces[:, 2], cell_faces[:, 0], np.zeros(N, np.int64),
                        cell_faces[:, 1], cell_faces[:, 3], cell_faces[:, 5]], axis=1)
    nb_sign = np.array([-1.0, -1.0, -1.0, 0.0, 1.0, 1.0, 1.0])
    n_int = nb_valid.sum(axis=1) - 1

    Lv = np.where(nb_valid, -(A / h), 0.0)
    Lv[:, 3] = n_int * (A / h)
    pin = int((n // 2) + n * (n // 2) + n * n * (n // 2))
    Lv[pin, 3] = Lv[pin, 3] + Lv[pin, 3] / 101.0
    Dv = np.where(nb_valid, nu * (A / h) / vol, 0.0)
    gcols = ghost_slot
    gvalid = face_is_bnd
    Dg = np.where(gvalid, nu * A / (0.5 * h) / vol, 0.0)
    offsum = np.where(nb_valid[:, [0, 1, 2, 4, 5, 6]], Dv[:, [0, 1, 2, 4, 5, 6]], 0.0).sum(axis=1)
    offsum = offsum + Dg.sum(axis=1)
    Dv[:, 3] = -offsum

    if ghost_cols:
        ld_cols = np.concatenate([nb_cols, gcols], axis=1)
        ld_valid = np.concatenate([nb_valid, gvalid], axis=1)
        L = _compress(ld_cols, np.concatenate([Lv, np.zeros((N, 6))], axis=1), ld_valid, NO)
        D = _compress(ld_cols, np.concatenate([Dv, Dg], axis=1), ld_valid, NO)
    else:
        L = _compress(nb_cols, Lv, nb_valid, NO)
        D = None

    # ---- Mres (N x F)
    Mres = _compress(cell_faces, mres_sign, np.ones((N, 6), bool), F)

    # ---- SO, SF (F rows); the owner is the low cell of an interior face
    f = np.arange(F, dtype=np.int64)
    axis = f // Fx
    r = f % Fx
    # decode (a, b, c) with the face coordinate along `axis` having n+1 values
    fa = np.empty(F, np.int64); fb = np.empty(F, np.int64); fc = np.empty(F, np.int64)
    m0 = axis == 0
    fa[m0] = r[m0] % (n + 1); fb[m0] = (r[m0] // (n + 1)) % n; fc[m0] = r[m0] // ((n + 1) * n)
    m1 = axis == 1
    fa[m1] = r[m1] % n; fb[m1] = (r[m1] // n) % (n + 1); fc[m1] = r[m1] // (n * (n + 1))
    m2 = axis == 2
    fa[m2] = r[m2] % n; fb[m2] = (r[m2] // n) % n; fc[m2] = r[m2] // (n * n)
    fpos = np.where(m0, fa, np.where(m1, fb, fc))        # coordinate along the normal
    interior_face = (fpos > 0) & (fpos < n)
    hi_cell = fa + n * fb + n * n * fc                     # the cell above the face
    lo_cell = hi_cell - strides[axis]
    so_cols = np.stack([lo_cell, hi_cell], axis=1)
    so_vals = np.stack([np.full(F, -(A / h)), np.full(F, A / h)], axis=1)
    so_valid = np.stack([interior_face, interior_face], axis=1)
    so_cols = np.where(so_valid, so_cols, 0)
    SO = _compress(so_cols, so_vals, so_valid, NO)
    SF = []
    for d in range(3):
        v = interior_face & (axis == d)
        SF.append(_compress(so_cols, np.full((F, 2), 0.5 * A), np.stack([v, v], axis=1), NO))

    # ---- M_d = -Mres SF_d : [lower nb, diag (walls along d), upper nb]
    Md, Gd = [], []
    for d in range(3):
        lo_ok = ~lo_bnd[:, d]
        hi_ok = ~hi_bnd[:, d]
        lo_v = np.where(lo_ok, 0.5 * A, 0.0)           # -(-1)(A/2)
        hi_v = np.where(hi_ok, -0.5 * A, 0.0)          # -(+1)(A/2)
        diag = (np.where(lo_ok, 0.5 * A, 0.0) + np.where(hi_ok, -0.5 * A, 0.0))
        cols = np.stack([lo_nb[:, d], idx, hi_nb[:, d]], axis=1)
        vals = np.stack([lo_v, diag, hi_v], axis=1)
        valid = np.stack([lo_ok, diag != 0.0, hi_ok], axis=1)
        Md.append(_compress(np.where(valid, cols, 0), vals, valid, NO))
        # G_d(i, j) = M_d(j, i) / Omega_i : lower nb j=i-s holds M_d(i-s, i) = -A/2
        gvals = np.stack([np.where(lo_ok, -0.5 * A, 0.0), diag, np.where(hi_ok, 0.5 * A, 0.0)],
                         axis=1) / vol
        gcols_d = np.where(valid, cols, 0)
        gm = np.zeros((NO, 3), bool); gm[:N] = valid
        gc = np.zeros((NO, 3), np.int64); gc[:N] = gcols_d
        gv = np.zeros((NO, 3)); gv[:N] = gvals
        Gd.append(_compress(gc, gv, gm, NO))

    # ---- Lb: ghost rows copy their adjacent cell
    lb_valid = np.zeros((NO, 1), bool); lb_valid[N:, 0] = True
    lb_cols = np.zeros((NO, 1), np.int64); lb_cols[N:, 0] = ghost_cell
    Lb = _compress(lb_cols, np.ones((NO, 1)), lb_valid, NO)

    # ---- Ec: rows follow D's nonzeros.  Per cell the entries are laid out as
    # [zm, ym, xm neighbour slots | 6 diagonal-slot faces | xp, yp, zp | 6 ghost slots]
    Ec = None
    if ghost_cols:
        wall_cell = face_is_bnd.any(axis=1)
        half = 0.5 / vol
        diag_vals = np.where(wall_cell[:, None] & ~face_is_bnd, mres_sign * half, 0.0)
        ec_cols = np.empty((N, 18), np.int32)
        ec_vals = np.empty((N, 18))
        ec_valid = np.empty((N, 18), bool)
        for s_, dst in ((0, 0), (1, 1), (2, 2), (4, 9), (5, 10), (6, 11)):
            ec_cols[:, dst] = nb_face[:, s_]
            ec_vals[:, dst] = (0.5 * nb_sign[s_]) / vol
            ec_valid[:, dst] = nb_valid[:, s_]
        ec_cols[:, 3:9] = cell_faces
        ec_vals[:, 3:9] = diag_vals
        ec_valid[:, 3:9] = True
        ec_cols[:, 12:18] = cell_faces
        ec_vals[:, 12:18] = 1.0 / vol
        ec_valid[:, 12:18] = gvalid
        counts = ec_valid.sum(axis=1)
        col = ec_cols[ec_valid]
        val = ec_vals[ec_valid]
        del ec_cols, ec_vals
        # row lengths in D's slot order: 1 per neighbour/ghost slot, 6 for the diagonal
        slot_len = np.concatenate([nb_valid.astype(np.int64), gvalid.astype(np.int64)], axis=1)
        slot_len[:, 3] = 6
        lens = slot_len[np.concatenate([nb_valid, gvalid], axis=1)]
        rowptr = np.zeros(lens.shape[0] + 1, np.int64)
        np.cumsum(lens, out=rowptr[1:])
        assert int(rowptr[-1]) == int(counts.sum())
        Ec = Csr(lens.shape[0], F, rowptr.astype(np.int32), col.astype(np.int32), val)

    # ---- fields
    u = np.zeros(NO); v = np.zeros(NO); w = np.zeros(NO); dxs = np.zeros(NO)
    dxs[:N] = h
    top = np.nonzero(hi_bnd[:, 2])[0]                  # cells under the lid, (i,j) order
    lid_g = ghost_slot[top, 5]
    if lid_profile is not None:
        prof = np.asarray(lid_profile, np.float64)
        if prof.shape != (n, n):
            raise ValueError("lid_profile must be n x n")
        u[lid_g] = prof[ci[top], cj[top]]
    else:
        u[lid_g] = lid

    ops = {"L": L, "Mres": Mres, "SO": SO, "SFx": SF[0], "SFy": SF[1], "SFz": SF[2],
           "Mx": Md[0], "My": Md[1], "Mz": Md[2], "Gx": Gd[0], "Gy": Gd[1], "Gz": Gd[2],
           "Lb": Lb}
    if D is not None:
        ops["D"] = D
        ops["Ec"] = Ec
    cell_k = np.concatenate([ck, ck[ghost_cell]])
    meta = CavityMeta(n, re, h, N, G, F, pin, None, None, lid_g, cell_k)
    case = GipCase(ops, {"u": u, "v": v, "w": w, "dxs": dxs},
                   Topo.single_rank(NO, N, G), Topo.single_rank(F, N, G))
    if permute_seed is not None:
        case, meta = permute(case, meta, permute_seed)
    return case, meta


def permute(case: GipCase, meta: CavityMeta, seed: int) -> tuple:
    """Renumber inner cells and faces with seeded random permutations.  Ghost cells
    keep their ids; every row keeps its nonzero order (so each product sums in the
    same order as before the renumbering)."""
    rng = np.random.default_rng(seed)
    N, NO, F = meta.n_inner, meta.n_inner + meta.n_ghost, meta.n_faces
    pc = rng.permutation(N)                    # natural cell i -> new id pc[i]
    pf = rng.permutation(F)
    cmap = np.concatenate([pc, np.arange(N, NO)])
    inv_c = np.empty(NO, np.int64); inv_c[cmap] = np.arange(NO)
    inv_f = np.empty(F, np.int64); inv_f[pf] = np.arange(F)
    row_order = {"inner": inv_c[:N], "owned": inv_c, "face": inv_f}
    from .formats import OPERATOR_SPACES, _row_nnz_index
    ops = {}
    for name, m in case.ops.items():
        rk, ck = OPERATOR_SPACES[name]
        if name == "Ec":
            continue
        order = row_order[rk][:m.nrows] if rk != "face" else row_order["face"]
        idx = _row_nnz_index(m.rowptr, order)
        lens = (m.rowptr[order + 1] - m.rowptr[order]).astype(np.int64)
        rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
        cm = cmap if ck == "cell" else pf
        ops[name] = Csr(m.nrows, m.ncols, rp, cm[m.col[idx]].astype(np.int32), m.val[idx])
    if "Ec" in case.ops:
        D = case.ops["D"]
        ec_rows = _row_nnz_index(D.rowptr, inv_c[:N])
        m = case.ops["Ec"]
        idx = _row_nnz_index(m.rowptr, ec_rows)
        lens = (m.rowptr[ec_rows + 1] - m.rowptr[ec_rows]).astype(np.int64)
        rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
        ops["Ec"] = Csr(m.nrows, m.ncols, rp, pf[m.col[idx]].astype(np.int32), m.val[idx])
    fields = {k: x[inv_c] for k, x in case.fields.items()}
    cell_k = meta.cell_k[inv_c]
    meta2 = dataclasses.replace(meta, pin_cell=int(pc[meta.pin_cell]), cell_perm=pc,
                                face_perm=pf, cell_k=cell_k)
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
