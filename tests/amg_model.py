"""Numpy restatement of the AMG preconditioner's host setup, for the CPU tests.

Test infrastructure only: the library's own setup (gip_b200/csrc/amg.cu) is what ships.
The AMG is an addition beyond GIP (whose solver is Jacobi-PCG), so there is no reference
routine to follow; this model restates the published smoothed-aggregation method as the
library applies it, step by step, so the tests can compare level sizes and nonzero counts:

* strength: every nonzero off-diagonal coupling is strong;
* aggregation, three greedy passes over the rows in order: (1) a row whose strong
  neighbours are all free starts an aggregate with them; (2) a free row joins the aggregate
  (from pass 1) of its strongest neighbour, the first in stored order on ties; (3) each row
  still free starts an aggregate with its free neighbours; aggregates are numbered in the
  order the passes create them;
* tentative prolongator P0[i, agg(i)] = z_i / |z over agg(i)|, smoothed by one weighted
  Jacobi step, P = (I - w D^-1 A) P0 with w = 4 / (3 rho), rho the Gershgorin bound of
  D^-1 A; coarse near-null vector = the aggregate norms;
* Galerkin coarse operator R A P with R = P^T (every structural product entry kept);
* sparsification: values made symmetric, couplings with |a_ij| < theta sqrt(a_ii a_jj)
  dropped and lumped onto the diagonal as a_ij z_j / z_i; a row whose diagonal would fall
  to half or less keeps its couplings (rows marked in order; a second failure leaves the
  level unsparsified);
* the first level of at most 1024 rows (below the finest) is the coarsest.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

COARSE = 1024


def aggregate(A: sp.csr_matrix):
    n = A.shape[0]
    rp, ci, v = A.indptr, A.indices, A.data

    def strong(i):
        return [k for k in range(rp[i], rp[i + 1]) if ci[k] != i and v[k] != 0.0]

    agg = -np.ones(n, np.int64)
    na = 0
    for i in range(n):  # pass 1
        if agg[i] != -1:
            continue
        ks = strong(i)
        if not ks or any(agg[ci[k]] != -1 for k in ks):
            continue
        agg[i] = na
        for k in ks:
            agg[ci[k]] = na
        na += 1
    first = agg.copy()
    for i in range(n):  # pass 2
        if first[i] != -1:
            continue
        best, bw = -1, 0.0
        for k in strong(i):
            if first[ci[k]] >= 0 and abs(v[k]) > bw:
                bw, best = abs(v[k]), first[ci[k]]
        if best >= 0:
            agg[i] = best
    for i in range(n):  # pass 3
        if agg[i] != -1:
            continue
        agg[i] = na
        for k in strong(i):
            if agg[ci[k]] == -1:
                agg[ci[k]] = na
        na += 1
    return agg, na


def prolongator(A: sp.csr_matrix, d, agg, p0, na: int, w: float) -> sp.csr_matrix:
    """(I - w D^-1 A) P0 with every aggregate a row touches stored (no cancellation)."""
    rows, cols, vals = [], [], []
    rp, ci, v = A.indptr, A.indices, A.data
    for i in range(A.shape[0]):
        e = {agg[i]: p0[i]}
        s = w / d[i]
        for k in range(rp[i], rp[i + 1]):
            j = ci[k]
            e[agg[j]] = e.get(agg[j], 0.0) - s * v[k] * p0[j]
        for c, val in e.items():
            rows.append(i)
            cols.append(c)
            vals.append(val)
    P = sp.coo_matrix((vals, (rows, cols)), shape=(A.shape[0], na)).tocsr()
    return P


def _pattern(M: sp.csr_matrix) -> sp.csr_matrix:
    B = M.copy().tocsr()
    B.data = np.ones_like(B.data)
    return B


def galerkin(A: sp.csr_matrix, P: sp.csr_matrix):
    """Dense values and the structural pattern (row, col arrays) of P^T A P."""
    R = P.T.tocsr()
    pat = (_pattern(R) @ (_pattern(A) @ _pattern(P))).tocoo()
    dense = (R @ (A @ P)).toarray()
    return dense, pat.row, pat.col


def sparsify(dense, prow, pcol, z, theta):
    """Returns (rows, cols, vals) of the sparsified operator (or the input when a row
    fails twice)."""
    n = dense.shape[0]
    sym = 0.5 * (dense + dense.T)
    d = np.diag(sym).copy()
    order = np.lexsort((pcol, prow))
    prow, pcol = prow[order], pcol[order]
    starts = np.searchsorted(prow, np.arange(n + 1))
    keep = np.zeros(n, bool)

    def droppable(i, j):
        a = sym[i, j]
        return (j != i and z[i] != 0.0 and z[j] != 0.0 and not keep[i] and not keep[j]
                and abs(a) < theta * np.sqrt(d[i] * d[j]))

    def lumped(i):
        return sum(sym[i, j] * z[j] / z[i] for j in pcol[starts[i]:starts[i + 1]]
                   if droppable(i, j))

    for i in range(n):
        if not (d[i] + lumped(i) > 0.5 * d[i]):
            keep[i] = True
    for i in range(n):
        if not keep[i] and not (d[i] + lumped(i) > 0.5 * d[i]):
            return prow, pcol, dense[prow, pcol]
    rows, cols, vals = [], [], []
    for i in range(n):
        lump = lumped(i)
        for j in pcol[starts[i]:starts[i + 1]]:
            if droppable(i, j):
                continue
            rows.append(i)
            cols.append(j)
            vals.append(sym[i, j] + (lump if j == i else 0.0))
    return np.array(rows), np.array(cols), np.array(vals)


def hierarchy(A: sp.csr_matrix, z, drop: float, max_levels: int = 16):
    """[(rows, nnz)] per level, finest first."""
    A = A.tocsr()
    z = np.asarray(z, float)
    out = []
    for level in range(max_levels):
        d = A.diagonal()
        out.append((A.shape[0], A.nnz))
        if A.shape[0] <= COARSE and level > 0:
            return out
        rho = max(float(np.max(np.asarray(abs(A).sum(axis=1)).ravel() / d)), 1e-300)
        w = 4.0 / (3.0 * rho)
        agg, na = aggregate(A)
        nrm = np.sqrt(np.bincount(agg, weights=z * z, minlength=na))
        p0 = np.where(nrm[agg] > 0, z / np.where(nrm[agg] > 0, nrm[agg], 1.0), 0.0)
        P = prolongator(A, d, agg, p0, na, w)
        dense, prow, pcol = galerkin(A, P)
        if drop > 0:
            r, c, v = sparsify(dense, prow, pcol, nrm, drop)
        else:
            r, c, v = prow, pcol, dense[prow, pcol]
        A = sp.csr_matrix((v, (r, c)), shape=(na, na))
        A.sum_duplicates()
        z = nrm
    return out
