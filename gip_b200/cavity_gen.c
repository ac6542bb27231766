/*
 * Host-side filler for the structured cavity operators (see gip_b200/cavity.py for the
 * conventions).  Every operator of an n^3 grid has a closed-form size, so the caller
 * allocates all arrays and this file writes them with independent per-row loops.
 * It also applies a row permutation with column renumbering to a CSR operator, which
 * the seeded cell/face renumbering of the large benchmark cavity uses.
 */
#include <stdint.h>
#include <string.h>

typedef struct {
  int* rp;
  int* col;
  double* val;
} gip_csr_out;

typedef struct {
  gip_csr_out L, D, Mres, SO, SF[3], M[3], G[3], Lb, Ec;
  double *u, *v, *w, *dxs;
  int* lid_ghost;   /* n*n: ghost id under lid cell (i,j), index i + n*j */
  int* cell_k;      /* N + G: z index of every owned cell */
  int* ghost_cell;  /* G: adjacent inner cell of every ghost */
} gip_cavity_out;

static inline int64_t ghost_of(int n, int axis, int hi, int a, int b) {
  /* wall face -> ghost index, ghost cells numbered in wall-face id order:
   * x walls (k, j, side), y walls (k, side, i), z walls (side, j, i) */
  const int64_t n2 = (int64_t)n * n;
  if (axis == 0) return 2 * ((int64_t)a + (int64_t)n * b) + hi;     /* a=j, b=k */
  if (axis == 1) return 2 * n2 + ((int64_t)b * 2 + hi) * n + a;     /* a=i, b=k */
  return 4 * n2 + (int64_t)hi * n2 + (int64_t)b * n + a;            /* a=i, b=j */
}

int gip_cavity_fill(int n, double re, double lid, const double* lid_profile, int ghost_cols,
                    gip_cavity_out* o) {
  if (n < 2) return 1;
  const int64_t N = (int64_t)n * n * n, n2 = (int64_t)n * n;
  const int64_t Fx = (int64_t)(n + 1) * n2, F = 3 * Fx;
  const double h = 1.0 / n, A = h * h, vol = h * h * h, nu = 1.0 / re;
  const int64_t pin = (n / 2) + (int64_t)n * (n / 2) + n2 * (n / 2);
  const int64_t strides[3] = {1, n, n2};

#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < N; ++c) {
    const int ci = (int)(c % n), cj = (int)((c / n) % n), ck = (int)(c / n2);
    const int coord[3] = {ci, cj, ck};
    int lo_b[3], hi_b[3];
    for (int d = 0; d < 3; ++d) {
      lo_b[d] = coord[d] == 0;
      hi_b[d] = coord[d] == n - 1;
    }
    /* faces of the cell, ascending: xm, xp, ym, yp, zm, zp */
    const int64_t fxm = ci + (int64_t)(n + 1) * (cj + (int64_t)n * ck);
    const int64_t fym = Fx + ci + (int64_t)n * (cj + (int64_t)(n + 1) * ck);
    const int64_t fzm = 2 * Fx + ci + (int64_t)n * (cj + (int64_t)n * ck);
    const int64_t faces[6] = {fxm, fxm + 1, fym, fym + n, fzm, fzm + n2};
    int isb[6];
    double sgn[6];
    int64_t gh[6];
    for (int d = 0; d < 3; ++d) {
      isb[2 * d] = lo_b[d];
      isb[2 * d + 1] = hi_b[d];
      sgn[2 * d] = lo_b[d] ? 1.0 : -1.0;
      sgn[2 * d + 1] = 1.0;
    }
    {
      /* ghost ids of wall faces */
      int a0[3] = {cj, ci, ci}, b0[3] = {ck, ck, cj};
      for (int d = 0; d < 3; ++d) {
        gh[2 * d] = lo_b[d] ? N + ghost_of(n, d, 0, a0[d], b0[d]) : -1;
        gh[2 * d + 1] = hi_b[d] ? N + ghost_of(n, d, 1, a0[d], b0[d]) : -1;
      }
    }
    int nint = 0;
    for (int f = 0; f < 6; ++f) nint += !isb[f];

    /* ---- L and D: [zm, ym, xm, diag, xp, yp, zp] then ghosts [xm, xp, ym, yp, zm, zp] */
    {
      const int64_t nbc[7] = {c - n2, c - n, c - 1, c, c + 1, c + n, c + n2};
      const int nbv[7] = {!lo_b[2], !lo_b[1], !lo_b[0], 1, !hi_b[0], !hi_b[1], !hi_b[2]};
      double dnb = nu * (A / h) / vol, dg = nu * A / (0.5 * h) / vol;
      double offsum = 0.0;
      for (int s = 0; s < 7; ++s)
        if (s != 3 && nbv[s]) offsum += dnb;
      for (int g = 0; g < 6; ++g)
        if (isb[g]) offsum += dg;
      int64_t k = ghost_cols ? 7 * c : 0;
      int64_t kl;
      if (ghost_cols) {
        kl = 7 * c;
      } else {
        /* rows without ghost columns: offset = 7c minus walls of earlier cells; the
         * caller passes rowptr precomputed for this case (L.rp), read it */
        kl = o->L.rp[c];
      }
      int64_t kd = k;
      for (int s = 0; s < 7; ++s) {
        if (!nbv[s]) continue;
        double lv = (s == 3) ? nint * (A / h) : -(A / h);
        if (s == 3 && c == pin) lv = lv + lv / 101.0;
        o->L.col[kl] = (int)nbc[s];
        o->L.val[kl] = lv;
        kl++;
        if (ghost_cols) {
          o->D.col[kd] = (int)nbc[s];
          o->D.val[kd] = (s == 3) ? -offsum : dnb;
          kd++;
        }
      }
      if (ghost_cols) {
        for (int g = 0; g < 6; ++g) {
          if (!isb[g]) continue;
          o->L.col[kl] = (int)gh[g];
          o->L.val[kl] = 0.0;
          kl++;
          o->D.col[kd] = (int)gh[g];
          o->D.val[kd] = dg;
          kd++;
        }
        o->L.rp[c + 1] = (int)(7 * (c + 1));
        o->D.rp[c + 1] = (int)(7 * (c + 1));
      }
    }
    if (!ghost_cols) continue;

    /* ---- Mres */
    for (int f = 0; f < 6; ++f) {
      o->Mres.col[6 * c + f] = (int)faces[f];
      o->Mres.val[6 * c + f] = sgn[f];
    }
    o->Mres.rp[c + 1] = (int)(6 * (c + 1));

    /* ---- M_d and G_d: [lower nb, diag (wall along d), upper nb], 2 entries per row */
    for (int d = 0; d < 3; ++d) {
      const int lo_ok = !lo_b[d], hi_ok = !hi_b[d];
      const double diag = (lo_ok ? 0.5 * A : 0.0) + (hi_ok ? -0.5 * A : 0.0);
      int64_t k = 2 * c;
      if (lo_ok) {
        o->M[d].col[k] = (int)(c - strides[d]);
        o->M[d].val[k] = 0.5 * A;
        o->G[d].col[k] = (int)(c - strides[d]);
        o->G[d].val[k] = -0.5 * A / vol;
        k++;
      }
      if (diag != 0.0) {
        o->M[d].col[k] = (int)c;
        o->M[d].val[k] = diag;
        o->G[d].col[k] = (int)c;
        o->G[d].val[k] = diag / vol;
        k++;
      }
      if (hi_ok) {
        o->M[d].col[k] = (int)(c + strides[d]);
        o->M[d].val[k] = -0.5 * A;
        o->G[d].col[k] = (int)(c + strides[d]);
        o->G[d].val[k] = 0.5 * A / vol;
        k++;
      }
      o->M[d].rp[c + 1] = (int)(2 * (c + 1));
      o->G[d].rp[c + 1] = (int)(2 * (c + 1));
    }

    /* ---- Ec: D's slots in D's order; 1 entry per neighbour/ghost slot, 6 for the diagonal */
    {
      int wall = 0;
      for (int f = 0; f < 6; ++f) wall |= isb[f];
      const int64_t nbface[7] = {faces[4], faces[2], faces[0], -1, faces[1], faces[3], faces[5]};
      const double nbsgn[7] = {-1.0, -1.0, -1.0, 0.0, 1.0, 1.0, 1.0};
      const int nbv[7] = {!lo_b[2], !lo_b[1], !lo_b[0], 1, !hi_b[0], !hi_b[1], !hi_b[2]};
      int64_t k = 12 * c;    /* nonzero position */
      int64_t r = 7 * c;     /* Ec row = D nonzero index */
      for (int s = 0; s < 7; ++s) {
        if (!nbv[s]) continue;
        if (s == 3) {
          for (int f = 0; f < 6; ++f) {
            o->Ec.col[k] = (int)faces[f];
            o->Ec.val[k] = (wall && !isb[f]) ? sgn[f] * (0.5 / vol) : 0.0;
            k++;
          }
        } else {
          o->Ec.col[k] = (int)nbface[s];
          o->Ec.val[k] = (0.5 * nbsgn[s]) / vol;
          k++;
        }
        o->Ec.rp[r + 1] = (int)k;
        r++;
      }
      for (int g = 0; g < 6; ++g) {
        if (!isb[g]) continue;
        o->Ec.col[k] = (int)faces[g];
        o->Ec.val[k] = 1.0 / vol;
        k++;
        o->Ec.rp[r + 1] = (int)k;
        r++;
      }
    }

    /* ---- fields and ghost bookkeeping */
    o->u[c] = 0.0;
    o->v[c] = 0.0;
    o->w[c] = 0.0;
    o->dxs[c] = h;
    o->cell_k[c] = ck;
    for (int f = 0; f < 6; ++f) {
      if (!isb[f]) continue;
      const int64_t g = gh[f];
      o->ghost_cell[g - N] = (int)c;
      o->cell_k[g] = ck;
      o->u[g] = 0.0;
      o->v[g] = 0.0;
      o->w[g] = 0.0;
      o->dxs[g] = 0.0;
      if (f == 5) { /* lid: top face z = 1, moving along +x */
        o->lid_ghost[ci + (int64_t)n * cj] = (int)g;
        o->u[g] = lid_profile ? lid_profile[ci * (int64_t)n + cj] : lid;
      }
    }
  }
  if (!ghost_cols) return 0;
  o->L.rp[0] = o->D.rp[0] = o->Mres.rp[0] = o->Ec.rp[0] = 0;
  for (int d = 0; d < 3; ++d) {
    o->M[d].rp[0] = o->G[d].rp[0] = 0;
    for (int64_t g = N + 1; g <= N + 6 * n2; ++g) o->G[d].rp[g] = (int)(2 * N); /* ghost rows empty */
  }

  /* ---- face rows: SO and SF_d, 2 entries per interior face; owner = low cell */
  {
    int64_t k = 0;
    int64_t kd[3] = {0, 0, 0};
    o->SO.rp[0] = 0;
    for (int d = 0; d < 3; ++d) o->SF[d].rp[0] = 0;
    for (int64_t f = 0; f < F; ++f) {
      const int axis = (int)(f / Fx);
      const int64_t r = f % Fx;
      int64_t a, b, cc, pos;
      if (axis == 0) {
        a = r % (n + 1); b = (r / (n + 1)) % n; cc = r / ((int64_t)(n + 1) * n); pos = a;
      } else if (axis == 1) {
        a = r % n; b = (r / n) % (n + 1); cc = r / ((int64_t)n * (n + 1)); pos = b;
      } else {
        a = r % n; b = (r / n) % n; cc = r / n2; pos = cc;
      }
      if (pos > 0 && pos < n) {
        const int64_t hi = a + (int64_t)n * b + n2 * cc;
        const int64_t lo = hi - strides[axis];
        o->SO.col[k] = (int)lo;
        o->SO.val[k] = -(A / h);
        o->SO.col[k + 1] = (int)hi;
        o->SO.val[k + 1] = A / h;
        k += 2;
        int64_t q = kd[axis];
        o->SF[axis].col[q] = (int)lo;
        o->SF[axis].val[q] = 0.5 * A;
        o->SF[axis].col[q + 1] = (int)hi;
        o->SF[axis].val[q + 1] = 0.5 * A;
        kd[axis] += 2;
      }
      o->SO.rp[f + 1] = (int)k;
      for (int d = 0; d < 3; ++d) o->SF[d].rp[f + 1] = (int)kd[d];
    }
  }
  /* ---- Lb: ghost rows copy their adjacent cell */
  {
    const int64_t G = 6 * n2;
    for (int64_t i = 0; i <= N; ++i) o->Lb.rp[i] = 0;
    for (int64_t g = 0; g < G; ++g) {
      o->Lb.col[g] = o->ghost_cell[g];
      o->Lb.val[g] = 1.0;
      o->Lb.rp[N + g + 1] = (int)(g + 1);
    }
  }
  return 0;
}

/* out row r = in row order[r]; columns through colmap (NULL = unchanged).  out_rp must be
 * filled by the caller (prefix sum of the permuted row lengths). */
void gip_permute_rows(int64_t nrows, const int* rp, const int* col, const double* val,
                      const int64_t* order, const int* colmap, const int* out_rp, int* out_col,
                      double* out_val) {
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < nrows; ++r) {
    const int64_t s = order[r];
    const int b = rp[s], e = rp[s + 1];
    int64_t o = out_rp[r];
    for (int k = b; k < e; ++k, ++o) {
      out_col[o] = colmap ? colmap[col[k]] : col[k];
      out_val[o] = val[k];
    }
  }
}
