/*
 * ORACLE -- test infrastructure only (see gip_oracle.h).  Each function restates the
 * GIP routine it cites, with the same loop order and the same IEEE operations, so at
 * one rank it reproduces GIP's CPU build bit for bit.  Compiled with
 * -ffp-contract=off (no FMA contraction), like oracle/_ref.
 */
#include "gip_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* GIP_MatrixMulticore::spmv (GIP_MatrixMulticore.cpp:64-143): sequential row sum
 * `sum += x[col]*val`; rows with rowptr[i]==rowptr[i+1] are skipped. */
void orc_spmv(const orc_csr* A, const double* x, double* y, double alpha, double beta,
              int mode) {
  for (int i = 0; i < A->nrows; ++i) {
    int jb = A->rowptr[i], je = A->rowptr[i + 1];
    double sum = 0;
    for (int j = jb; j < je; ++j) sum += x[A->col[j]] * A->val[j];
    if (jb != je) y[i] = mode ? alpha * sum + beta * y[i] : sum;
  }
}

/* GIP_MatrixMulticore::setUpDiagonal (GIP_MatrixMulticore.cpp:177-210). */
int orc_inverse_diagonal(const orc_csr* A, double* dinv) {
  int missing = 0;
  for (int i = 0; i < A->nrows; ++i) {
    int found = 0;
    dinv[i] = 0.0;
    for (int j = A->rowptr[i]; j < A->rowptr[i + 1]; ++j)
      if (A->col[j] == i) {
        dinv[i] = 1.0 / A->val[j];
        found = 1;
      }
    missing += !found;
  }
  return missing;
}

/* GIP_VectorMulticore::dot (GIP_VectorMulticore.cpp:93-128): tdot += a[i]*b[i]. */
double orc_dot(int n, const double* a, const double* b) {
  double t = 0.0;
  for (int i = 0; i < n; ++i) t += a[i] * b[i];
  return t;
}

/* GIP_VectorMulticore::norm (GIP_VectorMulticore.cpp:130-164): max |a[i]|. */
double orc_norminf(int n, const double* a) {
  double t = 0.0;
  for (int i = 0; i < n; ++i)
    if (fabs(a[i]) > t) t = fabs(a[i]);
  return t;
}

/* GIP_VectorMulticore::axpy (GIP_VectorMulticore.cpp:44-67): y += alpha*x. */
static void axpy(int n, double* y, const double* x, double alpha) {
  for (int i = 0; i < n; ++i) y[i] += alpha * x[i];
}

/* GIP_VectorMulticore::axpy(x,alpha,beta) (GIP_VectorMulticore.cpp:69-92). */
static void axpby(int n, double* y, const double* x, double alpha, double beta) {
  for (int i = 0; i < n; ++i) y[i] = alpha * x[i] + beta * y[i];
}

/* Jacobi apply as GIP does it: a diagonal CSR SpMV, sum = 0 + r[i]*dinv[i]. */
static void jacobi(int n, const double* dinv, const double* r, double* z) {
  for (int i = 0; i < n; ++i) {
    double sum = 0;
    sum += r[i] * dinv[i];
    z[i] = sum;
  }
}

/* GIP_LinearSolver::solve (GIP_LinearSolver.h:44-117).  GIP runs exactly maxIt
 * iterations and never reads `tol` (:34); mode 1 adds a stopping rule checked after
 * each residual update: ||r||_2 <= tol*||b||_2 over the inner range. */
int orc_pcg(const orc_csr* A, const double* dinv, const double* b, double* x, const double* x0,
            int n_all, int maxit, int mode, double tol, double* work, double* rr_out) {
  const int n = A->nrows; /* the inner range: L has one row per inner cell */
  double* dp = work;
  double* dAx = work + n_all;
  double* dr = work + 2 * (size_t)n_all;
  double* ds = work + 3 * (size_t)n_all;
  memcpy(dp, x0, sizeof(double) * n_all);   /* dx0->copyTo(&dp,_ALL_)   :56 */
  memcpy(dr, b, sizeof(double) * n);        /* db->copyTo(&dr,_INNER_)  :65 */
  memcpy(dAx, x0, sizeof(double) * n_all);  /* dx0->copyTo(&dAx,_ALL_)  :66 */
  memcpy(x, x0, sizeof(double) * n_all);    /* dx0->copyTo(dx,_ALL_)    :67 */
  orc_spmv(A, x, dAx, 0, 0, 0);             /* :69 */
  axpy(n, dr, dAx, -1.0);                   /* :70 */
  jacobi(n, dinv, dr, dp);                  /* :74 */
  double r1 = orc_dot(n, dr, dp);           /* :80 */
  double bb = 0, rr = 0;
  if (mode == 1) {
    bb = orc_dot(n, b, b);
    rr = orc_dot(n, dr, dr);
    if (!(sqrt(rr) > tol * sqrt(bb))) {
      if (rr_out) *rr_out = rr;
      return 0;
    }
  }
  int k = 1;
  while (k <= maxit) {                      /* :85 */
    orc_spmv(A, dp, dAx, 0, 0, 0);          /* :89 */
    double dn = orc_dot(n, dp, dAx);        /* :91 */
    double alpha = r1 / dn;                 /* :93 */
    axpy(n, x, dp, alpha);                  /* :95 */
    axpy(n, dr, dAx, -1.0 * alpha);         /* :97 */
    jacobi(n, dinv, dr, ds);                /* :100 */
    double r0 = r1;                         /* :107 */
    r1 = orc_dot(n, dr, ds);                /* :109 */
    if (mode == 1) {
      rr = orc_dot(n, dr, dr);
      if (!(sqrt(rr) > tol * sqrt(bb))) break;
    }
    double beta = r1 / r0;                  /* :111 */
    axpby(n, dp, ds, 1.0, beta);            /* :113 */
    k++;
  }
  if (rr_out) *rr_out = (mode == 1) ? rr : orc_dot(n, dr, dr);
  return (k > maxit) ? maxit : k;
}

/* GIP_NonLinearMulticore::getCFL (GIP_NonLinearMulticore.cpp:3-55). */
double orc_cfl(int n, const double* u, const double* v, const double* w, const double* dxs,
               double gamma, double rho) {
  double dt = 1e20;
  double convCoef = 0.25;
  double normit = 0.0;
  for (int i = 0; i < n; i++) {
    double ut = u[i], vt = v[i], wt = w[i], dx = dxs[i];
    if (fabs(ut) > fabs(vt))
      normit = fabs(ut);
    else
      normit = fabs(vt);
    if (normit < fabs(wt)) normit = fabs(wt);
    if (!(dx / normit < 1e-17)) {
      if (dt > convCoef * dx / (normit)) dt = convCoef * dx / (normit);
    }
    if (!(dx * dx * rho / gamma < 1e-17)) {
      if (dt > 0.2 * dx * dx * rho / gamma) dt = 0.2 * dx * dx * rho / gamma;
    }
  }
  double final = dt; /* MPI_Allreduce(MIN) at one rank */
  if (0.8 * final > 1e-1)
    dt = 1e-1;
  else
    dt = 0.8 * final;
  return dt;
}

/* GIP_DNS::integrate and its phases (GIP_DNS.h:99-113, 309-414). */
int orc_dns_run(const orc_ops* ops, const orc_params* prm, orc_state* st, int nsteps,
                double* time_out, double* dt_out, double* massr_out, int* iters_out,
                double* rr_out) {
  const int N = ops->n_inner, NO = ops->n_owned;
  double* dinv = (double*)malloc(sizeof(double) * (size_t)(ops->L.nrows > 0 ? ops->L.nrows : 1));
  double* work = (double*)malloc(sizeof(double) * 4 * (size_t)NO);
  if (!dinv || !work) {
    free(dinv);
    free(work);
    return -1;
  }
  orc_inverse_diagonal(&ops->L, dinv);  /* cg.setUp (GIP_LinearSolver.h:40) */
  orc_csr C = ops->D;                    /* C has D's pattern, values from Ec.mf */
  C.val = st->cval;

  if (!st->started) { /* :102-103 */
    st->dt = orc_cfl(N, st->u, st->v, st->w, st->dxs, prm->gamma, prm->rho);
    st->sigma = 1.0 / st->dt;
    st->started = 1;
  }
  for (int it = 0; it < nsteps; ++it) {
    /* PredictorVelocity :309-338 */
    orc_spmv(&ops->Ec, st->mf, st->cval, 0, 0, 0);
    orc_spmv(&ops->D, st->u, st->ax, 0, 0, 0);
    orc_spmv(&ops->D, st->v, st->ay, 0, 0, 0);
    orc_spmv(&ops->D, st->w, st->az, 0, 0, 0);
    orc_spmv(&C, st->u, st->ax, -1.0, 1.0, 1);
    orc_spmv(&C, st->v, st->ay, -1.0, 1.0, 1);
    orc_spmv(&C, st->w, st->az, -1.0, 1.0, 1);
    double alpha1 = 1.5 * st->dt;
    double alpha2 = -0.5 * st->dt;
    axpy(N, st->u, st->ax, alpha1);
    axpy(N, st->u, st->ax0, alpha2);
    axpy(N, st->v, st->ay, alpha1);
    axpy(N, st->v, st->ay0, alpha2);
    axpy(N, st->w, st->az, alpha1);
    axpy(N, st->w, st->az0, alpha2);
    memcpy(st->ax0, st->ax, sizeof(double) * N);
    memcpy(st->ay0, st->ay, sizeof(double) * N);
    memcpy(st->az0, st->az, sizeof(double) * N);

    /* PoissonEquation :341-354 */
    orc_spmv(&ops->Mx, st->u, st->rhs, 0, 0, 0);
    orc_spmv(&ops->My, st->v, st->rhs, 1.0, 1.0, 1);
    orc_spmv(&ops->Mz, st->w, st->rhs, st->sigma, st->sigma, 1);
    double rr = 0;
    int iters = orc_pcg(&ops->L, dinv, st->rhs, st->p, st->p0, NO, prm->cg_maxit, prm->cg_mode,
                        prm->cg_tol, work, &rr);
    memcpy(st->p0, st->p, sizeof(double) * N);
    memcpy(st->p, st->p0, sizeof(double) * NO);
    orc_spmv(&ops->Lb, st->p0, st->p, 1.0, 1.0, 1);

    /* VelocityCorrection :357-376 */
    orc_spmv(&ops->Gx, st->p, st->gpx, 0, 0, 0);
    orc_spmv(&ops->Gy, st->p, st->gpy, 0, 0, 0);
    orc_spmv(&ops->Gz, st->p, st->gpz, 0, 0, 0);
    double fact = -1.0 / (prm->rho * st->sigma);
    axpy(N, st->u, st->gpx, fact);
    axpy(N, st->v, st->gpy, fact);
    axpy(N, st->w, st->gpz, fact);

    /* MassFluxes :379-391 */
    double fact1 = -1.0 / st->sigma;
    double fact2 = 1.0 / st->sigma;
    orc_spmv(&ops->SO, st->p, st->mf, fact1, 0.0, 1);
    orc_spmv(&ops->SFx, st->gpx, st->mf, fact2, 1.0, 1);
    orc_spmv(&ops->SFy, st->gpy, st->mf, fact2, 1.0, 1);
    orc_spmv(&ops->SFz, st->gpz, st->mf, fact2, 1.0, 1);
    orc_spmv(&ops->SFx, st->u, st->mf, prm->rho, 1.0, 1);
    orc_spmv(&ops->SFy, st->v, st->mf, prm->rho, 1.0, 1);
    orc_spmv(&ops->SFz, st->w, st->mf, prm->rho, 1.0, 1);

    /* CFLCondition :394-414 */
    orc_spmv(&ops->Mres, st->mf, st->temp, 0, 0, 0);
    double massres = orc_norminf(N, st->temp);
    st->time += st->dt;
    if (time_out) time_out[it] = st->time;
    if (dt_out) dt_out[it] = st->dt;
    if (massr_out) massr_out[it] = massres;
    if (iters_out) iters_out[it] = iters;
    if (rr_out) rr_out[it] = rr;
    st->dt = orc_cfl(N, st->u, st->v, st->w, st->dxs, prm->gamma, prm->rho);
    st->sigma = 1.0 / st->dt;
  }
  free(dinv);
  free(work);
  return 0;
}
