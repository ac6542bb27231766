/*
 * ORACLE -- test infrastructure only.  A plain-C restatement of GIP's CPU path for
 * the fractional-step timestep, used by the tests, the smoke check and the CPU leg of
 * the benchmark as the checker.  It is never part of the product library.
 *
 * Pinned against GIP's own goldens: driven through oracle/oracle.py on the C100K
 * operators merged to one rank it prints README.md:73-82 digit for digit, and its
 * fields match GIP's own CPU build (oracle/_ref/gip_ref_cpu) bit for bit at one rank.
 */
#ifndef GIP_ORACLE_H
#define GIP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nrows, ncols, nnz;
  const int* rowptr;
  const int* col;
  const double* val;
} orc_csr;

/* The fifteen operators of GIP_DNS (GIP_DNS.h:27-43) plus the sizes of GIP_Topo. */
typedef struct {
  orc_csr D, Ec, L, Lb, Mx, My, Mz, Mres, Gx, Gy, Gz, SFx, SFy, SFz, SO;
  int n_inner;  /* GIP_Topo::getInnerSize   */
  int n_owned;  /* GIP_Topo::getOwnedSize   */
  int n_faces;  /* faces topology allsize   */
} orc_ops;

/* Every vector GIP_DNS keeps (GIP_DNS.h:47-62); sizes n_owned (cells), n_faces (mf)
 * and D.nnz (cval: the value array of C, which GIP loads from the D file). */
typedef struct {
  double *u, *v, *w, *dxs;
  double *ax, *ay, *az, *ax0, *ay0, *az0;
  double *rhs, *p, *p0, *gpx, *gpy, *gpz, *temp;
  double *mf, *cval;
  double dt, sigma, time;
  int started; /* 0: integrate() has not computed the first dt yet */
} orc_state;

typedef struct {
  double rho, gamma;
  int cg_maxit;     /* GIP: 100 (GIP_DNS.h:183)                                      */
  int cg_mode;      /* 0: exactly cg_maxit iterations (GIP); 1: stop at cg_tol          */
  double cg_tol;    /* mode 1: ||r||_2 <= cg_tol * ||b||_2 (r = recursive residual)    */
} orc_params;

/* y = A x (mode 0) or y = alpha A x + beta y (mode 1); empty rows leave y untouched
 * (GIP_MatrixMulticore.cpp:64-103). */
void orc_spmv(const orc_csr* A, const double* x, double* y, double alpha, double beta, int mode);

/* Jacobi inverse diagonal (GIP_MatrixMulticore::setUpDiagonal, :177-210). Returns the
 * number of rows without a diagonal entry (their dinv is 0). */
int orc_inverse_diagonal(const orc_csr* A, double* dinv);

/* GIP_LinearSolver::solve (GIP_LinearSolver.h:44-117) with x (size n_all) warm-started
 * from x0; work holds 4*n_all doubles.  Returns iterations done; *rr_out = r.r at exit. */
int orc_pcg(const orc_csr* A, const double* dinv, const double* b, double* x, const double* x0,
            int n_all, int maxit, int mode, double tol, double* work, double* rr_out);

double orc_dot(int n, const double* a, const double* b);
double orc_norminf(int n, const double* a);

/* GIP_NonLinearMulticore::getCFL (GIP_NonLinearMulticore.cpp:3-55) at one rank. */
double orc_cfl(int n, const double* u, const double* v, const double* w, const double* dxs,
               double gamma, double rho);

/* GIP_DNS::integrate (GIP_DNS.h:99-113) for nsteps timesteps (continuing from *st).
 * Per step it writes time, dt, massr, CG iterations and the final CG r.r. */
int orc_dns_run(const orc_ops* ops, const orc_params* prm, orc_state* st, int nsteps,
                double* time_out, double* dt_out, double* massr_out, int* iters_out,
                double* rr_out);

#ifdef __cplusplus
}
#endif
#endif
