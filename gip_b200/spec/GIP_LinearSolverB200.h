// Optional faster forms of GIP_LinearSolver<GIP_MatrixB200,GIP_VectorB200>::solve in place of
// GIP's per-operation loop (src/Algorithms/GIP_LinearSolver.h:44-117), which pays seven
// launches and two blocking host round trips per iteration.  Include after
// GIP_LinearSolver.h and B200.h, before the GIP_DNS instantiation, with one of:
//
//  GIPB200_FUSED_PCG  the whole solve as one device-resident PCG (libgipb200
//                     gipb200_pcg_*, FIXED mode = GIP's maxIt iterations);
//  GIPB200_FUSED_OPS  GIP's loop kept on the host, each iteration three fused calls
//                     (gipb200_matrix_spmv_dot, gipb200_cg_update_dot,
//                     gipb200_cg_direction) whose scalars stay on the device, so the host
//                     never waits inside the solve.
//
// Either keeps its device state in the solver's Jacobi-diagonal member (`diagonal`, a
// GIP_MatrixB200): it is built on the first solve after setUp, rebuilt when the operator,
// maxIt or the vector size change, and freed with the solver object.
#ifndef _gip_linearsolver_b200_
#define _gip_linearsolver_b200_

#include "../../Algorithms/GIP_LinearSolver.h"
#include "B200.h"
#include "GIP_B200Check.h"

#if defined(GIPB200_FUSED_PCG) && defined(GIPB200_FUSED_OPS)
#error "choose one of GIPB200_FUSED_PCG and GIPB200_FUSED_OPS"
#endif

#ifdef GIPB200_FUSED_PCG
template <>
inline void GIP_LinearSolver<GIP_MatrixB200, GIP_VectorB200>::solve(GIP_VectorB200* db,
                                                                    GIP_VectorB200* dx,
                                                                    GIP_VectorB200* dx0) {
  GIP_MatrixB200::SolverState& st = diagonal.solver_state();
  const int n_all = myTopo->getAllSize();
  if (!st.pcg || st.op != dA->handle() || st.maxit != maxIt || st.n_all != n_all) {
    diagonal.release_solver_state();
    gipb200_pcg_params p;
    p.mode = GIPB200_PCG_FIXED;
    p.maxit = maxIt;
    p.tol = tol;
    p.inner_tol = 0.0;
    p.inner_maxit = 0;
    p.max_outer = 0;
    p.precond = GIPB200_PRECOND_JACOBI;  // GIP_LinearSolver.h:70-80
    gipb200_require(gipb200_pcg_create(dA->handle(), n_all, &p, &st.pcg), "gipb200_pcg_create");
    st.op = dA->handle();
    st.maxit = maxIt;
    st.n_all = n_all;
  }
  dx0->update();
  gipb200_pcg_result r;
  gipb200_require(gipb200_pcg_solve(st.pcg, db->getDevicePtr(), dx->getDevicePtr(),
                                    dx0->getDevicePtr(), 0, &r),
                  "gipb200_pcg_solve");
}
#endif

#ifdef GIPB200_FUSED_OPS
template <>
inline void GIP_LinearSolver<GIP_MatrixB200, GIP_VectorB200>::solve(GIP_VectorB200* db,
                                                                    GIP_VectorB200* dx,
                                                                    GIP_VectorB200* dx0) {
  GIP_MatrixB200::SolverState& st = diagonal.solver_state();
  const int n = myTopo->getInnerSize(), n_all = myTopo->getAllSize();
  gipb200_matrix A = dA->handle();
  if (!st.work || st.op != A || st.n != n || st.n_all != n_all) {
    diagonal.release_solver_state();
    void* w = 0;
    gipb200_require(gipb200_malloc(&w, sizeof(double) * (4 * (size_t)n_all + n) +
                                           sizeof(gipb200_cg_scalars)),
                    "gipb200_malloc");
    st.work = static_cast<double*>(w);
    st.op = A;
    st.n = n;
    st.n_all = n_all;
    double* dinv = st.work + 4 * (size_t)n_all;
    if (precond) {
      int missing = 0;
      gipb200_require(gipb200_matrix_inverse_diagonal(A, dinv, &missing), "inverse diagonal");
    } else {
      gipb200_require(gipb200_dfill(n, dinv, 1.0, 0), "dfill");  // z = r exactly
    }
  }
  double* dp = st.work;
  double* dAx = dp + n_all;
  double* dr = dAx + n_all;
  double* ds = dr + n_all;
  const double* dinv = ds + n_all;
  gipb200_cg_scalars* sc = reinterpret_cast<gipb200_cg_scalars*>(ds + n_all + n);
  double* x = dx->getDevicePtr();
  const double* x0 = dx0->getDevicePtr();
  // set-up, GIP_LinearSolver.h:54-80
  dx0->update();
  gipb200_require(gipb200_dcopy(n_all, dp, x0, 0), "dcopy");             // dp = x0 (ALL)
  gipb200_require(gipb200_dcopy(n, dr, db->getDevicePtr(), 0), "dcopy"); // dr = b (INNER)
  gipb200_require(gipb200_dcopy(n_all, dAx, x0, 0), "dcopy");            // dAx = x0 (ALL)
  gipb200_require(gipb200_dcopy(n_all, x, x0, 0), "dcopy");              // dx = x0 (ALL)
  gipb200_require(gipb200_matrix_spmv(A, x, dAx, 0.0, 0.0, 0, 0), "spmv");
  gipb200_require(gipb200_daxpy(n, dr, dAx, -1.0, 0), "daxpy");           // dr -= dAx
  if (precond) {  // dp = D dr fused with r1 = dr.dp
    gipb200_require(gipb200_matrix_spmv_dot(diagonal.handle(), dr, dp, n, &sc->rz, 0),
                    "spmv_dot");
  } else {        // dp = dr, r1 = dr.dp (one-time host dot, then to the device scalars)
    gipb200_require(gipb200_dcopy(n, dp, dr, 0), "dcopy");
    double r1 = 0.0;
    gipb200_require(gipb200_ddot(n, dr, dp, &r1, 0), "ddot");
    gipb200_require(gipb200_memcpy_h2d(&sc->rz, &r1, sizeof(double), 0), "h2d");
  }
  // GIP_LinearSolver.h:85-116: three launches per iteration, no host wait.  GIP's
  // dp.update() (:87) is the halo exchange, empty at the single rank this Specification
  // runs on (GIP_VectorB200::update refuses multi-rank topologies).
  for (int k = 1; k <= maxIt; ++k) {
    gipb200_require(gipb200_matrix_spmv_dot(A, dp, dAx, n, &sc->pAp, 0), "spmv_dot");
    gipb200_require(gipb200_cg_update_dot(A, n, x, dr, ds, dp, dAx, dinv, sc, 0),
                    "cg_update_dot");
    gipb200_require(gipb200_cg_direction(n, dp, ds, sc, 0), "cg_direction");
  }
}
#endif
#endif
