// Optional: GIP_LinearSolver<GIP_MatrixB200,GIP_VectorB200>::solve as one device-resident
// PCG (libgipb200 gipb200_pcg_*, FIXED mode = GIP's maxIt iterations) instead of GIP's
// per-operation loop (src/Algorithms/GIP_LinearSolver.h:44-117) with its two host
// round trips per iteration.  Include after GIP_LinearSolver.h and B200.h, before the
// GIP_DNS instantiation (DrivenCavity.cpp includes it beside B200.h).
#ifndef _gip_linearsolver_b200_
#define _gip_linearsolver_b200_
#include <map>

#include "../../Algorithms/GIP_LinearSolver.h"
#include "B200.h"
#include "GIP_B200Check.h"

template <>
inline void GIP_LinearSolver<GIP_MatrixB200, GIP_VectorB200>::solve(GIP_VectorB200* db,
                                                                    GIP_VectorB200* dx,
                                                                    GIP_VectorB200* dx0) {
  static std::map<const void*, gipb200_pcg> solvers;
  gipb200_pcg& S = solvers[this];
  if (!S) {
    gipb200_pcg_params p;
    p.mode = GIPB200_PCG_FIXED;
    p.maxit = maxIt;
    p.tol = tol;
    p.inner_tol = 0.0;
    p.inner_maxit = 0;
    p.max_outer = 0;
    p.precond = GIPB200_PRECOND_JACOBI;  // GIP_LinearSolver.h:70-80
    gipb200_require(gipb200_pcg_create(dA->handle(), myTopo->getAllSize(), &p, &S),
                    "gipb200_pcg_create");
  }
  dx0->update();
  gipb200_pcg_result r;
  gipb200_require(gipb200_pcg_solve(S, db->getDevicePtr(), dx->getDevicePtr(),
                                    dx0->getDevicePtr(), 0, &r),
                  "gipb200_pcg_solve");
}
#endif
