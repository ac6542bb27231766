// Optional: GIP_DNS<B200 types>::integrate handed to the fused device engine
// (libgipb200 gipb200_dns_*): the same fractional step as GIP_DNS.h:99-414, with every
// phase fused, dt/sigma/time on the device and each step one CUDA graph.  GIP_DNS's
// setUp still loads the operators and fields through the B200 Specification.  Each
// integrate() builds an engine from GIP_DNS's current state -- the velocities, the AB2
// history ax0/ay0/az0, the face mass fluxes mf, the pressure p and its warm start p0, and
// the simulated time -- so consecutive calls continue exactly like GIP's own integrate()
// (which starts each call with a fresh CFL dt from u, v, w, GIP_DNS.h:102-103).  C's
// values need no upload: every predictor rebuilds them from mf (GIP_DNS.h:311).  The
// engine prints GIP's per-step line and writes every field back into GIP_DNS's vectors.
// Include after GIP_DNS.h and B200.h.
#ifndef _gip_dns_b200_
#define _gip_dns_b200_
#include <mpi.h>

#include <iostream>
#include <vector>

#include "../../Algorithms/GIP_DNS.h"
#include "B200.h"
#include "GIP_B200Check.h"

namespace gipb200_spec {
inline gipb200_host_csr host_csr(GIP_Matrix& m) {
  gipb200_host_csr h;
  h.nrows = m.getNumRows();
  h.nnz = m.getNumNnz();
  int ncols = m.getNumCols();
  const int* c = m.getCsrColIndA();
  for (int k = 0; k < h.nnz; ++k)
    if (c[k] + 1 > ncols) ncols = c[k] + 1;
  h.ncols = ncols;
  h.rowptr = m.getCsrRowIndA();
  h.col = c;
  h.val = m.getCsrValA();
  return h;
}
}  // namespace gipb200_spec

template <>
inline void GIP_DNS<GIP_MatrixB200, GIP_VectorB200, GIP_ArchB200, GIP_NonLinearB200>::integrate() {
  using gipb200_spec::host_csr;
  gipb200_dns_ops ops;
  ops.D = host_csr(D);
  ops.Ec = host_csr(Ec);
  ops.L = host_csr(L);
  ops.Lb = host_csr(Lb);
  ops.Mx = host_csr(Mx);
  ops.My = host_csr(My);
  ops.Mz = host_csr(Mz);
  ops.Mres = host_csr(Mres);
  ops.Gx = host_csr(Gx);
  ops.Gy = host_csr(Gy);
  ops.Gz = host_csr(Gz);
  ops.SFx = host_csr(SFx);
  ops.SFy = host_csr(SFy);
  ops.SFz = host_csr(SFz);
  ops.SO = host_csr(SO);
  ops.n_inner = topoCols.getInnerSize();
  ops.n_owned = topoCols.getOwnedSize();
  ops.n_faces = topoFaces.getAllSize();
  gipb200_dns_params prm;
  prm.rho = rho;
  prm.gamma = gamma;
  prm.pcg.mode = GIPB200_PCG_FIXED;
  prm.pcg.maxit = 100;  // GIP_DNS::uploadPoisson (GIP_DNS.h:180-185)
  prm.pcg.tol = 1e-10;
  prm.pcg.inner_tol = 0.0;
  prm.pcg.inner_maxit = 0;
  prm.pcg.max_outer = 0;
  prm.pcg.precond = GIPB200_PRECOND_JACOBI;
  prm.use_graph = 1;
  prm.reorder = 1;
  gipb200_dns E = 0;
  gipb200_require(gipb200_dns_create(&ops, u.getHostPtr(), v.getHostPtr(), w.getHostPtr(),
                                     dxs.getHostPtr(), &prm, &E),
                  "gipb200_dns_create");
  // the state earlier integrate() calls (or the caller) left in GIP_DNS's members
  struct {
    const char* name;
    GIP_VectorB200* vec;
    int n;
  } state[] = {{"ax0", &ax0, ops.n_owned}, {"ay0", &ay0, ops.n_owned},
               {"az0", &az0, ops.n_owned}, {"p", &p, ops.n_owned},
               {"p0", &p0, ops.n_owned},   {"mf", &mf, ops.n_faces}};
  for (size_t k = 0; k < sizeof(state) / sizeof(state[0]); ++k)
    gipb200_require(gipb200_dns_set_field(E, state[k].name, state[k].vec->getHostPtr(), 0,
                                          state[k].n, 0),
                    "gipb200_dns_set_field");
  gipb200_require(gipb200_dns_set_time(E, time, 0), "gipb200_dns_set_time");
  gipb200_require(gipb200_dns_advance(E, maxIt, 0), "gipb200_dns_advance");
  int steps = 0;
  std::vector<double> t(maxIt > 0 ? maxIt : 1), dtv(t.size()), mr(t.size()), rr(t.size());
  std::vector<int> its(t.size());
  gipb200_require(gipb200_dns_history(E, &steps, t.data(), dtv.data(), mr.data(), its.data(),
                                      rr.data(), 0, 0),
                  "gipb200_dns_history");
  int rank;
  MPI_Comm_rank(MPI_COMM_WORLD, &rank);
  for (it = 0; it < steps; ++it)
    if (rank == 0)
      cout << "time " << t[it] << " [dt::" << dtv[it] << "] massr " << mr[it] << " ite " << it + 1
           << endl;
  double sg = 0.0;
  gipb200_require(gipb200_dns_scalars(E, &dt, &sg, &time), "gipb200_dns_scalars");
  sigma = 1.0 / dt;
  // fields back into GIP_DNS's vectors
  struct {
    const char* name;
    GIP_VectorB200* vec;
  } back[] = {{"u", &u},     {"v", &v},     {"w", &w},     {"p", &p},     {"p0", &p0},
              {"ax", &ax},   {"ay", &ay},   {"az", &az},   {"ax0", &ax0}, {"ay0", &ay0},
              {"az0", &az0}, {"gpx", &gpx}, {"gpy", &gpy}, {"gpz", &gpz}, {"rhs", &rhs},
              {"mf", &mf},   {"temp", &temp}};
  for (size_t k = 0; k < sizeof(back) / sizeof(back[0]); ++k) {
    gipb200_require(gipb200_dns_copy_field(E, back[k].name, back[k].vec->getDevicePtr(),
                                           back[k].vec->getSize(), 0),
                    "gipb200_dns_copy_field");
  }
  // u0 <- u over the inner cells at every step's end (GIP_DNS.h:410-412)
  GIP_VectorB200* now[] = {&u, &v, &w};
  GIP_VectorB200* old_[] = {&u0, &v0, &w0};
  for (int k = 0; k < 3; ++k)
    gipb200_require(gipb200_dcopy(ops.n_inner, old_[k]->getDevicePtr(), now[k]->getDevicePtr(), 0),
                    "gipb200_dcopy");
  gipb200_require(gipb200_stream_sync(0), "sync");
  gipb200_dns_destroy(E);
}
#endif
