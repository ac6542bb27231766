// Standalone fused CG operations for hosts that drive GIP's solver loop themselves.
//
// GIP_LinearSolver::solve (src/Algorithms/GIP_LinearSolver.h:85-116) runs, per iteration,
// an SpMV, two dot products and three vector updates, each a separate pass over the
// vectors, with a blocking host round trip after every dot (GIP's Cuda Specification
// sums the dot's block partials on the host, libgpu.cu:160-203).  These entry points
// fuse that sequence into three kernels whose scalars stay on the device:
//
//   gipb200_matrix_spmv_dot   Ap = A p and p.Ap                  (:89-93)
//   gipb200_cg_update_dot     alpha = r.z / p.Ap; x += alpha p; r -= alpha Ap;
//                             z = dinv r; r.z, r.r; beta          (:95-111)
//   gipb200_cg_direction      p = z + beta p                      (:113)
//
// so a host loop issues three launches per iteration and never waits on the device.
// Every element uses GIP's CPU rounding (no FMA contraction); only the order of the dot
// products' partial sums differs from GIP's sequential loop (a fixed two-level order that
// depends on the launch shape alone).
#include <stdint.h>

#include "device.cuh"
#include "internal.cuh"

namespace gipb200 {
namespace {

struct StoreDot {
  double* out;
  __device__ void operator()(const double* t) const { *out = t[0]; }
};

// y = A x with GIP's row semantics (a row without stored nonzeros keeps y) and
// out = sum_{i < n_dot} x_i y_i over the rows' final values.
__global__ void __launch_bounds__(256, 8) k_spmv_dot(SellView<double> A, const double* __restrict__ x,
                                                     double* __restrict__ y, int n_dot,
                                                     ReduceScratch rs, double* out) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  double acc[1] = {0.0};
  for (int s = gw; s < A.nslices; s += nw) {
    double sum = 0.0;
    bool any = false;
    sell_row_f64(A, x, s, lane, sum, any);
    const int i = s * 32 + lane;
    if (i < A.nrows) {
      const double v = any ? sum : y[i];
      if (any) y[i] = v;
      if (i < n_dot) acc[0] = dadd(acc[0], dmul(x[i], v));
    }
  }
  grid_reduce<SumOp, 1>(acc, rs, StoreDot{out});
}

struct UpdateFinish {
  gipb200_cg_scalars* sc;
  double alpha;
  __device__ void operator()(const double* t) const {
    const double r0 = sc->rz;
    sc->alpha = alpha;
    sc->rz = t[0];
    sc->rr = t[1];
    sc->beta = ddiv(t[0], r0);
  }
};

__device__ __forceinline__ void cg_elem(double& x, double& r, double& z, double p, double q,
                                        double d, double alpha, double malpha, double (&acc)[2]) {
  x = dadd(x, dmul(alpha, p));        // dx->axpy(&dp, alpha)
  r = dadd(r, dmul(malpha, q));       // dr.axpy(&dAx, -1.0*alpha)
  z = dadd(0.0, dmul(r, d));          // diagonal.spmv(&dr, &ds): one-entry rows
  acc[0] = dadd(acc[0], dmul(r, z));  // r1 = dr.dot(&ds)
  acc[1] = dadd(acc[1], dmul(r, r));
}

// V2: two rows per 16-byte access (every pointer 16-byte aligned), same IEEE operations.
template <bool V2>
__global__ void __launch_bounds__(256) k_cg_update(int n, double* __restrict__ x,
                                                   double* __restrict__ r, double* __restrict__ z,
                                                   const double* __restrict__ p,
                                                   const double* __restrict__ q,
                                                   const double* __restrict__ dinv,
                                                   gipb200_cg_scalars* sc, ReduceScratch rs) {
  const double alpha = ddiv(sc->rz, sc->pAp);  // alpha = r1 / dn
  const double malpha = dmul(-1.0, alpha);
  double acc[2] = {0.0, 0.0};
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  int i0 = 0;
  if (V2) {
    const int n2 = n >> 1;
    for (int k = tid; k < n2; k += stride) {
      double2 xv = reinterpret_cast<double2*>(x)[k], rv = reinterpret_cast<double2*>(r)[k];
      const double2 pv = reinterpret_cast<const double2*>(p)[k];
      const double2 qv = reinterpret_cast<const double2*>(q)[k];
      const double2 dv = reinterpret_cast<const double2*>(dinv)[k];
      double2 zv;
      cg_elem(xv.x, rv.x, zv.x, pv.x, qv.x, dv.x, alpha, malpha, acc);
      cg_elem(xv.y, rv.y, zv.y, pv.y, qv.y, dv.y, alpha, malpha, acc);
      reinterpret_cast<double2*>(x)[k] = xv;
      reinterpret_cast<double2*>(r)[k] = rv;
      reinterpret_cast<double2*>(z)[k] = zv;
    }
    i0 = 2 * n2;
  }
  for (int i = i0 + tid; i < n; i += stride) {
    double xi = x[i], ri = r[i], zi;
    cg_elem(xi, ri, zi, p[i], q[i], dinv[i], alpha, malpha, acc);
    x[i] = xi;
    r[i] = ri;
    z[i] = zi;
  }
  grid_reduce<SumOp, 2>(acc, rs, UpdateFinish{sc, alpha});
}

// p = 1.0 z + beta p   (dp.axpy(&ds, 1.0, beta))
template <bool V2>
__global__ void __launch_bounds__(256) k_cg_direction(int n, double* __restrict__ p,
                                                      const double* __restrict__ z,
                                                      const gipb200_cg_scalars* sc) {
  const double beta = sc->beta;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  int i0 = 0;
  if (V2) {
    const int n2 = n >> 1;
    for (int k = tid; k < n2; k += stride) {
      double2 pv = reinterpret_cast<double2*>(p)[k];
      const double2 zv = reinterpret_cast<const double2*>(z)[k];
      pv.x = dadd(dmul(1.0, zv.x), dmul(beta, pv.x));
      pv.y = dadd(dmul(1.0, zv.y), dmul(beta, pv.y));
      reinterpret_cast<double2*>(p)[k] = pv;
    }
    i0 = 2 * n2;
  }
  for (int i = i0 + tid; i < n; i += stride) p[i] = dadd(dmul(1.0, z[i]), dmul(beta, p[i]));
}

bool aligned16(const void* a) { return (reinterpret_cast<uintptr_t>(a) & 15u) == 0; }

}  // namespace
}  // namespace gipb200

using namespace gipb200;

extern "C" {

int gipb200_matrix_spmv_dot(gipb200_matrix A, const double* d_x, double* d_y, int n_dot,
                            double* d_dot, void* stream) {
  if (!A || !d_x || !d_y || !d_dot) return fail(GIPB200_ERR_ARG, "spmv_dot: null argument");
  if (n_dot < 0 || n_dot > A->S.nrows)
    return fail(GIPB200_ERR_ARG, "spmv_dot: n_dot=%d outside [0, rows=%d]", n_dot, A->S.nrows);
  if (d_x == d_y) return fail(GIPB200_ERR_ARG, "spmv_dot: x and y must not alias");
  cudaStream_t s = as_stream(stream);
  int blocks = 1;
  GIPB_TRY(grid_blocks(256, std::max(A->S.nslices, 1) * 32, 1, kMaxReduceBlocks, &blocks));
  k_spmv_dot<<<blocks, 256, 0, s>>>(A->S.view(), d_x, d_y, n_dot, A->rs, d_dot);
  GIPB_LAUNCH_CHECK();
  return GIPB200_OK;
}

int gipb200_cg_update_dot(gipb200_matrix A, int n, double* d_x, double* d_r, double* d_z,
                          const double* d_p, const double* d_q, const double* d_dinv,
                          gipb200_cg_scalars* d_sc, void* stream) {
  if (!A || !d_x || !d_r || !d_z || !d_p || !d_q || !d_dinv || !d_sc)
    return fail(GIPB200_ERR_ARG, "cg_update_dot: null argument");
  if (n < 0 || n > A->S.nrows)
    return fail(GIPB200_ERR_ARG, "cg_update_dot: n=%d outside [0, rows=%d]", n, A->S.nrows);
  cudaStream_t s = as_stream(stream);
  int blocks = 1;
  GIPB_TRY(grid_blocks(256, std::max(n, 1), 4, kMaxReduceBlocks, &blocks));
  const bool v2 = aligned16(d_x) && aligned16(d_r) && aligned16(d_z) && aligned16(d_p) &&
                  aligned16(d_q) && aligned16(d_dinv);
  if (v2)
    k_cg_update<true><<<blocks, 256, 0, s>>>(n, d_x, d_r, d_z, d_p, d_q, d_dinv, d_sc, A->rs);
  else
    k_cg_update<false><<<blocks, 256, 0, s>>>(n, d_x, d_r, d_z, d_p, d_q, d_dinv, d_sc, A->rs);
  GIPB_LAUNCH_CHECK();
  return GIPB200_OK;
}

int gipb200_cg_direction(int n, double* d_p, const double* d_z, const gipb200_cg_scalars* d_sc,
                         void* stream) {
  if (n < 0 || (n > 0 && (!d_p || !d_z || !d_sc)))
    return fail(GIPB200_ERR_ARG, "cg_direction: bad size or null argument");
  if (n == 0) return GIPB200_OK;
  cudaStream_t s = as_stream(stream);
  int blocks = 1;
  GIPB_TRY(grid_blocks(256, n, 4, 0, &blocks));
  if (aligned16(d_p) && aligned16(d_z))
    k_cg_direction<true><<<blocks, 256, 0, s>>>(n, d_p, d_z, d_sc);
  else
    k_cg_direction<false><<<blocks, 256, 0, s>>>(n, d_p, d_z, d_sc);
  GIPB_LAUNCH_CHECK();
  return GIPB200_OK;
}

}  // extern "C"
