// Jacobi-PCG on the device.
//
// FP64 modes restate GIP_LinearSolver::solve (src/Algorithms/GIP_LinearSolver.h:44-117)
// with three kernels per iteration and every scalar kept on the device:
//   A: Ap = L p fused with p.Ap                      -> alpha = r.z / p.Ap
//   B: x += alpha p, r -= alpha Ap, z = dinv r, r.z, r.r  -> beta, stop test
//   C: p = z + beta p   (z recomputed from r, bit-identical to B's)
// The products and sums of every vector element use GIP's IEEE operations, so only the
// order of the two dot products differs from the CPU build.
//
// MIXED runs FP64 iterative refinement: r = b - L x in FP64 (sliced FP64 operator), then
// an FP32 CG on the Jacobi-scaled system (S L S) y = S r with S = diag(1/sqrt(L_ii)),
// which is Jacobi-PCG in exact arithmetic but needs no dinv stream, then x += S y.
//
// GIP's pressure operator is a pure-Neumann Laplacian L_N made definite by one weak pin,
// L = L_N + pin e_p e_p^T (GIP pins 1/101 of the diagonal).  Its smallest eigenvalue
// ~ 1/(101 N) times FP32 rounding makes a plain FP32 CG blow up along the constant mode.
// With that structure detected, the correction d of L d = r is split exactly:
//   summing the rows gives pin d_p = sum(r)            (1^T L_N = 0),
//   L_N d = r - e_p sum(r)                              (consistent, singular),
// so the FP32 CG runs on S L_N S with the pinned residual entry adjusted, and the
// constant is fixed afterwards: d = S y + (sum(r)/pin - s_p y_p) 1.
#include <math.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "device.cuh"
#include "pcg.cuh"

namespace gipb200 {

// ------------------------------------------------------------------ FP64 kernels
// A while-node condition is set by the kernel that decides it: value = keep looping.
__device__ __forceinline__ void set_loop(int use, cudaGraphConditionalHandle h, int keep) {
  if (use) cudaGraphSetConditional(h, keep ? 1u : 0u);
}

// Start of every FP32 loop kernel: count the launch; the SpMV, first kernel of an
// iteration, also sets the loop's graph condition from the stop flag.
__device__ __forceinline__ void mx_enter(PcgScalars* S, int use_cond,
                                         cudaGraphConditionalHandle loop_cond) {
  dep_begin();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    atomicAdd(&S->kernels, 1);
    set_loop(use_cond, loop_cond, !S->done);
  }
}


struct PcgInitFinish {
  PcgScalars* S;
  int mode, maxit;
  double tol;
  int use_cond;
  cudaGraphConditionalHandle cond;
  __device__ void operator()(const double* t) const {
    S->rz = t[0];
    S->rr = t[1];
    S->bb = t[2];
    S->iter = 0;
    S->status = GIPB200_OK;
    S->done = (maxit <= 0) ? 1 : 0;
    if (mode == GIPB200_PCG_TOL && !(sqrt(t[1]) > tol * sqrt(t[2]))) S->done = 1;
    if (mode != GIPB200_PCG_FIXED && !(isfinite(t[1]) && isfinite(t[2]))) {
      S->status = GIPB200_ERR_BREAKDOWN;  // a non-finite right-hand side or start
      S->done = 1;
    }
    set_loop(use_cond, cond, !S->done);
  }
};

// r = b - L x;  z = dinv r;  p = z;  (rz, rr, bb)   -- GIP_LinearSolver.h:63-80
__global__ void __launch_bounds__(256, 8) k_pcg_init(SellView<double> L, const double* __restrict__ x,
                                                  const double* __restrict__ b,
                                                  const double* __restrict__ dinv,
                                                  double* __restrict__ r, double* __restrict__ p,
                                                  double* __restrict__ Ap, PcgScalars* S,
                                                  ReduceScratch rs, int mode, int maxit,
                                                  double tol, int use_cond,
                                                  cudaGraphConditionalHandle cond) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int s = gw; s < L.nslices; s += nw) {
    double sum = 0.0;
    bool any = false;
    sell_row_f64(L, x, s, lane, sum, any);
    const int i = s * 32 + lane;
    if (i < L.nrows) {
      const double ax = any ? sum : Ap[i];   // dAx starts as a copy of x0 (:66)
      Ap[i] = ax;
      const double bi = b[i];
      const double ri = dadd(bi, dmul(-1.0, ax));
      const double zi = dadd(0.0, dmul(ri, dinv[i]));
      r[i] = ri;
      p[i] = zi;
      acc[0] = dadd(acc[0], dmul(ri, zi));
      acc[1] = dadd(acc[1], dmul(ri, ri));
      acc[2] = dadd(acc[2], dmul(bi, bi));
    }
  }
  grid_reduce<SumOp, 3>(acc, rs, PcgInitFinish{S, mode, maxit, tol, use_cond, cond});
}

struct AlphaFinish {
  PcgScalars* S;
  int mode;
  __device__ void operator()(const double* t) const {
    S->pAp = t[0];
    S->alpha = ddiv(S->rz, t[0]);
    if (mode != GIPB200_PCG_FIXED && (!(t[0] > 0.0) || !isfinite(S->alpha))) {
      S->status = GIPB200_ERR_BREAKDOWN;
      S->done = 1;
    }
  }
};

// Ap = L p ; p.Ap  -- GIP_LinearSolver.h:89-93
__global__ void __launch_bounds__(256, 8) k_pcg_spmv_dot(SellView<double> L,
                                                      const double* __restrict__ p,
                                                      double* __restrict__ Ap, PcgScalars* S,
                                                      ReduceScratch rs, int mode) {
  if (S->done) return;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  double acc[1] = {0.0};
  // slot range of the slice after next, loaded one iteration ahead of its L2 prefetch
  long long n0 = -1, n1 = -1;
  if (gw + nw < L.nslices) n0 = __ldg(L.sptr + gw + nw), n1 = __ldg(L.sptr + gw + nw + 1);
  for (int s = gw; s < L.nslices; s += nw) {
    if (lane == 0 && n0 >= 0 && n1 > n0) {  // this warp's next slice streams into L2
      prefetch_l2(L.col + n0, (unsigned)(n1 - n0) * 4u);
      prefetch_l2(L.val + n0, (unsigned)(n1 - n0) * 8u);
    }
    const int s2 = s + 2 * nw;
    n0 = -1;
    if (s2 < L.nslices) n0 = __ldg(L.sptr + s2), n1 = __ldg(L.sptr + s2 + 1);
    double sum = 0.0;
    bool any = false;
    sell_row_f64(L, p, s, lane, sum, any);
    const int i = s * 32 + lane;
    if (i < L.nrows) {
      const double v = any ? sum : Ap[i];
      if (any) Ap[i] = v;
      acc[0] = dadd(acc[0], dmul(p[i], v));
    }
  }
  grid_reduce<SumOp, 1>(acc, rs, AlphaFinish{S, mode});
}

struct BetaFinish {
  PcgScalars* S;
  int mode, maxit;
  double tol;
  __device__ void operator()(const double* t) const {
    const double r0 = S->rz;
    S->rz = t[0];
    S->rr = t[1];
    S->beta = ddiv(t[0], r0);
    S->iter += 1;
    if (mode == GIPB200_PCG_TOL && !(sqrt(t[1]) > tol * sqrt(S->bb))) S->done = 1;
    if (S->iter >= maxit) {
      if (mode == GIPB200_PCG_TOL && !S->done) S->status = GIPB200_ERR_NOT_CONVERGED;
      S->done = 1;
    }
  }
};

// x += alpha p; r -= alpha Ap; z = dinv r; r.z, r.r  -- GIP_LinearSolver.h:95-111
// x += alpha p; r -= alpha Ap; z = dinv r; r.z, r.r  -- GIP_LinearSolver.h:95-111.
// V2: two rows per access (16-byte loads and stores; x must be 16-byte aligned), the
// same IEEE operations per element.
template <bool V2>
__global__ void __launch_bounds__(256) k_pcg_update(int n, double* __restrict__ x,
                                                    double* __restrict__ r,
                                                    const double* __restrict__ p,
                                                    const double* __restrict__ Ap,
                                                    const double* __restrict__ dinv,
                                                    PcgScalars* S, ReduceScratch rs, int mode,
                                                    int maxit, double tol) {
  if (S->done) return;
  const double alpha = S->alpha;
  const double malpha = dmul(-1.0, alpha);
  double acc[2] = {0.0, 0.0};
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  int i0 = 0;
  if (V2) {
    const int n2 = n >> 1;
    double2* x2 = reinterpret_cast<double2*>(x);
    double2* r2 = reinterpret_cast<double2*>(r);
    const double2* p2 = reinterpret_cast<const double2*>(p);
    const double2* a2 = reinterpret_cast<const double2*>(Ap);
    const double2* d2 = reinterpret_cast<const double2*>(dinv);
    for (int q = tid; q < n2; q += stride) {
      double2 xv = x2[q], rv = r2[q];
      const double2 pv = p2[q], av = a2[q], dv = d2[q];
      xv.x = dadd(xv.x, dmul(alpha, pv.x));
      xv.y = dadd(xv.y, dmul(alpha, pv.y));
      rv.x = dadd(rv.x, dmul(malpha, av.x));
      rv.y = dadd(rv.y, dmul(malpha, av.y));
      x2[q] = xv;
      r2[q] = rv;
      const double zx = dadd(0.0, dmul(rv.x, dv.x)), zy = dadd(0.0, dmul(rv.y, dv.y));
      acc[0] = dadd(acc[0], dmul(rv.x, zx));
      acc[1] = dadd(acc[1], dmul(rv.x, rv.x));
      acc[0] = dadd(acc[0], dmul(rv.y, zy));
      acc[1] = dadd(acc[1], dmul(rv.y, rv.y));
    }
    i0 = 2 * n2;
  }
  for (int i = i0 + tid; i < n; i += stride) {
    x[i] = dadd(x[i], dmul(alpha, p[i]));
    const double ri = dadd(r[i], dmul(malpha, Ap[i]));
    r[i] = ri;
    const double zi = dadd(0.0, dmul(ri, dinv[i]));
    acc[0] = dadd(acc[0], dmul(ri, zi));
    acc[1] = dadd(acc[1], dmul(ri, ri));
  }
  grid_reduce<SumOp, 2>(acc, rs, BetaFinish{S, mode, maxit, tol});
}

// p = 1.0 z + beta p  -- GIP_LinearSolver.h:113
// ---- FP64 tolerance mode with the AMG preconditioner: the update keeps GIP's x and r
// steps and tests r.r; z = M r, r.z and beta come from the V-cycle; then p = z + beta p.
struct BetaFinishAmg {
  PcgScalars* S;
  int maxit;
  double tol;
  __device__ void operator()(const double* t) const {
    S->rr = t[0];
    S->iter += 1;
    if (!isfinite(t[0])) {
      S->status = GIPB200_ERR_BREAKDOWN;
      S->done = 1;
    } else if (!(sqrt(t[0]) > tol * sqrt(S->bb))) {
      S->done = 1;
    }
    if (S->iter >= maxit) {
      if (!S->done) S->status = GIPB200_ERR_NOT_CONVERGED;
      S->done = 1;
    }
  }
};

__global__ void __launch_bounds__(256) k_pcg_update_amg(int n, double* __restrict__ x,
                                                        double* __restrict__ r,
                                                        const double* __restrict__ p,
                                                        const double* __restrict__ Ap,
                                                        PcgScalars* S, ReduceScratch rs, int maxit,
                                                        double tol) {
  if (S->done) return;
  const double alpha = S->alpha;
  const double malpha = dmul(-1.0, alpha);
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = dadd(x[i], dmul(alpha, p[i]));
    const double ri = dadd(r[i], dmul(malpha, Ap[i]));
    r[i] = ri;
    acc[0] = dadd(acc[0], dmul(ri, ri));
  }
  grid_reduce<SumOp, 1>(acc, rs, BetaFinishAmg{S, maxit, tol});
}

// p = z + beta p; counted on the device with the V-cycle's kernels
__global__ void __launch_bounds__(256) k_pcg_pupdate_z(int n, double* __restrict__ p,
                                                       const double* __restrict__ z,
                                                       PcgScalars* S, int use_cond,
                                                       cudaGraphConditionalHandle cond) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    atomicAdd(&S->kernels, 1);
    set_loop(use_cond, cond, !S->done);
  }
  if (S->done) return;
  const double beta = S->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = dadd(z[i], dmul(beta, p[i]));
}

__global__ void __launch_bounds__(256) k_pcg_pupdate(int n, double* __restrict__ p,
                                                     const double* __restrict__ r,
                                                     const double* __restrict__ dinv,
                                                     const PcgScalars* S, int use_cond,
                                                     cudaGraphConditionalHandle cond) {
  if (blockIdx.x == 0 && threadIdx.x == 0) set_loop(use_cond, cond, !S->done);
  if (S->done) return;
  const double beta = S->beta;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  const int n2 = n >> 1;  // p, r and dinv are the solver's own (aligned) buffers
  double2* p2 = reinterpret_cast<double2*>(p);
  const double2* r2 = reinterpret_cast<const double2*>(r);
  const double2* d2 = reinterpret_cast<const double2*>(dinv);
  for (int q = tid; q < n2; q += stride) {
    double2 pv = p2[q];
    const double2 rv = r2[q], dv = d2[q];
    const double zx = dadd(0.0, dmul(rv.x, dv.x)), zy = dadd(0.0, dmul(rv.y, dv.y));
    pv.x = dadd(dmul(1.0, zx), dmul(beta, pv.x));
    pv.y = dadd(dmul(1.0, zy), dmul(beta, pv.y));
    p2[q] = pv;
  }
  for (int i = 2 * n2 + tid; i < n; i += stride) {
    const double zi = dadd(0.0, dmul(r[i], dinv[i]));
    p[i] = dadd(dmul(1.0, zi), dmul(beta, p[i]));
  }
}

// ------------------------------------------------------------------ MIXED kernels
// Reliable-update mixed CG.  The FP32 CG runs on the scaled operator A^ = S L S (pin
// removed when L is pinned-Neumann) with its search direction kept for the whole solve;
// the FP64 true residual r = b - L x replaces the FP32 one ("reliable update") whenever
// the FP32 residual has fallen by the factor delta since the last replacement or
// predicts convergence.  x accumulates in FP64: x += S y + kappa at each replacement.

struct ResidualFinish {
  PcgScalars* S;
  int first;
  double tol, delta;
  int maxit, max_updates;
  int pin_row;
  double pin_val;
  const double* scale;
  float* r32;
  float* p32;
  int use_cond;
  cudaGraphConditionalHandle loop_cond;
  int amg;  // beta and r.z come from the preconditioner's last kernel instead
  __device__ void operator()(const double* t) const {
    // t[0] = r.r (FP64 true residual), t[1] = r^.r^ before the pin projection,
    // t[2] = b.b, t[3] = sum(r)
    if (first) S->bb = t[2];
    S->rr = t[0];
    double rz = t[1];
    S->kappa_c = 0.0;
    if (pin_row >= 0) {
      const float old = __ldcg(r32 + pin_row);
      const float nw = (float)((double)old - scale[pin_row] * t[3]);
      r32[pin_row] = nw;
      if (first) p32[pin_row] = nw;
      rz = rz - (double)old * (double)old + (double)nw * (double)nw;
      S->kappa_c = t[3] / pin_val;
    }
    if (!first) {
      if (!amg) S->beta = rz / S->rz;  // continue the direction with the replaced residual
      S->outer += 1;
    }
    if (!amg) S->rz = rz;
    S->maxr2 = rz;
    // FP32 level at which the predicted true residual reaches tol*||b|| / 2
    const double goal = 0.5 * tol * sqrt(S->bb);
    S->trig = (t[0] > 0.0) ? rz * (goal * goal) / t[0] : 0.0;
    S->upd = 0;
    const bool finite = isfinite(t[0]) && isfinite(S->bb);
    const bool conv = finite && !(sqrt(t[0]) > tol * sqrt(S->bb));
    if (conv || !finite || S->total_inner >= maxit || S->outer >= max_updates) {
      if (!conv) S->status = finite ? GIPB200_ERR_NOT_CONVERGED : GIPB200_ERR_BREAKDOWN;
      S->done = 1;
    }
    (void)delta;
    if (first) set_loop(use_cond, loop_cond, !S->done);
  }
};

// r = b - L x (FP64); r^ = S r (FP32); first call: p = r^, y = 0.  Later calls run only
// when a replacement is due (S->upd).
__global__ void __launch_bounds__(256) k_mx_residual(SellView<double> L, const double* __restrict__ x,
                                                     const double* __restrict__ b,
                                                     const double* __restrict__ scale,
                                                     float* __restrict__ r32, float* __restrict__ p32,
                                                     float* __restrict__ y32, PcgScalars* S,
                                                     ReduceScratch rs, int first, double tol,
                                                     double delta, int maxit, int max_updates,
                                                     int pin_row, double pin_val, int use_cond,
                                                     cudaGraphConditionalHandle loop_cond, int amg) {
  mx_enter(S, 0, 0);
  if (!first && (!S->upd || S->done)) return;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int s = gw; s < L.nslices; s += nw) {
    double sum = 0.0;
    bool any = false;
    sell_row_f64(L, x, s, lane, sum, any);
    const int i = s * 32 + lane;
    if (i < L.nrows) {
      const double bi = b[i];
      const double ri = bi - sum;
      const float rh = (float)(ri * scale[i]);
      r32[i] = rh;
      if (first) {
        p32[i] = rh;
        y32[i] = 0.f;
      }
      acc[0] += ri * ri;
      acc[1] += (double)rh * (double)rh;
      acc[2] += bi * bi;
      acc[3] += ri;
    }
  }
  grid_reduce<SumOp, 4>(acc, rs,
                        ResidualFinish{S, first, tol, delta, maxit, max_updates, pin_row, pin_val,
                                       scale, r32, p32, use_cond, loop_cond, amg});
}

// The same residual from the packed operator's columns with L's FP64 values from a 4-bit
// table (each row's inner entries in column order) against b' = b - L_ghost x_ghost,
// which the solve forms once (x's ghost entries do not change during a solve); slices
// stored plain use L's own row against b.  Streams 24 instead of ~100 bytes per row.
__global__ void __launch_bounds__(256, 8) k_mx_residual_packed(
    SellView<double> L, const uint4* __restrict__ delta, const int* __restrict__ base,
    const unsigned char* __restrict__ plain, const unsigned* __restrict__ lidx,
    const double* __restrict__ ltable, const double* __restrict__ bp,
    const double* __restrict__ x, const double* __restrict__ b,
    const double* __restrict__ scale, float* __restrict__ r32, float* __restrict__ p32,
    float* __restrict__ y32, PcgScalars* S, ReduceScratch rs, int first, double tol,
    double delta_f, int maxit, int max_updates, int pin_row, double pin_val, int use_cond,
    cudaGraphConditionalHandle loop_cond, int amg) {
  mx_enter(S, 0, 0);
  if (!first && (!S->upd || S->done)) return;
  __shared__ double tab[16];
  if (threadIdx.x < 16) tab[threadIdx.x] = ltable[threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int s = gw; s < L.nslices; s += nw) {
    const int i = s * 32 + lane;
    const int pl = __ldg(plain + s);
    const uint4 d = ld_stream(delta + i);
    const unsigned w = ld_stream(lidx + i);
    int c[8];
    packed_cols(base, s, d, c);
    double sum = 0.0;
    if (pl) {
      bool any = false;
      sell_row_f64(L, x, s, lane, sum, any);
    } else {
      double xv[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) xv[j] = __ldg(x + c[j]);
#pragma unroll
      for (int j = 0; j < 8; ++j) sum = dadd(sum, dmul(xv[j], tab[(w >> (4 * j)) & 15u]));
    }
    if (i < L.nrows) {
      const double bi = b[i];
      const double ri = (pl ? bi : bp[i]) - sum;
      const float rh = (float)(ri * scale[i]);
      r32[i] = rh;
      if (first) {
        p32[i] = rh;
        y32[i] = 0.f;
      }
      acc[0] += ri * ri;
      acc[1] += (double)rh * (double)rh;
      acc[2] += bi * bi;
      acc[3] += ri;
    }
  }
  grid_reduce<SumOp, 4>(acc, rs,
                        ResidualFinish{S, first, tol, delta_f, maxit, max_updates, pin_row,
                                       pin_val, scale, r32, p32, use_cond, loop_cond, amg});
}

// b' = b - L_ghost x for the rows with ghost columns (b' = b elsewhere, copied before)
__global__ void k_mx_ghost_rhs(int ng, const int* __restrict__ rows, const int* __restrict__ rp,
                               const int* __restrict__ col, const double* __restrict__ val,
                               const double* __restrict__ x, const double* __restrict__ b,
                               double* __restrict__ bp) {
  dep_begin();
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
    double sum = 0.0;
    for (int k = rp[g]; k < rp[g + 1]; ++k) sum = dadd(sum, dmul(x[col[k]], val[k]));
    const int i = rows[g];
    bp[i] = b[i] - sum;
  }
}

struct AlphaFinish32 {
  PcgScalars* S;
  __device__ void operator()(const double* t) const {
    S->pAp = t[0];
    S->alpha = S->rz / t[0];
    if (!(t[0] > 0.0) || !isfinite(S->alpha)) {  // FP32 direction lost: force a replacement
      S->alpha = 0.0;
    }
  }
};

// One row of the plain FP32 layout, the gathered vector being the new search direction
// p = r + beta p_in formed on the fly (the same FMA as a separate update would do, so
// the same values), summed slot by slot.
template <int CH>
__device__ __forceinline__ float sell_row_dir(const SellView<float>& A, const float* __restrict__ r,
                                              const float* __restrict__ pin, float beta, int s,
                                              int lane) {
  long long base;
  int len;
  slice_range(A, s, base, len);
  const int* cp = A.col + base + lane;
  const float* vp = A.val + base + lane;
  float sum = 0.f;
  for (int j0 = 0; j0 < len; j0 += CH) {
    int c[CH];
    float v[CH];
#pragma unroll
    for (int t = 0; t < CH; ++t) {
      if (j0 + t < len) {
        c[t] = ld_stream(cp + (size_t)(j0 + t) * 32);
        v[t] = ld_stream(vp + (size_t)(j0 + t) * 32);
      } else {
        c[t] = -1;
        v[t] = 0.f;
      }
    }
    float xv[CH];
#pragma unroll
    for (int t = 0; t < CH; ++t)
      xv[t] = (c[t] >= 0) ? fmaf(beta, __ldg(pin + c[t]), __ldg(r + c[t])) : 0.f;
#pragma unroll
    for (int t = 0; t < CH; ++t) sum = fmaf(xv[t], v[t], sum);
  }
  return sum;
}

// Ap = Â p and p.Ap with p = r + beta p_in (the direction update of GIP_LinearSolver.h:
// 113-115 folded into the product): rows write p_out, gathers form p from r and p_in.
// REC (the AMG path, where beta is small): the product of the new direction comes from the
// recurrence A p = A z + beta A p_in, so the rows gather z alone (one gather per nonzero
// instead of two) and read their own previous product Apin; rounding errors of the
// recurrence are damped by beta every iteration.  beta = 0 (the first iteration of a
// solve, or a restart) takes A z alone and reads no previous product.
template <bool REC>
__global__ void __launch_bounds__(256, 8) k_mx_spmv_dot(SellView<float> A, const float* __restrict__ r,
                                                     const float* __restrict__ pin,
                                                     float* __restrict__ pout,
                                                     float* __restrict__ Ap, PcgScalars* S,
                                                     ReduceScratch rs, int use_cond,
                                                     cudaGraphConditionalHandle loop_cond,
                                                     const float* __restrict__ Apin) {
  mx_enter(S, use_cond, loop_cond);
  if (S->done) return;
  const float beta = (float)S->beta;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  double acc[1] = {0.0};
  // slot range of the slice after next, loaded one iteration ahead of its L2 prefetch
  long long n0 = -1, n1 = -1;
  if (gw + nw < A.nslices) n0 = __ldg(A.sptr + gw + nw), n1 = __ldg(A.sptr + gw + nw + 1);
  for (int s = gw; s < A.nslices; s += nw) {
    if (lane == 0 && n0 >= 0 && n1 > n0) {  // this warp's next slice streams into L2
      prefetch_l2(A.col + n0, (unsigned)(n1 - n0) * 4u);
      prefetch_l2(A.val + n0, (unsigned)(n1 - n0) * 4u);
    }
    const int s2 = s + 2 * nw;
    n0 = -1;
    if (s2 < A.nslices) n0 = __ldg(A.sptr + s2), n1 = __ldg(A.sptr + s2 + 1);
    const float sum = REC ? sell_row_f32<2>(A, r, s, lane) : sell_row_dir<4>(A, r, pin, beta, s, lane);
    const int i = s * 32 + lane;
    if (i < A.nrows) {
      const float pi = fmaf(beta, pin[i], r[i]);
      const float api = (REC && beta != 0.f) ? fmaf(beta, Apin[i], sum) : sum;
      pout[i] = pi;
      Ap[i] = api;
      acc[0] += (double)pi * (double)api;
    }
  }
  grid_reduce<SumOp, 1>(acc, rs, AlphaFinish32{S});
}

// Same product as k_mx_spmv_dot from the packed layout: the same FMA order slot by slot.
// Every slot gathers (padding and stored zeros point at a valid column through delta 0
// and multiply by table entry 0 = 0.0f, adding zero where the plain kernel adds x*0), so
// the loop has no branches.  A warp owns a slice; in a packed slice each lane loads its
// row's 16-byte delta word and its index word, then issues K independent pairs of
// gathers (r and p_in).  K = 7 when no packed row has an eighth slot.
template <int NIB, int K, bool REC>
__global__ void __launch_bounds__(256, 8) k_mxp_spmv_dot(SellView<float> A,
                                                         const uint4* __restrict__ delta,
                                                         const void* __restrict__ idx,
                                                         const int* __restrict__ base,
                                                         const unsigned char* __restrict__ plain,
                                                         const float* __restrict__ table,
                                                         const float* __restrict__ r,
                                                         const float* __restrict__ pin,
                                                         float* __restrict__ pout,
                                                         float* __restrict__ Ap, PcgScalars* S,
                                                         ReduceScratch rs, int use_cond,
                                                         cudaGraphConditionalHandle loop_cond,
                                                         const float* __restrict__ Apin) {
  mx_enter(S, use_cond, loop_cond);
  if (S->done) return;
  constexpr int NT = 1 << NIB;
  __shared__ float tab[NT];
  for (int t = threadIdx.x; t < NT; t += blockDim.x) tab[t] = table[t];
  __syncthreads();
  const float beta = (float)S->beta;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  double acc[1] = {0.0};
  PackedWords cur;
  for (int s = gw; s < A.nslices; s += nw) {
    // (the slot bases after the plain test: hoisted with the words, as the V-cycle's
    // packed kernel has them, this kernel measured 150 against 138 us)
    packed_words<NIB>(delta, idx, plain, s, lane, cur);
    const int i = s * 32 + lane;
    float sum;
    if (cur.plain) {  // rare fallback: few registers
      sum = REC ? sell_row_f32<2>(A, r, s, lane) : sell_row_dir<2>(A, r, pin, beta, s, lane);
    } else {
      int c[8];
      packed_cols(base, s, cur.d, c);
      float xv[K];
#pragma unroll
      for (int j = 0; j < K; ++j)
        xv[j] = REC ? __ldg(r + c[j]) : fmaf(beta, __ldg(pin + c[j]), __ldg(r + c[j]));
      sum = 0.f;
#pragma unroll
      for (int j = 0; j < K; ++j) sum = fmaf(xv[j], tab[packed_index<NIB>(cur, j)], sum);
    }
    if (i < A.nrows) {
      const float pi = fmaf(beta, pin[i], r[i]);
      const float api = (REC && beta != 0.f) ? fmaf(beta, Apin[i], sum) : sum;
      pout[i] = pi;
      Ap[i] = api;
      acc[0] += (double)pi * (double)api;
    }
  }
  grid_reduce<SumOp, 1>(acc, rs, AlphaFinish32{S});
}

// ------------------------------------------------------------------ bounded barrier waits
// Shared-memory mbarrier waits with an iteration bound: a wait that would never complete
// gives up after about one second of SM clock and reports instead of hanging the GPU.
namespace mbar {
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase with the given parity; gives up after ~1 s of SM clock.
__device__ __forceinline__ bool wait(unsigned long long* bar, unsigned parity) {
  const long long t0 = clock64();
  while (!try_wait(bar, parity))
    if (clock64() - t0 > 2000000000LL) return false;
  return true;
}
}  // namespace mbar

// A wait that can never complete (no arrival): the bounded wait must give up.
__global__ void k_bounded_wait_check(int* status) {
  __shared__ __align__(8) unsigned long long bar;
  if (threadIdx.x == 0) {
    mbar::init(&bar, 1);
    mbar::init_fence();
    *status = mbar::wait(&bar, 0) ? GIPB200_OK : GIPB200_ERR_TIMEOUT;
  }
}

struct BetaFinish32 {
  PcgScalars* S;
  double delta;
  int maxit;
  int pin_row;
  const double* scale;
  const float* y32;
  int use_cond;
  cudaGraphConditionalHandle upd_cond;
  int amg;  // beta and r.z come from the preconditioner's last kernel instead
  __device__ void operator()(const double* t) const {
    S->iter += 1;
    S->total_inner += 1;
    const double rz_new = t[0];
    if (rz_new > S->maxr2) S->maxr2 = rz_new;
    const bool upd = !(rz_new > S->trig) || !(rz_new > delta * delta * S->maxr2) ||
                     S->alpha == 0.0 || S->total_inner >= maxit || !isfinite(rz_new);
    if (upd) {
      S->upd = 1;
      S->kappa = (pin_row >= 0) ? S->kappa_c - scale[pin_row] * (double)__ldcg(y32 + pin_row) : 0.0;
    } else if (!amg) {
      S->beta = rz_new / S->rz;
      S->rz = rz_new;
    }
    set_loop(use_cond, upd_cond, upd);
  }
};

// y += alpha p; r^ -= alpha A^p; r^.r^; decide on a replacement
// y += alpha p, r -= alpha Ap, r.r; four rows per thread per pass (16-byte accesses).
// All grids stride through their rows in step, so a kernel's most recent accesses are the
// end of its sweep, still in L2.  This update sweeps backwards from the last row, where
// the SpMV (forward) ended, and p = r + beta p sweeps forwards from the first row, where
// this update ended.
__global__ void __launch_bounds__(256) k_mx_update(int n, float* __restrict__ y,
                                                   float* __restrict__ r,
                                                   const float* __restrict__ p,
                                                   const float* __restrict__ Ap, PcgScalars* S,
                                                   ReduceScratch rs, double delta, int maxit,
                                                   int pin_row, const double* __restrict__ scale,
                                                   int use_cond, cudaGraphConditionalHandle upd_cond,
                                                   int amg) {
  mx_enter(S, 0, 0);
  if (S->done) return;
  const float alpha = (float)S->alpha;
  double acc[1] = {0.0};
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  const int n4 = n >> 2;
  float4* y4 = reinterpret_cast<float4*>(y);
  float4* r4 = reinterpret_cast<float4*>(r);
  const float4* p4 = reinterpret_cast<const float4*>(p);
  const float4* a4 = reinterpret_cast<const float4*>(Ap);
  for (int t = tid; t < n4; t += stride) {
    const int q = n4 - 1 - t;
    float4 yv = y4[q], rv = r4[q];
    const float4 pv = p4[q], av = a4[q];
    yv.x = fmaf(alpha, pv.x, yv.x);
    yv.y = fmaf(alpha, pv.y, yv.y);
    yv.z = fmaf(alpha, pv.z, yv.z);
    yv.w = fmaf(alpha, pv.w, yv.w);
    rv.x = fmaf(-alpha, av.x, rv.x);
    rv.y = fmaf(-alpha, av.y, rv.y);
    rv.z = fmaf(-alpha, av.z, rv.z);
    rv.w = fmaf(-alpha, av.w, rv.w);
    y4[q] = yv;
    r4[q] = rv;
    acc[0] += (double)rv.x * (double)rv.x + (double)rv.y * (double)rv.y +
              (double)rv.z * (double)rv.z + (double)rv.w * (double)rv.w;
  }
  for (int i = 4 * n4 + tid; i < n; i += stride) {
    y[i] = fmaf(alpha, p[i], y[i]);
    const float ri = fmaf(-alpha, Ap[i], r[i]);
    r[i] = ri;
    acc[0] += (double)ri * (double)ri;
  }
  grid_reduce<SumOp, 1>(acc, rs,
                        BetaFinish32{S, delta, maxit, pin_row, scale, y, use_cond, upd_cond, amg});
}

// x += S y + kappa (FP64); y = 0   -- only when a replacement is due
__global__ void __launch_bounds__(256) k_mx_apply(int n, double* __restrict__ x, float* __restrict__ y,
                                                  const double* __restrict__ scale,
                                                  PcgScalars* S) {
  mx_enter(S, 0, 0);
  if (!S->upd || S->done) return;
  const double kappa = S->kappa;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] += scale[i] * (double)y[i] + kappa;
    y[i] = 0.f;
  }
}

// p = r^ + beta p; sets the while-loop value

// scale = 1/sqrt(L_ii); lhat = S L S (columns outside the unknowns dropped to 0)
__global__ void k_mx_scale(int n, const int* __restrict__ rp, const int* __restrict__ col,
                           const double* __restrict__ val, double* __restrict__ scale) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = 0.0;
    for (int j = rp[i]; j < rp[i + 1]; ++j)
      if (col[j] == i) d = val[j];
    scale[i] = (d > 0.0) ? 1.0 / sqrt(d) : 0.0;
  }
}
__global__ void k_mx_lhat(SellView<double> L, const double* __restrict__ scale, int n,
                          int pin_row, double pin_val, float* __restrict__ lhat) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int s = gw; s < L.nslices; s += nw) {
    long long base;
    int len;
    slice_range(L, s, base, len);
    const int i = s * 32 + lane;
    for (int j = 0; j < len; ++j) {
      const long long k = base + 32LL * j + lane;
      const int c = L.col[k];
      float v = 0.f;
      if (c >= 0 && c < n && i < L.nrows) {
        const double a = (i == pin_row && c == pin_row) ? L.val[k] - pin_val : L.val[k];
        v = (float)(scale[i] * a * scale[c]);
      }
      lhat[k] = v;
    }
  }
}

// GIP_MatrixMulticore::setUpDiagonal (GIP_MatrixMulticore.cpp:177-210): 1/A_ii, the last
// diagonal entry of a row wins; rows without one get 0.
__global__ void k_pcg_inv_diag(int nrows, const int* __restrict__ rp, const int* __restrict__ col,
                               const double* __restrict__ val, double* __restrict__ dinv,
                               int* missing) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrows; i += gridDim.x * blockDim.x) {
    double d = 0.0;
    bool found = false;
    for (int j = rp[i]; j < rp[i + 1]; ++j)
      if (col[j] == i) {
        d = ddiv(1.0, val[j]);
        found = true;
      }
    dinv[i] = d;
    if (!found) atomicAdd(missing, 1);
  }
}

// ------------------------------------------------------------------ host side
Pcg::~Pcg() {
  if (h_sc) cudaFreeHost(h_sc);
  for (auto& bs : body_stream)
    if (bs) cudaStreamDestroy(bs);
}

int Pcg::init(const Sell* Lm, int nall, const gipb200_pcg_params& params, cudaStream_t s) {
  if (!Lm) return fail(GIPB200_ERR_ARG, "null operator");
  if (params.mode < 0 || params.mode > 2) return fail(GIPB200_ERR_ARG, "bad PCG mode");
  if (nall < Lm->nrows) return fail(GIPB200_ERR_ARG, "n_all (%d) < operator rows (%d)", nall, Lm->nrows);
  for (int k = 0; k < Lm->nnz; ++k)
    if (Lm->h_col[k] >= nall)
      return fail(GIPB200_ERR_ARG, "operator column %d beyond n_all=%d", Lm->h_col[k], nall);
  L = Lm;
  n = Lm->nrows;
  n_all = nall;
  prm = params;
  if (prm.mode != GIPB200_PCG_FIXED && !(prm.tol > 0)) return fail(GIPB200_ERR_ARG, "tol must be > 0");
  if (prm.precond != GIPB200_PRECOND_JACOBI && prm.precond != GIPB200_PRECOND_AMG)
    return fail(GIPB200_ERR_ARG, "unknown preconditioner %d", prm.precond);
  if (prm.precond == GIPB200_PRECOND_AMG && prm.mode == GIPB200_PCG_FIXED)
    return fail(GIPB200_ERR_ARG, "the AMG preconditioner needs a tolerance mode (TOL or MIXED)");
  if (prm.mode == GIPB200_PCG_MIXED) {
    if (!(prm.inner_tol > 0 && prm.inner_tol < 1))
      return fail(GIPB200_ERR_ARG, "inner_tol (replacement factor) must be in (0,1)");
    if (prm.max_outer <= 0) return fail(GIPB200_ERR_ARG, "max_outer must be positive");
  }
  GIPB_TRY(reduce_scratch_alloc(&partials, &ticket, &rs));
  GIPB_TRY(sc.alloc(1));
  GIPB_TRY(sc.zero(s));
  GIPB_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h_sc), sizeof(PcgScalars)));
  for (auto& bs : body_stream) GIPB_CUDA(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking));
  GIPB_TRY(grid_blocks(256, L->nslices * 32, 1, kMaxReduceBlocks, &blocks_spmv));
  GIPB_TRY(grid_blocks(256, std::max(n, 1), 4, kMaxReduceBlocks, &blocks_vec));
  if (prm.mode == GIPB200_PCG_MIXED) {
    GIPB_TRY(scale.alloc(n));
    GIPB_TRY(lhat.alloc((size_t)std::max<long long>(L->nslots, 1)));
    GIPB_TRY(p32.alloc(n_all));
    GIPB_TRY(p32.zero(s));
    GIPB_TRY(p32b.alloc(n_all));
    GIPB_TRY(p32b.zero(s));
    GIPB_TRY(Ap32.alloc(n));
    GIPB_TRY(Ap32.zero(s));
    // the product recurrence on the AMG path (beta small): its second product buffer
    // (GIPB200_AP_RECURRENCE=1; measured on the 256^3 cavity it saves no time: the
    // kernel is bound by latency, not by its second gather)
    rec = prm.precond == GIPB200_PRECOND_AMG && getenv("GIPB200_AP_RECURRENCE") != nullptr;
    if (rec) {
      GIPB_TRY(Ap32b.alloc(n));
      GIPB_TRY(Ap32b.zero(s));
    }
    GIPB_TRY(r32.alloc(n));
    GIPB_TRY(y32.alloc(n));
    if (n > 0) {
      int b;
      GIPB_TRY(grid_blocks(256, n, 1, 0, &b));
      k_mx_scale<<<b, 256, 0, s>>>(n, L->rowptr.p, L->csr_col.p, L->csr_val.p, scale.p);
      GIPB_LAUNCH_CHECK();
      setup_mark("solver buffers, scale");
      // pinned-Neumann detection on the host copy of L
      {
        std::vector<double> hval((size_t)std::max(L->nnz, 1));
        GIPB_CUDA(cudaMemcpy(hval.data(), L->csr_val.p, (size_t)L->nnz * 8, cudaMemcpyDeviceToHost));
        int npin = 0, prow = -1;
        double pval = 0.0;
        for (int i = 0; i < n; ++i) {
          double rsum = 0.0, diag = 0.0, amax = 0.0;
          for (int k = L->h_rowptr[i]; k < L->h_rowptr[i + 1]; ++k) {
            rsum += hval[k];
            amax = std::max(amax, std::fabs(hval[k]));
            if (L->h_col[k] == i) diag = hval[k];
          }
          if (std::fabs(rsum) > 1e-9 * amax) {
            ++npin;
            prow = i;
            pval = rsum;
            if (!(rsum > 0.0 && rsum < diag)) npin = 1 << 20;
          }
        }
        if (npin == 1) {
          pin_row = prow;
          pin_val = pval;
        }
      }
      setup_mark("pinned-Neumann detection");
      k_mx_lhat<<<blocks_spmv, 256, 0, s>>>(L->view(), scale.p, n, pin_row, pin_val, lhat.p);
      GIPB_LAUNCH_CHECK();
      GIPB_TRY(sort_fp32_rows(s));
      GIPB_CUDA(cudaStreamSynchronize(s));
      setup_mark("FP32 operator");
      if (prm.mode == GIPB200_PCG_MIXED && !getenv("GIPB200_NO_COMPRESS")) GIPB_TRY(build_compressed(s));
      setup_mark("packed FP32 operator");
      if (prm.precond == GIPB200_PRECOND_AMG) GIPB_TRY(build_amg(s));
    }
  } else {
    GIPB_TRY(dinv.alloc(n));
    GIPB_TRY(p.alloc(n_all));
    GIPB_TRY(Ap.alloc(n));
    GIPB_TRY(r.alloc(n));
    if (n > 0) {
      DevBuf<int> miss;
      GIPB_TRY(miss.alloc(1));
      GIPB_TRY(miss.zero(s));
      int b;
      GIPB_TRY(grid_blocks(256, n, 1, 0, &b));
      k_pcg_inv_diag<<<b, 256, 0, s>>>(n, L->rowptr.p, L->csr_col.p, L->csr_val.p, dinv.p, miss.p);
      GIPB_LAUNCH_CHECK();
      GIPB_CUDA(cudaStreamSynchronize(s));
    }
    if (prm.precond == GIPB200_PRECOND_AMG) GIPB_TRY(build_amg64(s));
  }
  GIPB_CUDA(cudaStreamSynchronize(s));
  return GIPB200_OK;
}

// AMG hierarchy of the inner system: the Jacobi-scaled operator S L S with the pin
// removed (the pure-Neumann part when L has the pinned structure), columns < n.  Its
// near-null vector is S^-1 1 (L_N 1 = 0).
int Pcg::build_amg(cudaStream_t s) {
  std::vector<double> hval((size_t)std::max(L->nnz, 1)), hs((size_t)std::max(n, 1));
  GIPB_CUDA(cudaMemcpyAsync(hval.data(), L->csr_val.p, (size_t)L->nnz * 8, cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaMemcpyAsync(hs.data(), scale.p, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaStreamSynchronize(s));
  std::vector<int> rp((size_t)n + 1, 0), ci;
  std::vector<double> v;
  ci.reserve((size_t)L->nnz);
  v.reserve((size_t)L->nnz);
  for (int i = 0; i < n; ++i) {
    for (int k = L->h_rowptr[i]; k < L->h_rowptr[i + 1]; ++k) {
      const int j = L->h_col[k];
      if (j >= n) continue;
      double a = hval[k];
      if (i == pin_row && j == pin_row) a -= pin_val;
      ci.push_back(j);
      v.push_back(hs[i] * a * hs[j]);
    }
    rp[i + 1] = (int)ci.size();
  }
  std::vector<double> z((size_t)n);
  for (int i = 0; i < n; ++i) z[i] = hs[i] > 0.0 ? 1.0 / hs[i] : 0.0;
  setup_mark("AMG: scaled operator on host");
  amg.reset(new Amg());
  GIPB_TRY(amg->build(n, rp.data(), ci.data(), v.data(), z.data(), pin_row >= 0, n, s));
  GIPB_TRY(z32.alloc((size_t)n_all));
  GIPB_TRY(z32.zero(s));
  return GIPB200_OK;
}

// FP64 AMG hierarchy of L itself (columns < n; GIP's pin keeps L definite), near-null
// vector the constants.
int Pcg::build_amg64(cudaStream_t s) {
  std::vector<double> hval((size_t)std::max(L->nnz, 1));
  GIPB_CUDA(cudaMemcpyAsync(hval.data(), L->csr_val.p, (size_t)L->nnz * 8, cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaStreamSynchronize(s));
  std::vector<int> rp((size_t)n + 1, 0), ci;
  std::vector<double> v;
  for (int i = 0; i < n; ++i) {
    for (int k = L->h_rowptr[i]; k < L->h_rowptr[i + 1]; ++k)
      if (L->h_col[k] < n) {
        ci.push_back(L->h_col[k]);
        v.push_back(hval[k]);
      }
    rp[i + 1] = (int)ci.size();
  }
  std::vector<double> z((size_t)n, 1.0);
  amg64.reset(new Amg64());
  GIPB_TRY(amg64->build(n, rp.data(), ci.data(), v.data(), z.data(), false, n_all, s));
  GIPB_TRY(z64.alloc((size_t)n));
  GIPB_TRY(z64.zero(s));
  return GIPB200_OK;
}

// Sorts each row of the FP32 operator by column (the mixed form's inner product order is
// free; L itself keeps GIP's order) and drops the zero-valued ghost columns to padding.
// Sorted rows give every slot of a slice one neighbour direction, which keeps the column
// spread per slot small for the packed layout.
int Pcg::sort_fp32_rows(cudaStream_t s) {
  const int ns = L->nslices;
  const long long nslots = L->nslots;
  if (ns == 0 || nslots == 0) return GIPB200_OK;
  std::vector<long long> sptr((size_t)ns + 1);
  std::vector<int> col((size_t)nslots);
  std::vector<float> val((size_t)nslots);
  std::vector<double> lval((size_t)nslots);
  GIPB_CUDA(cudaMemcpyAsync(sptr.data(), L->sptr.p, sptr.size() * 8, cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaMemcpyAsync(col.data(), L->col.p, col.size() * 4, cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaMemcpyAsync(val.data(), lhat.p, val.size() * 4, cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaMemcpyAsync(lval.data(), L->val.p, lval.size() * 8, cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaStreamSynchronize(s));
  const int nu = n;
  // ghost entries (columns >= n) per row, for the packed FP64 residual's constant part:
  // counted and listed from the original slots, before the rows are sorted
  const int nr = L->nrows;
  std::vector<int> gcount((size_t)nr + 1, 0);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nr; ++i) {
    const int sl = i >> 5, l = i & 31;
    const long long b0 = sptr[sl];
    const int len = (int)((sptr[sl + 1] - b0) >> 5);
    int g = 0;
    for (int j = 0; j < len; ++j) g += col[b0 + 32LL * j + l] >= nu ? 1 : 0;
    gcount[(size_t)i + 1] = g;
  }
  ghost_rows.clear();
  ghost_rp.assign(1, 0);
  for (int i = 0; i < nr; ++i)
    if (gcount[(size_t)i + 1] > 0) {
      ghost_rows.push_back(i);
      ghost_rp.push_back(ghost_rp.back() + gcount[(size_t)i + 1]);
    }
  ghost_col.assign((size_t)ghost_rp.back(), 0);
  ghost_val.assign((size_t)ghost_rp.back(), 0.0);
#pragma omp parallel for schedule(static)
  for (int g = 0; g < (int)ghost_rows.size(); ++g) {
    const int i = ghost_rows[g], sl = i >> 5, l = i & 31;
    const long long b0 = sptr[sl];
    const int len = (int)((sptr[sl + 1] - b0) >> 5);
    int o = ghost_rp[g];
    for (int j = 0; j < len; ++j) {
      const long long k = b0 + 32LL * j + l;
      if (col[k] >= nu) {
        ghost_col[(size_t)o] = col[k];
        ghost_val[(size_t)o] = lval[k];
        ++o;
      }
    }
  }
  // each row's inner entries sorted by column; L's FP64 values follow in lval_sorted (the
  // packed FP64 residual reads them in this order)
  lval_sorted.assign((size_t)nslots, 0.0);
#pragma omp parallel for schedule(static)
  for (int sl = 0; sl < ns; ++sl) {
    const long long b0 = sptr[sl];
    const int len = (int)((sptr[sl + 1] - b0) >> 5);
    struct E {
      int c;
      float v;
      double lv;
    };
    std::vector<E> row((size_t)len);
    for (int l = 0; l < 32; ++l) {
      int m = 0;
      for (int j = 0; j < len; ++j) {
        const long long k = b0 + 32LL * j + l;
        const int c = col[k];
        if (c >= 0 && c < nu) row[m++] = {c, val[k], lval[k]};
      }
      std::stable_sort(row.begin(), row.begin() + m,
                       [](const E& x, const E& y) { return x.c < y.c; });
      for (int j = 0; j < len; ++j) {
        const long long k = b0 + 32LL * j + l;
        col[k] = j < m ? row[j].c : -1;
        val[k] = j < m ? row[j].v : 0.0f;
        lval_sorted[k] = j < m ? row[j].lv : 0.0;
      }
    }
  }
  GIPB_TRY(col32.upload(col.data(), col.size(), s));
  GIPB_CUDA(cudaMemcpyAsync(lhat.p, val.data(), val.size() * 4, cudaMemcpyHostToDevice, s));
  GIPB_CUDA(cudaStreamSynchronize(s));
  return GIPB200_OK;
}

int Pcg::build_compressed(cudaStream_t s) {
  const int ns = L->nslices;
  const long long nslots = L->nslots;
  if (ns == 0 || nslots == 0) return GIPB200_OK;
  std::vector<long long> sptr((size_t)ns + 1);
  std::vector<int> col((size_t)nslots);
  std::vector<float> val((size_t)nslots);
  GIPB_CUDA(cudaMemcpyAsync(sptr.data(), L->sptr.p, sptr.size() * 8, cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaMemcpyAsync(col.data(), col32.p, col.size() * 4, cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaMemcpyAsync(val.data(), lhat.p, val.size() * 4, cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaStreamSynchronize(s));
  // value table over the nonzero values (index 0 = 0.0f)
  std::vector<unsigned> keys;
  for (long long k = 0; k < nslots; ++k) {
    if (col[k] < 0 || val[k] == 0.0f) continue;
    unsigned bits;
    memcpy(&bits, &val[k], 4);
    if (std::find(keys.begin(), keys.end(), bits) == keys.end()) {
      if (keys.size() >= 255) return GIPB200_OK;  // no table: plain layout only
      keys.push_back(bits);
    }
  }
  std::sort(keys.begin(), keys.end());
  const int nib = keys.size() <= 15 ? 4 : 8;
  std::vector<float> table((size_t)1 << nib, 0.0f);
  for (size_t t = 0; t < keys.size(); ++t) memcpy(&table[t + 1], &keys[t], 4);
  auto index_of = [&](float v) -> unsigned {
    if (v == 0.0f) return 0u;
    unsigned bits;
    memcpy(&bits, &v, 4);
    return 1u + (unsigned)(std::lower_bound(keys.begin(), keys.end(), bits) - keys.begin());
  };
  const size_t nrow_pad = (size_t)ns * 32;
  std::vector<uint4> delta(nrow_pad, make_uint4(0u, 0u, 0u, 0u));
  std::vector<unsigned> idx4(nib == 4 ? nrow_pad : 0, 0u);
  std::vector<uint2> idx8(nib == 8 ? nrow_pad : 0, make_uint2(0u, 0u));
  std::vector<int> base((size_t)ns * 8, 0);
  std::vector<unsigned char> plain((size_t)ns, 1);
  long long packed_slots = 0, plain_slots = 0, packed_slices = 0;
  int max_len = 0;
#pragma omp parallel for schedule(static) reduction(+ : packed_slots, plain_slots, packed_slices) \
    reduction(max : max_len)
  for (int sl = 0; sl < ns; ++sl) {
    const long long b0 = sptr[sl];
    const int len = (int)((sptr[sl + 1] - b0) >> 5);
    bool ok = len <= 8;
    int lo[8], hi[8];
    for (int j = 0; j < 8; ++j) lo[j] = 0x7fffffff, hi[j] = -1;
    for (int j = 0; j < len && ok; ++j) {
      for (int l = 0; l < 32; ++l) {
        const long long k = b0 + 32LL * j + l;
        if (col[k] >= 0 && val[k] != 0.0f) {
          lo[j] = std::min(lo[j], col[k]);
          hi[j] = std::max(hi[j], col[k]);
        }
      }
      if (hi[j] >= 0 && hi[j] - lo[j] > 65535) ok = false;
    }
    if (!ok) {
      plain_slots += 32LL * len;
      for (int j = 0; j < 8; ++j) base[(size_t)sl * 8 + j] = -1;  // marks a plain slice
      continue;
    }
    plain[sl] = 0;
    packed_slots += 32LL * len;
    packed_slices += 1;
    max_len = std::max(max_len, len);
    for (int j = 0; j < 8; ++j) base[(size_t)sl * 8 + j] = hi[j] >= 0 ? lo[j] : 0;
    for (int l = 0; l < 32; ++l) {
      unsigned dw[4] = {0u, 0u, 0u, 0u};
      unsigned long long iw = 0ull;
      for (int j = 0; j < len; ++j) {
        const long long k = b0 + 32LL * j + l;
        if (col[k] < 0 || val[k] == 0.0f) continue;
        const unsigned d = (unsigned)(col[k] - lo[j]);
        dw[j >> 1] |= d << (16 * (j & 1));
        iw |= (unsigned long long)index_of(val[k]) << (nib * j);
      }
      const size_t r = (size_t)sl * 32 + l;
      delta[r] = make_uint4(dw[0], dw[1], dw[2], dw[3]);
      if (nib == 4) idx4[r] = (unsigned)iw;
      else idx8[r] = make_uint2((unsigned)iw, (unsigned)(iw >> 32));
    }
  }
  cop.compressed_fraction = (double)packed_slots / (double)nslots;
  if (cop.compressed_fraction < 0.5) return GIPB200_OK;  // not worth a second layout
  GIPB_TRY(cop.delta.upload(delta.data(), delta.size(), s));
  if (nib == 4) GIPB_TRY(cop.idx4.upload(idx4.data(), idx4.size(), s));
  else GIPB_TRY(cop.idx8.upload(idx8.data(), idx8.size(), s));
  GIPB_TRY(cop.base.upload(base.data(), base.size(), s));
  GIPB_TRY(cop.plain.upload(plain.data(), plain.size(), s));
  GIPB_TRY(cop.table.upload(table.data(), table.size(), s));
  GIPB_CUDA(cudaStreamSynchronize(s));
  cop.index_bits = nib;
  cop.slots = max_len <= 7 ? 7 : 8;
  cop.ntable = (int)keys.size() + 1;
  // streamed bytes: packed rows (delta + index words), their slot bases; plain slices
  // (column + value per slot, slice offsets); the plain flags; per row r and the old
  // direction read once, the new direction and the product written once
  const double packed_rows = 32.0 * (double)packed_slices;
  cop.bytes_per_launch = packed_rows * (16.0 + nib) + (double)packed_slices * 32.0 +
                         (double)plain_slots * 8.0 + (double)(ns - packed_slices) * 16.0 +
                         (double)ns + (double)L->nrows * 16.0;
  cop.enabled = true;
  // The FP64 residual from the same packed columns: a 4-bit index per slot into a table of
  // L's (at most 15 distinct nonzero) values in the sorted slot order.  Left off when L has
  // more values, or a slot the FP32 packing dropped (a stored zero of S L S) holds a
  // nonzero of L.
  lpacked = false;
  if (!getenv("GIPB200_NO_PACKED_RESIDUAL") && lval_sorted.size() == (size_t)nslots) {
    std::vector<unsigned long long> lkeys;
    bool ok = true;
    for (long long k = 0; k < nslots && ok; ++k) {
      if (col[k] < 0) continue;
      const double v = lval_sorted[(size_t)k];
      if (val[k] == 0.0f) {
        ok = v == 0.0;
        continue;
      }
      unsigned long long bits;
      memcpy(&bits, &v, 8);
      if (v != 0.0 && std::find(lkeys.begin(), lkeys.end(), bits) == lkeys.end()) {
        if (lkeys.size() >= 15) ok = false;
        else lkeys.push_back(bits);
      }
    }
    if (ok) {
      std::sort(lkeys.begin(), lkeys.end());
      std::vector<double> ltab(16, 0.0);
      for (size_t t = 0; t < lkeys.size(); ++t) memcpy(&ltab[t + 1], &lkeys[t], 8);
      std::vector<unsigned> lidx(nrow_pad, 0u);
#pragma omp parallel for schedule(static)
      for (int sl = 0; sl < ns; ++sl) {
        if (plain[sl]) continue;
        const long long b0 = sptr[sl];
        const int len = (int)((sptr[sl + 1] - b0) >> 5);
        for (int l = 0; l < 32; ++l) {
          unsigned w = 0u;
          for (int j = 0; j < len; ++j) {
            const long long k = b0 + 32LL * j + l;
            if (col[k] < 0 || val[k] == 0.0f) continue;
            const double v = lval_sorted[(size_t)k];
            unsigned long long bits;
            memcpy(&bits, &v, 8);
            const unsigned t =
                v == 0.0 ? 0u
                         : 1u + (unsigned)(std::lower_bound(lkeys.begin(), lkeys.end(), bits) -
                                           lkeys.begin());
            w |= t << (4 * j);
          }
          lidx[(size_t)sl * 32 + l] = w;
        }
      }
      GIPB_TRY(lidx4.upload(lidx.data(), lidx.size(), s));
      GIPB_TRY(ltable.upload(ltab.data(), ltab.size(), s));
      const int ng = (int)ghost_rows.size();
      // (an empty list uploads nothing: the buffer keeps its one-element minimum)
      GIPB_TRY(d_ghost_rows.upload(ghost_rows.data(), (size_t)ng, s));
      GIPB_TRY(d_ghost_rp.upload(ghost_rp.data(), ghost_rp.size(), s));
      GIPB_TRY(d_ghost_col.upload(ghost_col.data(), ghost_col.size(), s));
      GIPB_TRY(d_ghost_val.upload(ghost_val.data(), ghost_val.size(), s));
      GIPB_TRY(bprime.alloc((size_t)std::max(n, 1)));
      GIPB_CUDA(cudaStreamSynchronize(s));
      lpacked = true;
    }
  }
  lval_sorted.clear();
  lval_sorted.shrink_to_fit();
  return GIPB200_OK;
}

double Pcg::iteration_bytes() const {
  const double nn = n, nnz = L->nnz;
  if (prm.mode == GIPB200_PCG_MIXED) {
    // plain FP32 operator stream: column + value per slot, slice offsets
    const double plain = (double)L->nslots * 8.0 + (L->nslices + 1.0) * 8.0;
    const double spmv = (cop.enabled ? cop.bytes_per_launch : plain + 16.0 * nn) +
                        (rec ? 4.0 * nn : 0.0);  // the previous A p read by the recurrence
    double b = spmv + 24.0 * nn;  // SpMV-dot (direction formed inside), y/r update
    if (amg) b += amg->cycle_bytes(cop.enabled ? cop.bytes_per_launch - 16.0 * nn : plain);
    return b;
  }
  const double spmv = 12.0 * nnz + 16.0 * nn;
  if (amg64) {  // update (x, r read and written; p, Ap read), cycle, p = z + beta p
    const double a0 = (double)L->nslots * 12.0 + (L->nslices + 1.0) * 8.0;
    return spmv + 48.0 * nn + amg64->cycle_bytes(a0) + 24.0 * nn;
  }
  return spmv + 56.0 * nn + 32.0 * nn;  // GIP's loop: x, r, z, dots; p = z + beta p
}

double Pcg::replacement_bytes() const {
  if (prm.mode != GIPB200_PCG_MIXED) return 0.0;
  const double nn = n;
  if (lpacked)  // packed columns, value indices, slot bases, b', scale read, r^ written, fold
    return (16.0 + 4.0 + 8.0 + 8.0 + 4.0) * nn + 32.0 * L->nslices + 8.0 * n_all +
           (16.0 + 8.0 + 4.0 + 4.0) * nn;
  // FP64 r = b - L x with the FP32 restart (L, x gathered, b, scale read, r^ written) and
  // the fold x += S y + kappa, y = 0
  return 12.0 * L->nnz + (L->nslices + 1.0) * 8.0 + 8.0 * n_all + 16.0 * nn + 4.0 * nn +
         (16.0 + 8.0 + 4.0 + 4.0) * nn;
}

int Pcg::set_launch(int spmv_blocks, int vec_blocks) {
  if (spmv_blocks < 0 || vec_blocks < 0 || spmv_blocks > kMaxReduceBlocks ||
      vec_blocks > kMaxReduceBlocks)
    return fail(GIPB200_ERR_ARG, "launch blocks must be in [0, %d]", kMaxReduceBlocks);
  if (spmv_blocks) blocks_spmv = spmv_blocks;
  else GIPB_TRY(grid_blocks(256, L->nslices * 32, 1, kMaxReduceBlocks, &blocks_spmv));
  if (vec_blocks) blocks_vec = vec_blocks;
  else GIPB_TRY(grid_blocks(256, std::max(n, 1), 4, kMaxReduceBlocks, &blocks_vec));
  return GIPB200_OK;
}

int Pcg::read_flag(cudaStream_t s, int which, int* v) {
  GIPB_CUDA(cudaMemcpyAsync(h_sc, sc.p, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaStreamSynchronize(s));
  *v = which == 0 ? h_sc->done : h_sc->inner_done;
  return GIPB200_OK;
}

static void launch_mx_spmv(const Pcg& P, const float* pin, float* pout, const float* Apin,
                           float* Ap, PcgScalars* sc, int use_cond, cudaGraphConditionalHandle h,
                           cudaStream_t s);

// ------------------------------------------------------------------ conditional while-nodes
static bool capturing(cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &st) != cudaSuccess) return false;
  return st == cudaStreamCaptureStatusActive;
}

static int make_handle(cudaStream_t cs, unsigned def, unsigned flags,
                       cudaGraphConditionalHandle* h) {
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  GIPB_CUDA(cudaStreamGetCaptureInfo(cs, &st, nullptr, &g, nullptr, nullptr));
  if (st != cudaStreamCaptureStatusActive || !g)
    return fail(GIPB200_ERR_STATE, "stream is not capturing");
  GIPB_CUDA(cudaGraphConditionalHandleCreate(h, g, def, flags));
  return GIPB200_OK;
}

// Appends a while-node after everything captured so far on `cs`; returns its body graph
// and makes the node the capture frontier of `cs`.
static int add_while(cudaStream_t cs, cudaGraphConditionalHandle h, cudaGraph_t* body) {
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  GIPB_CUDA(cudaStreamGetCaptureInfo(cs, &st, nullptr, &g, &deps, &nd));
  // the parameter union has no default constructor: zeroed raw storage
  alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
  memset(raw, 0, sizeof(raw));
  cudaGraphNodeParams& p = *reinterpret_cast<cudaGraphNodeParams*>(raw);
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  GIPB_CUDA(cudaGraphAddNode(&node, g, deps, nd, &p));
  *body = p.conditional.phGraph_out[0];
  GIPB_CUDA(cudaStreamUpdateCaptureDependencies(cs, &node, 1, cudaStreamSetCaptureDependencies));
  return GIPB200_OK;
}

// Host-driven solves read the device's stop flag every 16 iterations (each read is a host
// wait); GIPB200_HOST_POLL=k reads it every k (profiling: 1 leaves no finished-solve
// launches in a launch list).
static int host_poll_interval() {
  const char* e = getenv("GIPB200_HOST_POLL");
  const int k = e ? atoi(e) : 16;
  return k > 0 ? k : 16;
}

int Pcg::enqueue(const double* b, double* x, const double* x0, cudaStream_t s, bool host_sync) {
  if (!host_sync && prm.mode != GIPB200_PCG_FIXED && capturing(s)) {
    if (!body_stream[0]) {
      return fail(GIPB200_ERR_STATE, "capture streams missing");
    }
    return prm.mode == GIPB200_PCG_MIXED ? enqueue_mixed_graph(b, x, x0, s)
                                         : enqueue_fp64_graph(b, x, x0, s);
  }
  if (prm.mode == GIPB200_PCG_MIXED) return enqueue_mixed(b, x, x0, s, host_sync);
  return enqueue_fp64(b, x, x0, s, host_sync);
}

// TOL mode inside a graph: init, then while(!done) { A; B; C }.  C sets the loop value
// from the stop flag; the flag is set by a convergence test or the maxit cap, so the
// loop always ends.
void Pcg::launch_pcg_update(double* x, cudaStream_t s) {
  if ((reinterpret_cast<uintptr_t>(x) & 15u) == 0)
    k_pcg_update<true><<<blocks_vec, 256, 0, s>>>(n, x, r.p, p.p, Ap.p, dinv.p, sc.p, rs, prm.mode,
                                                  prm.maxit, prm.tol);
  else
    k_pcg_update<false><<<blocks_vec, 256, 0, s>>>(n, x, r.p, p.p, Ap.p, dinv.p, sc.p, rs,
                                                   prm.mode, prm.maxit, prm.tol);
}

int Pcg::enqueue_fp64_graph(const double* b, double* x, const double* x0, cudaStream_t s) {
  cudaGraphConditionalHandle h;
  GIPB_TRY(make_handle(s, 0, 0, &h));
  if (x != x0) GIPB_CUDA(cudaMemcpyAsync(x, x0, (size_t)n_all * 8, cudaMemcpyDeviceToDevice, s));
  GIPB_CUDA(cudaMemcpyAsync(p.p, x0, (size_t)n_all * 8, cudaMemcpyDeviceToDevice, s));
  if (n > 0) GIPB_CUDA(cudaMemcpyAsync(Ap.p, x0, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
  k_pcg_init<<<blocks_spmv, 256, 0, s>>>(L->view(), x, b, dinv.p, r.p, p.p, Ap.p, sc.p, rs,
                                          prm.mode, prm.maxit, prm.tol, 1, h);
  GIPB_LAUNCH_CHECK();
  if (amg64) {  // z = M r, p = z
    GIPB_TRY(amg64->enqueue(L->view(), r.p, z64.p, sc.p, rs, 1, s));
    k_pcg_pupdate_z<<<blocks_vec, 256, 0, s>>>(n, p.p, z64.p, sc.p, 1, h);
  }
  cudaGraph_t body;
  GIPB_TRY(add_while(s, h, &body));
  cudaStream_t bs = body_stream[0];
  GIPB_CUDA(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed));
  k_pcg_spmv_dot<<<blocks_spmv, 256, 0, bs>>>(L->view(), p.p, Ap.p, sc.p, rs, prm.mode);
  int ast = GIPB200_OK;
  if (amg64) {
    k_pcg_update_amg<<<blocks_vec, 256, 0, bs>>>(n, x, r.p, p.p, Ap.p, sc.p, rs, prm.maxit, prm.tol);
    ast = amg64->enqueue(L->view(), r.p, z64.p, sc.p, rs, 0, bs);
    k_pcg_pupdate_z<<<blocks_vec, 256, 0, bs>>>(n, p.p, z64.p, sc.p, 1, h);
  } else {
    launch_pcg_update(x, bs);
    k_pcg_pupdate<<<blocks_vec, 256, 0, bs>>>(n, p.p, r.p, dinv.p, sc.p, 1, h);
  }
  cudaError_t le = cudaGetLastError();
  cudaGraph_t out = nullptr;
  GIPB_CUDA(cudaStreamEndCapture(bs, &out));
  if (ast != GIPB200_OK) return ast;
  if (le != cudaSuccess) return fail(GIPB200_ERR_CUDA, "launch in loop body: %s", cudaGetErrorString(le));
  launches += 4;
  return GIPB200_OK;
}

// MIXED inside a graph:
//   residual (first); while(!done) { A; B; if(upd) { apply; residual }; C }
// B decides a replacement on the device and sets the if-node; C sets the loop value.
static int add_if(cudaStream_t cs, cudaGraphConditionalHandle h, cudaGraph_t* body) {
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  GIPB_CUDA(cudaStreamGetCaptureInfo(cs, &st, nullptr, &g, &deps, &nd));
  alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
  memset(raw, 0, sizeof(raw));
  cudaGraphNodeParams& p = *reinterpret_cast<cudaGraphNodeParams*>(raw);
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeIf;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  GIPB_CUDA(cudaGraphAddNode(&node, g, deps, nd, &p));
  *body = p.conditional.phGraph_out[0];
  GIPB_CUDA(cudaStreamUpdateCaptureDependencies(cs, &node, 1, cudaStreamSetCaptureDependencies));
  return GIPB200_OK;
}

int Pcg::enqueue_mixed_graph(const double* b, double* x, const double* x0, cudaStream_t s) {
  const PackedView pk0 = packed();
  cudaGraphConditionalHandle hl;
  GIPB_TRY(make_handle(s, 0, 0, &hl));
  if (x != x0) GIPB_CUDA(cudaMemcpyAsync(x, x0, (size_t)n_all * 8, cudaMemcpyDeviceToDevice, s));
  GIPB_CUDA(cudaMemsetAsync(sc.p, 0, sizeof(PcgScalars), s));
  if (amg) GIPB_TRY(amg->reset_tail(s));
  GIPB_TRY(launch_mixed_residual(b, x, 1, s, 1, hl));
  if (amg) GIPB_TRY(amg->enqueue(a32(), r32.p, z32.p, sc.p, rs, 0, s, &pk0));
  cudaGraph_t loop_body;
  GIPB_TRY(add_while(s, hl, &loop_body));
  cudaStream_t os = body_stream[0], is = body_stream[1];
  GIPB_CUDA(cudaStreamBeginCaptureToGraph(os, loop_body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed));
  // two iterations per body: the first reads direction buffer p32 and writes p32b, the
  // second the reverse.  Each kernel returns at once when the solve has finished, and
  // the SpMV sets the loop condition, so the loop ends within one body of the stop flag.
  int st = [&]() -> int {
    for (int half = 0; half < 2; ++half) {
      float* pin = half ? p32b.p : p32.p;
      float* pout = half ? p32.p : p32b.p;
      // with the product recurrence the products alternate like the directions
      float* apin = (rec && half) ? Ap32b.p : Ap32.p;
      float* apout = rec ? (half ? Ap32.p : Ap32b.p) : Ap32.p;
      cudaGraphConditionalHandle hu;
      GIPB_TRY(make_handle(os, 0, 0, &hu));
      launch_mx_spmv(*this, pin, pout, apin, apout, sc.p, 1, hl, os);
      launch_dep(k_mx_update, blocks_vec, 256, os, n, y32.p, r32.p, (const float*)pout,
                 (const float*)apout, sc.p, rs, prm.inner_tol, prm.maxit, pin_row,
                 (const double*)scale.p, 1, hu, amg ? 1 : 0);
      GIPB_LAUNCH_CHECK();
      cudaGraph_t if_body;
      GIPB_TRY(add_if(os, hu, &if_body));
      GIPB_CUDA(cudaStreamBeginCaptureToGraph(is, if_body, nullptr, nullptr, 0,
                                              cudaStreamCaptureModeRelaxed));
      launch_dep(k_mx_apply, blocks_vec, 256, is, n, x, y32.p, (const double*)scale.p, sc.p);
      int rst = launch_mixed_residual(b, x, 0, is, 0, 0);
      cudaError_t le = cudaGetLastError();
      cudaGraph_t out = nullptr;
      GIPB_CUDA(cudaStreamEndCapture(is, &out));
      if (rst != GIPB200_OK) return rst;
      if (le != cudaSuccess)
        return fail(GIPB200_ERR_CUDA, "launch in replacement body: %s", cudaGetErrorString(le));
      if (amg) GIPB_TRY(amg->enqueue(a32(), r32.p, z32.p, sc.p, rs, 0, os, &pk0));
    }
    return GIPB200_OK;
  }();
  cudaGraph_t out = nullptr;
  cudaError_t ce = cudaStreamEndCapture(os, &out);
  if (st != GIPB200_OK) return st;
  if (ce != cudaSuccess) return fail(GIPB200_ERR_CUDA, "loop body capture: %s", cudaGetErrorString(ce));
  launches += 8;
  return GIPB200_OK;
}

int Pcg::enqueue_fp64(const double* b, double* x, const double* x0, cudaStream_t s,
                      bool host_sync) {
  // dp = dAx = x = x0 over all cells (GIP_LinearSolver.h:56,66,67)
  if (x != x0) GIPB_CUDA(cudaMemcpyAsync(x, x0, (size_t)n_all * 8, cudaMemcpyDeviceToDevice, s));
  GIPB_CUDA(cudaMemcpyAsync(p.p, x0, (size_t)n_all * 8, cudaMemcpyDeviceToDevice, s));
  if (n > 0) GIPB_CUDA(cudaMemcpyAsync(Ap.p, x0, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
  k_pcg_init<<<blocks_spmv, 256, 0, s>>>(L->view(), x, b, dinv.p, r.p, p.p, Ap.p, sc.p, rs,
                                          prm.mode, prm.maxit, prm.tol, 0, 0);
  GIPB_LAUNCH_CHECK();
  launches += 1;
  if (amg64) {  // z = M r, p = z
    GIPB_TRY(amg64->enqueue(L->view(), r.p, z64.p, sc.p, rs, 1, s));
    k_pcg_pupdate_z<<<blocks_vec, 256, 0, s>>>(n, p.p, z64.p, sc.p, 0, 0);
  }
  const int poll = host_poll_interval();
  for (int k = 0; k < prm.maxit; ++k) {
    k_pcg_spmv_dot<<<blocks_spmv, 256, 0, s>>>(L->view(), p.p, Ap.p, sc.p, rs, prm.mode);
    if (amg64) {
      k_pcg_update_amg<<<blocks_vec, 256, 0, s>>>(n, x, r.p, p.p, Ap.p, sc.p, rs, prm.maxit,
                                                   prm.tol);
      GIPB_TRY(amg64->enqueue(L->view(), r.p, z64.p, sc.p, rs, 0, s));
      k_pcg_pupdate_z<<<blocks_vec, 256, 0, s>>>(n, p.p, z64.p, sc.p, 0, 0);
    } else {
      launch_pcg_update(x, s);
      k_pcg_pupdate<<<blocks_vec, 256, 0, s>>>(n, p.p, r.p, dinv.p, sc.p, 0, 0);
    }
    GIPB_LAUNCH_CHECK();
    launches += 3;
    if (host_sync && prm.mode != GIPB200_PCG_FIXED && (k + 1) % poll == 0) {
      int d;
      GIPB_TRY(read_flag(s, 0, &d));
      if (d) break;
    }
  }
  return GIPB200_OK;
}

static void launch_mx_spmv(const Pcg& P, const float* pin, float* pout, const float* Apin,
                           float* Ap, PcgScalars* sc, int use_cond, cudaGraphConditionalHandle h,
                           cudaStream_t s) {
  const CompressedOp& c = P.cop;
  const SellView<float> A = P.a32();
  const int nb = P.blocks_spmv;
  const float* r = P.amg ? P.z32.p : P.r32.p;  // direction from the preconditioned residual
  const void* ix = c.index_bits == 4 ? (const void*)c.idx4.p : (const void*)c.idx8.p;
#define GIPB_MXP(NIB, K, REC)                                                                 \
  launch_dep(k_mxp_spmv_dot<NIB, K, REC>, nb, 256, s, A, (const uint4*)c.delta.p, ix,           \
             (const int*)c.base.p, (const unsigned char*)c.plain.p, (const float*)c.table.p, r,  \
             pin, pout, Ap, sc, P.rs, use_cond, h, Apin)
  if (!c.enabled) {
    if (P.rec)
      launch_dep(k_mx_spmv_dot<true>, nb, 256, s, A, r, pin, pout, Ap, sc, P.rs, use_cond, h, Apin);
    else
      launch_dep(k_mx_spmv_dot<false>, nb, 256, s, A, r, pin, pout, Ap, sc, P.rs, use_cond, h,
                 Apin);
  } else if (c.index_bits == 4 && c.slots == 7) {
    if (P.rec) GIPB_MXP(4, 7, true); else GIPB_MXP(4, 7, false);
  } else if (c.index_bits == 4) {
    if (P.rec) GIPB_MXP(4, 8, true); else GIPB_MXP(4, 8, false);
  } else if (c.slots == 7) {
    if (P.rec) GIPB_MXP(8, 7, true); else GIPB_MXP(8, 7, false);
  } else {
    if (P.rec) GIPB_MXP(8, 8, true); else GIPB_MXP(8, 8, false);
  }
#undef GIPB_MXP
}

int Pcg::launch_mixed_residual(const double* b, const double* x, int first, cudaStream_t s,
                               int use_cond, cudaGraphConditionalHandle h) {
  if (lpacked) {
    if (first) {  // b' = b - L_ghost x for this solve (x's ghost entries stay fixed)
      GIPB_CUDA(cudaMemcpyAsync(bprime.p, b, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice,
                                s));
      const int ng = (int)ghost_rows.size();
      if (ng > 0) {
        int gb = 1;
        GIPB_TRY(grid_blocks(256, ng, 1, 0, &gb));
        k_mx_ghost_rhs<<<gb, 256, 0, s>>>(ng, d_ghost_rows.p, d_ghost_rp.p, d_ghost_col.p,
                                          d_ghost_val.p, x, b, bprime.p);
        launches += 1;
      }
    }
    launch_dep(k_mx_residual_packed, blocks_spmv, 256, s, L->view(),
               (const uint4*)cop.delta.p, (const int*)cop.base.p,
               (const unsigned char*)cop.plain.p, (const unsigned*)lidx4.p,
               (const double*)ltable.p, (const double*)bprime.p, (const double*)x, b,
               (const double*)scale.p, r32.p, p32.p, y32.p, sc.p, rs, first, prm.tol,
               prm.inner_tol, prm.maxit, prm.max_outer, pin_row, pin_val, use_cond, h,
               amg ? 1 : 0);
    GIPB_LAUNCH_CHECK();
    launches += 1;
    return GIPB200_OK;
  }
  launch_dep(k_mx_residual, blocks_spmv, 256, s, L->view(), (const double*)x, b,
             (const double*)scale.p, r32.p, p32.p, y32.p, sc.p, rs, first, prm.tol, prm.inner_tol,
             prm.maxit, prm.max_outer, pin_row, pin_val, use_cond, h, amg ? 1 : 0);
  GIPB_LAUNCH_CHECK();
  launches += 1;
  return GIPB200_OK;
}

int Pcg::enqueue_mixed(const double* b, double* x, const double* x0, cudaStream_t s,
                       bool host_sync) {
  const PackedView pk0 = packed();
  if (x != x0) GIPB_CUDA(cudaMemcpyAsync(x, x0, (size_t)n_all * 8, cudaMemcpyDeviceToDevice, s));
  GIPB_CUDA(cudaMemsetAsync(sc.p, 0, sizeof(PcgScalars), s));
  if (amg) GIPB_TRY(amg->reset_tail(s));
  GIPB_TRY(launch_mixed_residual(b, x, 1, s, 0, 0));
  if (amg) GIPB_TRY(amg->enqueue(a32(), r32.p, z32.p, sc.p, rs, 0, s, &pk0));
  const int poll = host_poll_interval();
  for (int k = 0; k < prm.maxit; ++k) {
    float* pin = (k & 1) ? p32b.p : p32.p;
    float* pout = (k & 1) ? p32.p : p32b.p;
    float* apin = (rec && (k & 1)) ? Ap32b.p : Ap32.p;
    float* apout = rec ? ((k & 1) ? Ap32.p : Ap32b.p) : Ap32.p;
    launch_mx_spmv(*this, pin, pout, apin, apout, sc.p, 0, 0, s);
    launch_dep(k_mx_update, blocks_vec, 256, s, n, y32.p, r32.p, (const float*)pout,
               (const float*)apout, sc.p, rs, prm.inner_tol, prm.maxit, pin_row,
               (const double*)scale.p, 0, (cudaGraphConditionalHandle)0, amg ? 1 : 0);
    launch_dep(k_mx_apply, blocks_vec, 256, s, n, x, y32.p, (const double*)scale.p, sc.p);
    GIPB_LAUNCH_CHECK();
    GIPB_TRY(launch_mixed_residual(b, x, 0, s, 0, 0));
    if (amg) GIPB_TRY(amg->enqueue(a32(), r32.p, z32.p, sc.p, rs, 0, s, &pk0));
    launches += 4;
    if (host_sync && (k + 1) % poll == 0) {
      int d;
      GIPB_TRY(read_flag(s, 0, &d));
      if (d) break;
    }
  }
  return GIPB200_OK;
}

int Pcg::time_update(int reps, cudaStream_t s, double* avg_ms, double* bytes) {
  if (reps <= 0) return fail(GIPB200_ERR_ARG, "reps must be positive");
  if (prm.mode != GIPB200_PCG_MIXED)
    return fail(GIPB200_ERR_STATE, "the FP32 update exists only in the mixed form");
  // zeroed scratch scalars: alpha = 0, so y += 0 p and r -= 0 Ap rewrite y and r unchanged,
  // and the kernel's decisions land in the scratch scalars
  DevBuf<PcgScalars> tsc;
  GIPB_TRY(tsc.alloc(1));
  GIPB_TRY(tsc.zero(s));
  cudaEvent_t e0, e1;
  GIPB_CUDA(cudaEventCreate(&e0));
  GIPB_CUDA(cudaEventCreate(&e1));
  for (int k = 0; k <= reps; ++k) {
    if (k == 1) GIPB_CUDA(cudaEventRecord(e0, s));
    k_mx_update<<<blocks_vec, 256, 0, s>>>(n, y32.p, r32.p, p32.p, Ap32.p, tsc.p, rs,
                                           prm.inner_tol, prm.maxit, -1, scale.p, 0, 0, amg ? 1 : 0);
  }
  GIPB_LAUNCH_CHECK();
  GIPB_CUDA(cudaEventRecord(e1, s));
  GIPB_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  GIPB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *avg_ms = (double)ms / reps;
  *bytes = 24.0 * n;  // y and r read and written, p and Ap read (FP32)
  return GIPB200_OK;
}

int Pcg::time_spmv(int mixed, int reps, cudaStream_t s, double* avg_ms, double* bytes) {
  if (reps <= 0) return fail(GIPB200_ERR_ARG, "reps must be positive");
  if (mixed && prm.mode != GIPB200_PCG_MIXED)
    return fail(GIPB200_ERR_STATE, "the FP32 kernel exists only in the mixed form");
  if (!mixed && prm.mode == GIPB200_PCG_MIXED)
    return fail(GIPB200_ERR_STATE, "the FP64 PCG kernel exists only in the FP64 forms");
  DevBuf<PcgScalars> tsc;
  GIPB_TRY(tsc.alloc(1));
  GIPB_TRY(tsc.zero(s));
  {  // a nonzero beta, so the timed kernel reads everything an iteration reads
    PcgScalars h{};
    h.beta = 0.5;
    GIPB_CUDA(cudaMemcpyAsync(tsc.p, &h, sizeof(h), cudaMemcpyHostToDevice, s));
    GIPB_CUDA(cudaStreamSynchronize(s));
  }
  DevBuf<float> tAp32;
  DevBuf<double> tAp;
  cudaEvent_t e0, e1;
  GIPB_CUDA(cudaEventCreate(&e0));
  GIPB_CUDA(cudaEventCreate(&e1));
  if (mixed) {
    GIPB_TRY(tAp32.alloc(n));
  } else {
    GIPB_TRY(tAp.alloc(n));
    GIPB_CUDA(cudaMemcpyAsync(tAp.p, Ap.p, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
  }
  // one untimed launch, then the timed ones (the scratch scalars never set a stop flag
  // that would skip work: p.Ap > 0 for the SPD operator and a nonzero p)
  for (int k = 0; k <= reps; ++k) {
    if (k == 1) GIPB_CUDA(cudaEventRecord(e0, s));
    if (mixed)
      launch_mx_spmv(*this, p32.p, p32b.p, Ap32.p, tAp32.p, tsc.p, 0, 0, s);
    else
      k_pcg_spmv_dot<<<blocks_spmv, 256, 0, s>>>(L->view(), p.p, tAp.p, tsc.p, rs,
                                                  GIPB200_PCG_FIXED);
  }
  GIPB_LAUNCH_CHECK();
  GIPB_CUDA(cudaEventRecord(e1, s));
  GIPB_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  GIPB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *avg_ms = (double)ms / reps;
  // compulsory bytes: stored values + indices once, slice offsets, p once, Ap once
  // (mixed: r and the old direction read, the new direction and the product written)
  const double vbytes = mixed ? 4.0 : 8.0;
  *bytes = (double)L->nnz * (vbytes + 4.0) + (double)(L->nslices + 1) * 8.0 +
           (double)L->nrows * (mixed ? 4.0 : 2.0) * vbytes;
  if (mixed && cop.enabled) *bytes = cop.bytes_per_launch;
  if (mixed && rec) *bytes += 4.0 * L->nrows;  // the previous A p, read by the recurrence
  return GIPB200_OK;
}

int Pcg::profile_vcycle(int reps, cudaStream_t s, int cap, int* n_kernels, int* level, int* kind,
                        double* ms, double* bytes) {
  if (reps <= 0 || cap < 0 || !n_kernels) return fail(GIPB200_ERR_ARG, "bad arguments");
  if (!amg && !amg64) return fail(GIPB200_ERR_STATE, "the solver has no AMG preconditioner");
  // scratch scalars: the cycle's kernels run only while `done` is 0, and its last kernel
  // writes beta and r.z, which must not touch the solver's own scalars
  DevBuf<PcgScalars> tsc;
  GIPB_TRY(tsc.alloc(1));
  GIPB_TRY(tsc.zero(s));
  if (amg) GIPB_TRY(amg->reset_tail(s));
  const PackedView pk0 = packed();
  const double plain32 = (double)L->nslots * 8.0 + (L->nslices + 1.0) * 8.0;
  const double a0 = amg ? (cop.enabled ? cop.bytes_per_launch - 16.0 * n : plain32)
                        : (double)L->nslots * 12.0 + (L->nslices + 1.0) * 8.0;
  // The cycle is captured into a graph with an event node before every kernel, so each
  // kernel is timed as a graph launch runs it (no host enqueue gaps between kernels).
  CycleTrace tr;
  tr.captured = true;
  cudaStream_t cs = body_stream[0];
  GIPB_CUDA(cudaStreamSynchronize(s));
  GIPB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  int st = amg ? amg->enqueue(a32(), r32.p, z32.p, tsc.p, rs, 1, cs, &pk0, &tr, a0)
               : amg64->enqueue(L->view(), r.p, z64.p, tsc.p, rs, 1, cs, nullptr, &tr, a0);
  cudaGraph_t g = nullptr;
  cudaError_t ce = cudaStreamEndCapture(cs, &g);
  if (st != GIPB200_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (ce != cudaSuccess) return fail(GIPB200_ERR_CUDA, "capture failed: %s", cudaGetErrorString(ce));
  cudaGraphExec_t ex = nullptr;
  ce = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess)
    return fail(GIPB200_ERR_CUDA, "instantiate failed: %s", cudaGetErrorString(ce));
  const int nk = (int)tr.kind.size();
  std::vector<double> sum((size_t)nk, 0.0);
  for (int k = 0; k <= reps && st == GIPB200_OK; ++k) {  // launch 0 is untimed
    if (cudaGraphLaunch(ex, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
      st = fail(GIPB200_ERR_CUDA, "profiled V-cycle failed");
      break;
    }
    for (int j = 0; j < nk && k > 0; ++j) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, tr.ev[j], tr.ev[j + 1]) != cudaSuccess) {
        st = fail(GIPB200_ERR_CUDA, "cudaEventElapsedTime failed");
        break;
      }
      sum[j] += t;
    }
  }
  cudaGraphExecDestroy(ex);
  GIPB_TRY(st);
  cycle_forms = tr.form;
  *n_kernels = nk;
  for (int j = 0; j < std::min(nk, cap); ++j) {
    if (level) level[j] = tr.level[j];
    if (kind) kind[j] = tr.kind[j];
    if (bytes) bytes[j] = tr.bytes[j];
    if (ms) ms[j] = sum[j] / reps;
  }
  return GIPB200_OK;
}

int Pcg::vcycle_forms(int cap, int* n_kernels, int* h_form) const {
  if (cap < 0 || !n_kernels || (cap > 0 && !h_form)) return fail(GIPB200_ERR_ARG, "bad arguments");
  if (cycle_forms.empty()) return fail(GIPB200_ERR_STATE, "no V-cycle has been profiled");
  *n_kernels = (int)cycle_forms.size();
  for (int k = 0; k < std::min(cap, (int)cycle_forms.size()); ++k) h_form[k] = cycle_forms[(size_t)k];
  return GIPB200_OK;
}

int Pcg::result(cudaStream_t s, gipb200_pcg_result* out) {
  GIPB_CUDA(cudaMemcpyAsync(h_sc, sc.p, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaStreamSynchronize(s));
  if (out) {
    out->iterations = prm.mode == GIPB200_PCG_MIXED ? h_sc->total_inner : h_sc->iter;
    out->outer = h_sc->outer;
    out->status = h_sc->status;
    out->rr = h_sc->rr;
    out->bb = h_sc->bb;
  }
  return GIPB200_OK;
}

}  // namespace gipb200

using namespace gipb200;

extern "C" {

int gipb200_pcg_create(gipb200_matrix L, int n_all, const gipb200_pcg_params* params,
                       gipb200_pcg* out) {
  if (!L || !params || !out) return fail(GIPB200_ERR_ARG, "null argument");
  *out = nullptr;
  gipb200_pcg S = new (std::nothrow) gipb200_pcg_s();
  if (!S) return fail(GIPB200_ERR_NOMEM, "host allocation failed");
  int st = S->P.init(&L->S, n_all, *params, 0);
  if (st != GIPB200_OK) {
    delete S;
    return st;
  }
  *out = S;
  return GIPB200_OK;
}

int gipb200_pcg_destroy(gipb200_pcg S) {
  delete S;
  return GIPB200_OK;
}

int gipb200_check_bounded_wait(void* stream, int* h_status) {
  if (!h_status) return fail(GIPB200_ERR_ARG, "null argument");
  cudaStream_t s = as_stream(stream);
  DevBuf<int> st;
  GIPB_TRY(st.alloc(1));
  k_bounded_wait_check<<<1, 32, 0, s>>>(st.p);
  GIPB_LAUNCH_CHECK();
  GIPB_CUDA(cudaMemcpyAsync(h_status, st.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaStreamSynchronize(s));
  return GIPB200_OK;
}

int gipb200_pcg_get_info(gipb200_pcg S, gipb200_pcg_info* info) {
  if (!S || !info) return fail(GIPB200_ERR_ARG, "null argument");
  info->pin_row = S->P.pin_row;
  info->compressed = S->P.cop.enabled;
  info->value_table = S->P.cop.index_bits;
  info->compressed_fraction = S->P.cop.compressed_fraction;
  const Amg* amg = S->P.amg.get();
  const Amg64* amg64 = S->P.amg64.get();
  info->amg_levels = amg ? (int)amg->lv.size() : amg64 ? (int)amg64->lv.size() : 0;
  info->amg_complexity = amg ? amg->op_complexity : amg64 ? amg64->op_complexity : 0.0;
  info->amg_setup_s = amg ? amg->setup_s : amg64 ? amg64->setup_s : 0.0;
  info->packed_residual = S->P.lpacked ? 1 : 0;
  return GIPB200_OK;
}

int gipb200_pcg_kernel_time(gipb200_pcg S, int reps, void* stream, double* avg_ms,
                            double* bytes) {
  if (!S || !avg_ms || !bytes) return fail(GIPB200_ERR_ARG, "null argument");
  return S->P.time_spmv(S->P.prm.mode == GIPB200_PCG_MIXED, reps, as_stream(stream), avg_ms,
                        bytes);
}

int gipb200_pcg_vcycle_profile(gipb200_pcg S, int reps, void* stream, int cap, int* n_kernels,
                               int* h_level, int* h_kind, double* h_ms, double* h_bytes) {
  if (!S) return fail(GIPB200_ERR_ARG, "null solver");
  return S->P.profile_vcycle(reps, as_stream(stream), cap, n_kernels, h_level, h_kind, h_ms,
                             h_bytes);
}

int gipb200_pcg_vcycle_forms(gipb200_pcg S, int cap, int* n_kernels, int* h_form) {
  if (!S) return fail(GIPB200_ERR_ARG, "null solver");
  return S->P.vcycle_forms(cap, n_kernels, h_form);
}

int gipb200_pcg_solve(gipb200_pcg S, const double* b, double* x, const double* x0, void* stream,
                      gipb200_pcg_result* res) {
  if (!S || !b || !x || !x0) return fail(GIPB200_ERR_ARG, "null argument");
  cudaStream_t s = as_stream(stream);
  GIPB_TRY(S->P.enqueue(b, x, x0, s, true));
  GIPB_TRY(S->P.result(s, res));
  return GIPB200_OK;
}

}  // extern "C"
