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
    set_loop(use_cond, cond, !S->done);
  }
};

// r = b - L x;  z = dinv r;  p = z;  (rz, rr, bb)   -- GIP_LinearSolver.h:63-80
__global__ void __launch_bounds__(256) k_pcg_init(SellView<double> L, const double* __restrict__ x,
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
__global__ void __launch_bounds__(256) k_pcg_spmv_dot(SellView<double> L,
                                                      const double* __restrict__ p,
                                                      double* __restrict__ Ap, PcgScalars* S,
                                                      ReduceScratch rs, int mode) {
  if (S->done) return;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  double acc[1] = {0.0};
  for (int s = gw; s < L.nslices; s += nw) {
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
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
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
__global__ void __launch_bounds__(256) k_pcg_pupdate(int n, double* __restrict__ p,
                                                     const double* __restrict__ r,
                                                     const double* __restrict__ dinv,
                                                     const PcgScalars* S, int use_cond,
                                                     cudaGraphConditionalHandle cond) {
  if (blockIdx.x == 0 && threadIdx.x == 0) set_loop(use_cond, cond, !S->done);
  if (S->done) return;
  const double beta = S->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double zi = dadd(0.0, dmul(r[i], dinv[i]));
    p[i] = dadd(dmul(1.0, zi), dmul(beta, p[i]));
  }
}

// ------------------------------------------------------------------ MIXED kernels
struct OuterFinish {
  PcgScalars* S;
  double tol, inner_tol;
  int max_outer;
  int pin_row;
  double pin_val;
  const double* scale;
  float* r32;
  float* p32;
  int use_cond;
  cudaGraphConditionalHandle inner_cond;
  __device__ void operator()(const double* t) const {
    // t[0] = r.r (FP64, true residual), t[1] = scaled r^.r^, t[2] = b.b, t[3] = sum(r)
    if (S->outer == 0) S->bb = t[2];
    S->rr = t[0];
    double rz = t[1];
    S->rsum = t[3];
    S->kappa_c = 0.0;
    if (pin_row >= 0) {
      // project the scaled residual: r^_p -= s_p sum(r)
      const float old = __ldcg(r32 + pin_row);
      const float nw = (float)((double)old - scale[pin_row] * t[3]);
      r32[pin_row] = nw;
      p32[pin_row] = nw;
      rz = rz - (double)old * (double)old + (double)nw * (double)nw;
      S->kappa_c = t[3] / pin_val;
    }
    S->rz = rz;
    S->rz_target = rz * inner_tol * inner_tol;
    S->iter = 0;
    const bool conv = !(sqrt(t[0]) > tol * sqrt(S->bb));
    if (conv || S->outer >= max_outer || !isfinite(t[0])) {
      if (!conv) S->status = isfinite(t[0]) ? GIPB200_ERR_NOT_CONVERGED : GIPB200_ERR_BREAKDOWN;
      S->done = 1;
      S->inner_done = 1;
    } else {
      S->outer += 1;
      S->inner_done = 0;
    }
    set_loop(use_cond, inner_cond, !S->inner_done);
  }
};

// r = b - L x (FP64); r^ = S r (FP32); p = r^; y = 0; (r.r, r^.r^, b.b)
__global__ void __launch_bounds__(256) k_mx_residual(SellView<double> L, const double* __restrict__ x,
                                                     const double* __restrict__ b,
                                                     const double* __restrict__ scale,
                                                     double* __restrict__ rtrue,
                                                     float* __restrict__ r32, float* __restrict__ p32,
                                                     float* __restrict__ y32, PcgScalars* S,
                                                     ReduceScratch rs, double tol, double inner_tol,
                                                     int max_outer, int pin_row, double pin_val,
                                                     int use_cond,
                                                     cudaGraphConditionalHandle inner_cond) {
  if (S->done) return;
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
      rtrue[i] = ri;
      const float rh = (float)(ri * scale[i]);
      r32[i] = rh;
      p32[i] = rh;
      y32[i] = 0.f;
      acc[0] += ri * ri;
      acc[1] += (double)rh * (double)rh;
      acc[2] += bi * bi;
      acc[3] += ri;
    }
  }
  grid_reduce<SumOp, 4>(acc, rs,
                        OuterFinish{S, tol, inner_tol, max_outer, pin_row, pin_val, scale, r32, p32,
                                    use_cond, inner_cond});
}

struct AlphaFinish32 {
  PcgScalars* S;
  __device__ void operator()(const double* t) const {
    S->pAp = t[0];
    S->alpha = S->rz / t[0];
    if (!(t[0] > 0.0) || !isfinite(S->alpha)) S->inner_done = 1;  // inner stagnated
  }
};

__global__ void __launch_bounds__(256) k_mx_spmv_dot(SellView<float> A, const float* __restrict__ p,
                                                     float* __restrict__ Ap, PcgScalars* S,
                                                     ReduceScratch rs) {
  if (S->inner_done) return;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  double acc[1] = {0.0};
  for (int s = gw; s < A.nslices; s += nw) {
    const float sum = sell_row_f32(A, p, s, lane);
    const int i = s * 32 + lane;
    if (i < A.nrows) {
      Ap[i] = sum;
      acc[0] += (double)p[i] * (double)sum;
    }
  }
  grid_reduce<SumOp, 1>(acc, rs, AlphaFinish32{S});
}

struct BetaFinish32 {
  PcgScalars* S;
  int inner_maxit;
  __device__ void operator()(const double* t) const {
    const double r0 = S->rz;
    S->rz = t[0];
    S->beta = t[0] / r0;
    S->iter += 1;
    S->total_inner += 1;
    if (!(t[0] > S->rz_target) || S->iter >= inner_maxit) S->inner_done = 1;
  }
};

__global__ void __launch_bounds__(256) k_mx_update(int n, float* __restrict__ y,
                                                   float* __restrict__ r,
                                                   const float* __restrict__ p,
                                                   const float* __restrict__ Ap, PcgScalars* S,
                                                   ReduceScratch rs, int inner_maxit) {
  if (S->inner_done) return;
  const float alpha = (float)S->alpha;
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    y[i] = fmaf(alpha, p[i], y[i]);
    const float ri = fmaf(-alpha, Ap[i], r[i]);
    r[i] = ri;
    acc[0] += (double)ri * (double)ri;
  }
  grid_reduce<SumOp, 1>(acc, rs, BetaFinish32{S, inner_maxit});
}

__global__ void __launch_bounds__(256) k_mx_pupdate(int n, float* __restrict__ p,
                                                    const float* __restrict__ r,
                                                    const PcgScalars* S, int use_cond,
                                                    cudaGraphConditionalHandle inner_cond) {
  if (blockIdx.x == 0 && threadIdx.x == 0) set_loop(use_cond, inner_cond, !S->inner_done);
  if (S->inner_done) return;
  const float beta = (float)S->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = fmaf(beta, p[i], r[i]);
}

// x += S y (+ the exact constant when the pinned-Neumann split is active)
__global__ void __launch_bounds__(256) k_mx_correct(int n, double* __restrict__ x,
                                                    const float* __restrict__ y,
                                                    const double* __restrict__ scale,
                                                    const PcgScalars* S, int pin_row, int use_cond,
                                                    cudaGraphConditionalHandle outer_cond) {
  if (blockIdx.x == 0 && threadIdx.x == 0) set_loop(use_cond, outer_cond, !S->done);
  if (S->done) return;
  const double kappa = (pin_row >= 0) ? S->kappa_c - scale[pin_row] * (double)y[pin_row] : 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] += scale[i] * (double)y[i] + kappa;
}

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
    const long long base = L.sptr[s];
    const int len = (int)((L.sptr[s + 1] - base) >> 5);
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
  if (prm.mode == GIPB200_PCG_MIXED) {
    if (!(prm.inner_tol > 0 && prm.inner_tol < 1)) return fail(GIPB200_ERR_ARG, "inner_tol in (0,1)");
    if (prm.inner_maxit <= 0 || prm.max_outer <= 0) return fail(GIPB200_ERR_ARG, "bad inner caps");
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
    GIPB_TRY(Ap32.alloc(n));
    GIPB_TRY(r32.alloc(n));
    GIPB_TRY(y32.alloc(n));
    GIPB_TRY(rtrue.alloc(n));
    if (n > 0) {
      int b;
      GIPB_TRY(grid_blocks(256, n, 1, 0, &b));
      k_mx_scale<<<b, 256, 0, s>>>(n, L->rowptr.p, L->csr_col.p, L->csr_val.p, scale.p);
      GIPB_LAUNCH_CHECK();
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
      k_mx_lhat<<<blocks_spmv, 256, 0, s>>>(L->view(), scale.p, n, pin_row, pin_val, lhat.p);
      GIPB_LAUNCH_CHECK();
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
  }
  GIPB_CUDA(cudaStreamSynchronize(s));
  return GIPB200_OK;
}

int Pcg::read_flag(cudaStream_t s, int which, int* v) {
  GIPB_CUDA(cudaMemcpyAsync(h_sc, sc.p, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaStreamSynchronize(s));
  *v = which == 0 ? h_sc->done : h_sc->inner_done;
  return GIPB200_OK;
}

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
int Pcg::enqueue_fp64_graph(const double* b, double* x, const double* x0, cudaStream_t s) {
  cudaGraphConditionalHandle h;
  GIPB_TRY(make_handle(s, 0, 0, &h));
  if (x != x0) GIPB_CUDA(cudaMemcpyAsync(x, x0, (size_t)n_all * 8, cudaMemcpyDeviceToDevice, s));
  GIPB_CUDA(cudaMemcpyAsync(p.p, x0, (size_t)n_all * 8, cudaMemcpyDeviceToDevice, s));
  if (n > 0) GIPB_CUDA(cudaMemcpyAsync(Ap.p, x0, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
  k_pcg_init<<<blocks_spmv, 256, 0, s>>>(L->view(), x, b, dinv.p, r.p, p.p, Ap.p, sc.p, rs,
                                          prm.mode, prm.maxit, prm.tol, 1, h);
  GIPB_LAUNCH_CHECK();
  cudaGraph_t body;
  GIPB_TRY(add_while(s, h, &body));
  cudaStream_t bs = body_stream[0];
  GIPB_CUDA(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed));
  k_pcg_spmv_dot<<<blocks_spmv, 256, 0, bs>>>(L->view(), p.p, Ap.p, sc.p, rs, prm.mode);
  k_pcg_update<<<blocks_vec, 256, 0, bs>>>(n, x, r.p, p.p, Ap.p, dinv.p, sc.p, rs, prm.mode,
                                            prm.maxit, prm.tol);
  k_pcg_pupdate<<<blocks_vec, 256, 0, bs>>>(n, p.p, r.p, dinv.p, sc.p, 1, h);
  cudaError_t le = cudaGetLastError();
  cudaGraph_t out = nullptr;
  GIPB_CUDA(cudaStreamEndCapture(bs, &out));
  if (le != cudaSuccess) return fail(GIPB200_ERR_CUDA, "launch in loop body: %s", cudaGetErrorString(le));
  launches += 4;
  return GIPB200_OK;
}

// MIXED inside a graph:
//   while(!done) { residual (sets done / inner_done); while(!inner_done) { A; B; C };
//                  correct (sets the outer loop value) }
int Pcg::enqueue_mixed_graph(const double* b, double* x, const double* x0, cudaStream_t s) {
  cudaGraphConditionalHandle ho;
  GIPB_TRY(make_handle(s, 1, cudaGraphCondAssignDefault, &ho));
  if (x != x0) GIPB_CUDA(cudaMemcpyAsync(x, x0, (size_t)n_all * 8, cudaMemcpyDeviceToDevice, s));
  GIPB_CUDA(cudaMemsetAsync(sc.p, 0, sizeof(PcgScalars), s));
  cudaGraph_t outer_body;
  GIPB_TRY(add_while(s, ho, &outer_body));
  const SellView<float> A{L->nrows, L->nslices, L->sptr.p, L->col.p, lhat.p};
  cudaStream_t os = body_stream[0], is = body_stream[1];
  GIPB_CUDA(cudaStreamBeginCaptureToGraph(os, outer_body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed));
  int st = [&]() -> int {
    cudaGraphConditionalHandle hi;
    GIPB_TRY(make_handle(os, 0, 0, &hi));
    k_mx_residual<<<blocks_spmv, 256, 0, os>>>(L->view(), x, b, scale.p, rtrue.p, r32.p, p32.p,
                                                y32.p, sc.p, rs, prm.tol, prm.inner_tol,
                                                prm.max_outer, pin_row, pin_val, 1, hi);
    GIPB_LAUNCH_CHECK();
    cudaGraph_t inner_body;
    GIPB_TRY(add_while(os, hi, &inner_body));
    GIPB_CUDA(cudaStreamBeginCaptureToGraph(is, inner_body, nullptr, nullptr, 0,
                                            cudaStreamCaptureModeRelaxed));
    k_mx_spmv_dot<<<blocks_spmv, 256, 0, is>>>(A, p32.p, Ap32.p, sc.p, rs);
    k_mx_update<<<blocks_vec, 256, 0, is>>>(n, y32.p, r32.p, p32.p, Ap32.p, sc.p, rs,
                                             prm.inner_maxit);
    k_mx_pupdate<<<blocks_vec, 256, 0, is>>>(n, p32.p, r32.p, sc.p, 1, hi);
    cudaError_t le = cudaGetLastError();
    cudaGraph_t out = nullptr;
    GIPB_CUDA(cudaStreamEndCapture(is, &out));
    if (le != cudaSuccess)
      return fail(GIPB200_ERR_CUDA, "launch in inner body: %s", cudaGetErrorString(le));
    k_mx_correct<<<blocks_vec, 256, 0, os>>>(n, x, y32.p, scale.p, sc.p, pin_row, 1, ho);
    GIPB_LAUNCH_CHECK();
    return GIPB200_OK;
  }();
  cudaGraph_t out = nullptr;
  cudaError_t ce = cudaStreamEndCapture(os, &out);
  if (st != GIPB200_OK) return st;
  if (ce != cudaSuccess) return fail(GIPB200_ERR_CUDA, "outer body capture: %s", cudaGetErrorString(ce));
  launches += 5;
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
  const int poll = 16;
  for (int k = 0; k < prm.maxit; ++k) {
    k_pcg_spmv_dot<<<blocks_spmv, 256, 0, s>>>(L->view(), p.p, Ap.p, sc.p, rs, prm.mode);
    k_pcg_update<<<blocks_vec, 256, 0, s>>>(n, x, r.p, p.p, Ap.p, dinv.p, sc.p, rs, prm.mode,
                                             prm.maxit, prm.tol);
    k_pcg_pupdate<<<blocks_vec, 256, 0, s>>>(n, p.p, r.p, dinv.p, sc.p, 0, 0);
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

int Pcg::enqueue_mixed(const double* b, double* x, const double* x0, cudaStream_t s,
                       bool host_sync) {
  if (x != x0) GIPB_CUDA(cudaMemcpyAsync(x, x0, (size_t)n_all * 8, cudaMemcpyDeviceToDevice, s));
  GIPB_CUDA(cudaMemsetAsync(sc.p, 0, sizeof(PcgScalars), s));
  const SellView<float> A{L->nrows, L->nslices, L->sptr.p, L->col.p, lhat.p};
  const int poll = 16;
  for (int o = 0; o <= prm.max_outer; ++o) {
    k_mx_residual<<<blocks_spmv, 256, 0, s>>>(L->view(), x, b, scale.p, rtrue.p, r32.p, p32.p,
                                               y32.p, sc.p, rs, prm.tol, prm.inner_tol,
                                               prm.max_outer, pin_row, pin_val, 0, 0);
    GIPB_LAUNCH_CHECK();
    launches += 1;
    if (host_sync) {
      int d;
      GIPB_TRY(read_flag(s, 0, &d));
      if (d) break;
    }
    for (int k = 0; k < prm.inner_maxit; ++k) {
      k_mx_spmv_dot<<<blocks_spmv, 256, 0, s>>>(A, p32.p, Ap32.p, sc.p, rs);
      k_mx_update<<<blocks_vec, 256, 0, s>>>(n, y32.p, r32.p, p32.p, Ap32.p, sc.p, rs,
                                              prm.inner_maxit);
      k_mx_pupdate<<<blocks_vec, 256, 0, s>>>(n, p32.p, r32.p, sc.p, 0, 0);
      GIPB_LAUNCH_CHECK();
      launches += 3;
      if (host_sync && (k + 1) % poll == 0) {
        int d;
        GIPB_TRY(read_flag(s, 1, &d));
        if (d) break;
      }
    }
    k_mx_correct<<<blocks_vec, 256, 0, s>>>(n, x, y32.p, scale.p, sc.p, pin_row, 0, 0);
    GIPB_LAUNCH_CHECK();
    launches += 1;
  }
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
  DevBuf<float> tAp32;
  DevBuf<double> tAp;
  cudaEvent_t e0, e1;
  GIPB_CUDA(cudaEventCreate(&e0));
  GIPB_CUDA(cudaEventCreate(&e1));
  const SellView<float> A{L->nrows, L->nslices, L->sptr.p, L->col.p, lhat.p};
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
      k_mx_spmv_dot<<<blocks_spmv, 256, 0, s>>>(A, p32.p, tAp32.p, tsc.p, rs);
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
  const double vbytes = mixed ? 4.0 : 8.0;
  *bytes = (double)L->nnz * (vbytes + 4.0) + (double)(L->nslices + 1) * 8.0 +
           (double)L->nrows * 2.0 * vbytes;
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

int gipb200_pcg_solve(gipb200_pcg S, const double* b, double* x, const double* x0, void* stream,
                      gipb200_pcg_result* res) {
  if (!S || !b || !x || !x0) return fail(GIPB200_ERR_ARG, "null argument");
  cudaStream_t s = as_stream(stream);
  GIPB_TRY(S->P.enqueue(b, x, x0, s, true));
  GIPB_TRY(S->P.result(s, res));
  return GIPB200_OK;
}

}  // extern "C"
