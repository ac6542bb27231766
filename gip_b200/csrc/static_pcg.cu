// A Jacobi-PCG solve that allocates nothing: gipb200_pcg_solve_static.
//
// Who needs it: callers that must not allocate device memory at solve time -- code that
// runs inside a host-side memory budget owned by someone else (a framework's caching
// allocator or a fixed arena), callers that solve from a context where cudaMalloc is
// unavailable or forbidden (it synchronises the device and is not allowed during stream
// capture), and embedders that cannot hand out a library handle.  They pass device
// pointers to a CSR operator and to the vectors; the solver's own work vectors and
// reduction scratch live in one file-scope device array of fixed size.
//
// Limits and sharing:
//  - the array holds 4 * kStaticMaxCells doubles (8 MiB) plus reduction scratch; every
//    GPU that loads the library holds it until the process exits;
//  - n_all (vector length, inner plus ghost cells) must not exceed kStaticMaxCells
//    (262144), else the call fails with GIPB200_ERR_ARG before launching anything;
//  - every call uses the same array: two calls whose kernels overlap on the GPU (other
//    streams, other host threads) race and corrupt each other.  Serialise them;
//  - the array keeps the last call's contents; every call clears the reduction counter
//    on its own stream before its first kernel (a 4-byte cudaMemsetAsync, ordered with the
//    caller's work on that stream, non-blocking streams included), and every reduction
//    returns it to zero.
//
// Set-up: the first call on a device (with that device current) resolves the array's
// device address with cudaGetSymbolAddress; make that first call before any stream
// capture.
//
// TOL mode stops on the device; the host polls the stop flag every kPollEvery iterations
// (a 4-byte copy into a host variable and a wait on the caller's stream), so a solve that
// converges early launches about 3 * kPollEvery kernels past convergence, not 3 * maxit.
//
// The arithmetic is the FP64 PCG of GIP_LinearSolver::solve (src/Algorithms/
// GIP_LinearSolver.h:44-117) with GIP's CPU rounding, one thread per CSR row.
#include <math.h>

#include <mutex>

#include "device.cuh"
#include "internal.cuh"

namespace gipb200 {
namespace {

constexpr int kStaticMaxCells = 262144;
constexpr int kPollEvery = 32;     // TOL mode: iterations between host reads of the stop flag
constexpr int kStaticBlocks = 1024;  // grid cap; partials for 3 sums per block
struct StaticScalars {
  double rz, pAp, alpha, beta, rr, bb;
  int iter, done, status, pad;
};
constexpr size_t kScalarSlots = (sizeof(StaticScalars) + 7) / 8;
constexpr size_t kStaticDoubles =
    4 * (size_t)kStaticMaxCells + (size_t)kMaxReduceWidth * kStaticBlocks + kScalarSlots + 32;

// dinv[0:n) | p[0:n_all) | Ap[0:n) | r[0:n) | partials | scalars | ticket
static __device__ __align__(256) double g_static_scratch[kStaticDoubles];

struct StaticLayout {
  double* dinv;
  double* p;
  double* Ap;
  double* r;
  ReduceScratch rs;  // partials stride kMaxReduceBlocks is not used here: see st_reduce
  StaticScalars* S;
};

// Device address of the array per device, resolved once.
struct DeviceSlot {
  bool ready = false;
  double* base = nullptr;
};
std::mutex g_static_mu;
DeviceSlot g_static_dev[64];

// Deterministic grid sum of K values with this file's partial layout
// ([k][kStaticBlocks]); the last block to arrive adds the partials in block order.
template <int K, class Fin>
__device__ __forceinline__ void st_reduce(const double (&v)[K], double* partials, unsigned* ticket,
                                          Fin fin) {
  __shared__ double sh[K][32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double w = warp_reduce<SumOp>(v[k]);
    if (lane == 0) sh[k][warp] = w;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double w = (lane < nwarps) ? sh[k][lane] : 0.0;
      w = warp_reduce<SumOp>(w);
      if (lane == 0) partials[k * kStaticBlocks + blockIdx.x] = w;
    }
  }
  if (threadIdx.x == 0) {
    __threadfence();
    last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double a = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
      a = dadd(a, __ldcg(&partials[k * kStaticBlocks + b]));
    a = warp_reduce<SumOp>(a);
    if (lane == 0) sh[k][warp] = a;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double a = 0.0;
      for (int w = 0; w < nwarps; ++w) a = dadd(a, sh[k][w]);
      tot[k] = a;
    }
    fin(tot);
    *ticket = 0u;
    __threadfence();
  }
}

__device__ __forceinline__ double st_row(const int* __restrict__ rp, const int* __restrict__ col,
                                         const double* __restrict__ val, const double* __restrict__ x,
                                         int i, bool* any) {
  const int jb = rp[i], je = rp[i + 1];
  double sum = 0.0;
  for (int j = jb; j < je; ++j) sum = dadd(sum, dmul(__ldg(x + col[j]), val[j]));
  *any = jb != je;
  return sum;
}

struct StInitFin {
  StaticScalars* S;
  int mode, maxit;
  double tol;
  __device__ void operator()(const double* t) const {
    S->rz = t[0];
    S->rr = t[1];
    S->bb = t[2];
    S->iter = 0;
    S->status = GIPB200_OK;
    S->done = (maxit <= 0) ? 1 : 0;
    if (mode == GIPB200_PCG_TOL && !(sqrt(t[1]) > tol * sqrt(t[2]))) S->done = 1;
  }
};

// dinv = 1/A_ii; r = b - A x (x = x0); z = dinv r; p = z   -- GIP_LinearSolver.h:63-80
__global__ void __launch_bounds__(256) k_st_init(int n, const int* __restrict__ rp,
                                                 const int* __restrict__ col,
                                                 const double* __restrict__ val,
                                                 const double* __restrict__ x,
                                                 const double* __restrict__ b, StaticLayout W,
                                                 unsigned* ticket, int mode, int maxit, double tol) {
  double acc[3] = {0.0, 0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = 0.0;
    for (int j = rp[i]; j < rp[i + 1]; ++j)
      if (col[j] == i) d = ddiv(1.0, val[j]);
    W.dinv[i] = d;
    bool any;
    const double s = st_row(rp, col, val, x, i, &any);
    const double ax = any ? s : x[i];  // GIP's dAx starts as a copy of x0
    W.Ap[i] = ax;
    const double bi = b[i];
    const double ri = dadd(bi, dmul(-1.0, ax));
    const double zi = dadd(0.0, dmul(ri, d));
    W.r[i] = ri;
    W.p[i] = zi;
    acc[0] = dadd(acc[0], dmul(ri, zi));
    acc[1] = dadd(acc[1], dmul(ri, ri));
    acc[2] = dadd(acc[2], dmul(bi, bi));
  }
  st_reduce<3>(acc, W.rs.partials, ticket, StInitFin{W.S, mode, maxit, tol});
}

struct StAlphaFin {
  StaticScalars* S;
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

__global__ void __launch_bounds__(256) k_st_spmv_dot(int n, const int* __restrict__ rp,
                                                     const int* __restrict__ col,
                                                     const double* __restrict__ val, StaticLayout W,
                                                     unsigned* ticket, int mode) {
  if (W.S->done) return;
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    bool any;
    const double s = st_row(rp, col, val, W.p, i, &any);
    const double v = any ? s : W.Ap[i];
    if (any) W.Ap[i] = v;
    acc[0] = dadd(acc[0], dmul(W.p[i], v));
  }
  st_reduce<1>(acc, W.rs.partials, ticket, StAlphaFin{W.S, mode});
}

struct StBetaFin {
  StaticScalars* S;
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

__global__ void __launch_bounds__(256) k_st_update(int n, double* __restrict__ x, StaticLayout W,
                                                   unsigned* ticket, int mode, int maxit,
                                                   double tol) {
  if (W.S->done) return;
  const double alpha = W.S->alpha;
  const double malpha = dmul(-1.0, alpha);
  double acc[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = dadd(x[i], dmul(alpha, W.p[i]));
    const double ri = dadd(W.r[i], dmul(malpha, W.Ap[i]));
    W.r[i] = ri;
    const double zi = dadd(0.0, dmul(ri, W.dinv[i]));
    acc[0] = dadd(acc[0], dmul(ri, zi));
    acc[1] = dadd(acc[1], dmul(ri, ri));
  }
  st_reduce<2>(acc, W.rs.partials, ticket, StBetaFin{W.S, mode, maxit, tol});
}

__global__ void __launch_bounds__(256) k_st_pupdate(int n, StaticLayout W) {
  if (W.S->done) return;
  const double beta = W.S->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double zi = dadd(0.0, dmul(W.r[i], W.dinv[i]));
    W.p[i] = dadd(dmul(1.0, zi), dmul(beta, W.p[i]));
  }
}

__global__ void k_st_stats(const StaticLayout W, double* out) {
  out[0] = (double)W.S->iter;
  out[1] = W.S->rr;
  out[2] = W.S->bb;
  out[3] = (double)W.S->status;
}

}  // namespace
}  // namespace gipb200

using namespace gipb200;

extern "C" int gipb200_pcg_solve_static(int n, int n_all, const int* d_rowptr, const int* d_col,
                                        const double* d_val, const double* d_b, double* d_x,
                                        const double* d_x0, int mode, int maxit, double tol,
                                        double* d_stats, void* stream) {
  if (n < 0 || n_all < n || !d_rowptr || !d_b || !d_x || !d_x0 || !d_stats ||
      (n > 0 && (!d_col || !d_val)))
    return fail(GIPB200_ERR_ARG, "gipb200_pcg_solve_static: bad sizes or null pointer");
  if (n_all > kStaticMaxCells)
    return fail(GIPB200_ERR_ARG,
                "gipb200_pcg_solve_static: n_all=%d exceeds the static scratch limit of %d cells",
                n_all, kStaticMaxCells);
  if (mode != GIPB200_PCG_FIXED && mode != GIPB200_PCG_TOL)
    return fail(GIPB200_ERR_ARG, "gipb200_pcg_solve_static: mode must be FIXED or TOL");
  if (mode == GIPB200_PCG_TOL && !(tol > 0))
    return fail(GIPB200_ERR_ARG, "gipb200_pcg_solve_static: tol must be > 0");
  int dev = 0;
  GIPB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(GIPB200_ERR_ARG, "device index out of range");
  cudaStream_t s = as_stream(stream);
  double* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_static_mu);
    DeviceSlot& slot = g_static_dev[dev];
    if (!slot.ready) {
      void* ptr = nullptr;
      GIPB_CUDA(cudaGetSymbolAddress(&ptr, g_static_scratch));
      slot.base = reinterpret_cast<double*>(ptr);
      slot.ready = true;
    }
    base = slot.base;
  }
  StaticLayout W;
  W.dinv = base;
  W.p = base + kStaticMaxCells;
  W.Ap = base + 2 * (size_t)kStaticMaxCells;
  W.r = base + 3 * (size_t)kStaticMaxCells;
  W.rs.partials = base + 4 * (size_t)kStaticMaxCells;
  W.S = reinterpret_cast<StaticScalars*>(W.rs.partials + (size_t)kMaxReduceWidth * kStaticBlocks);
  unsigned* ticket = reinterpret_cast<unsigned*>(reinterpret_cast<double*>(W.S) + kScalarSlots);
  W.rs.ticket = ticket;

  // the reduction counter starts at zero, ordered on the caller's stream; everything else
  // in the array is written before it is read
  GIPB_CUDA(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s));
  // x = x0 and p = x0 over all cells (GIP_LinearSolver.h:56,67): plain copies, no allocation
  GIPB_CUDA(cudaMemcpyAsync(d_x, d_x0, (size_t)n_all * 8, cudaMemcpyDeviceToDevice, s));
  GIPB_CUDA(cudaMemcpyAsync(W.p, d_x0, (size_t)n_all * 8, cudaMemcpyDeviceToDevice, s));
  int blocks = 1;
  GIPB_TRY(grid_blocks(256, n > 0 ? n : 1, 4, kStaticBlocks, &blocks));
  k_st_init<<<blocks, 256, 0, s>>>(n, d_rowptr, d_col, d_val, d_x, d_b, W, ticket, mode, maxit,
                                   tol);
  GIPB_LAUNCH_CHECK();
  for (int k = 0; k < maxit; ++k) {
    if (mode == GIPB200_PCG_TOL && k > 0 && k % kPollEvery == 0) {
      int done = 0;  // the device's stop flag, read into a host variable (no allocation)
      GIPB_CUDA(cudaMemcpyAsync(&done, &W.S->done, sizeof(int), cudaMemcpyDeviceToHost, s));
      GIPB_CUDA(cudaStreamSynchronize(s));
      if (done) break;
    }
    k_st_spmv_dot<<<blocks, 256, 0, s>>>(n, d_rowptr, d_col, d_val, W, ticket, mode);
    k_st_update<<<blocks, 256, 0, s>>>(n, d_x, W, ticket, mode, maxit, tol);
    k_st_pupdate<<<blocks, 256, 0, s>>>(n, W);
    GIPB_LAUNCH_CHECK();
  }
  k_st_stats<<<1, 1, 0, s>>>(W, d_stats);
  GIPB_LAUNCH_CHECK();
  return GIPB200_OK;
}
