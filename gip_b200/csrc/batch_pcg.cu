// Persistent mixed-precision Jacobi-PCG over a batch of independent pressure systems.
//
// One cooperative launch solves every instance of the batch.  Its CTAs are split into
// groups, one per instance, sized by the instance's share of the work (rows times the
// iterations it is expected to need).  A group runs its instance's whole solve: the
// reliable-update mixed CG of the single-instance engine (pcg.cu) -- an FP32 CG on the
// Jacobi-scaled operator S L S with the pinned-Neumann split, whose FP32 residual is
// replaced by the FP64 true residual r = b - L x whenever it has fallen by the factor
// delta -- and leaves the kernel when its instance has converged.  That exit is the
// per-instance convergence mask: a converged instance costs nothing further, and groups
// never wait on one another.
//
// Within a group, phases are separated by a group barrier: an arrival counter in global
// memory that each CTA increments after a fence and spins on (with a bounded wait; a wait
// that gives up sets the batch's error word and the CTA leaves).  Every reduction is
// deterministic and needs no second barrier: each CTA writes its block partial, and after
// the barrier every CTA sums the group's partials in CTA order, so all CTAs of a group hold
// bit-identical scalars and take the same branches.  Two partial buffers alternate, so a
// CTA that runs ahead never overwrites partials another CTA is still reading.  Vectors the
// launch itself writes are read through L2 (ld.global.cg), the operators through the
// streaming path.
//
// GIP's solver that this replaces for a batch is GIP_LinearSolver::solve
// (src/Algorithms/GIP_LinearSolver.h:44-117), run once per instance.
#include <algorithm>

#include "batch_pcg.cuh"
#include "device.cuh"

namespace gipb200 {
namespace {

constexpr long long kSpinCycles = 4000000000LL;  // about 2 s of SM clock

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

struct Group {
  unsigned* bar;
  double* part;
  int rank, ncta;
  unsigned epoch;
  int parity;
};

// All CTAs of the group have arrived, and their earlier writes are visible.  False in
// every thread of the CTA when the wait gave up.
__device__ bool group_sync(Group& G, int* s_ok) {
  __syncthreads();
  G.epoch += 1u;
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(G.bar, 1u);
    const unsigned target = G.epoch * (unsigned)G.ncta;
    const long long t0 = clock64();
    int ok = 1;
    while (ld_acquire(G.bar) < target) {
      if (clock64() - t0 > kSpinCycles) {
        ok = 0;
        break;
      }
    }
    __threadfence();
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

// W sums over the CTA; every thread receives the totals (warp sums added in warp order).
template <int W>
__device__ __forceinline__ void block_sum(double (&v)[W], double (*sh)[32]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < W; ++k) {
    const double t = warp_reduce<SumOp>(v[k]);
    if (lane == 0) sh[k][warp] = t;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < W; ++k) {
    double a = 0.0;
    for (int i = 0; i < nw; ++i) a = dadd(a, sh[k][i]);
    v[k] = a;
  }
  __syncthreads();
}

// W sums over the group: the same totals in every CTA (CTA partials added in rank order).
template <int W>
__device__ bool group_sum(double (&v)[W], Group& G, double (*sh)[32], int* s_ok) {
  static_assert(W <= kBatchWidth, "too many sums");
  block_sum<W>(v, sh);
  double* part = G.part + (size_t)G.parity * kBatchWidth * kBatchGroupMax;
  G.parity ^= 1;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < W; ++k) part[k * kBatchGroupMax + G.rank] = v[k];
  }
  if (!group_sync(G, s_ok)) return false;
#pragma unroll
  for (int k = 0; k < W; ++k) {
    double a = 0.0;
    for (int c = threadIdx.x; c < G.ncta; c += blockDim.x)
      a = dadd(a, __ldcg(part + k * kBatchGroupMax + c));
    v[k] = a;
  }
  block_sum<W>(v, sh);
  return true;
}

// Rows of SPW slices of the FP64 operator times x (x written inside the launch, so read
// through L2), each summed slot by slot with GIP's rounding.  The slices' slot loads, then
// their gathers, are issued together (four per lane in flight).
template <int SPW>
__device__ __forceinline__ void rows_l(const SellView<double>& L, const double* x,
                                       const int (&s)[SPW], int lane, double (&sum)[SPW]) {
  long long base[SPW];
  int len[SPW], lmax = 0;
#pragma unroll
  for (int u = 0; u < SPW; ++u) {
    sum[u] = 0.0;
    base[u] = 0;
    len[u] = 0;
    if (s[u] < L.nslices) {
      slice_range(L, s[u], base[u], len[u]);
    }
    lmax = max(lmax, len[u]);
  }
  constexpr int CH = 4 / SPW;  // slots per slice per pass: four gathers in flight per lane
  for (int j0 = 0; j0 < lmax; j0 += CH) {
    int c[SPW][CH];
    double v[SPW][CH], xv[SPW][CH];
#pragma unroll
    for (int u = 0; u < SPW; ++u)
#pragma unroll
      for (int t = 0; t < CH; ++t) {
        const bool in = j0 + t < len[u];
        c[u][t] = in ? ld_stream(L.col + base[u] + 32LL * (j0 + t) + lane) : -1;
        v[u][t] = in ? ld_stream(L.val + base[u] + 32LL * (j0 + t) + lane) : 0.0;
      }
#pragma unroll
    for (int u = 0; u < SPW; ++u)
#pragma unroll
      for (int t = 0; t < CH; ++t) xv[u][t] = (c[u][t] >= 0) ? __ldcg(x + c[u][t]) : 0.0;
#pragma unroll
    for (int u = 0; u < SPW; ++u)
#pragma unroll
      for (int t = 0; t < CH; ++t)
        if (c[u][t] >= 0) sum[u] = dadd(sum[u], dmul(xv[u][t], v[u][t]));
  }
}

// Rows of SPW slices of the FP32 operator times the new direction p = r + beta p_in, formed
// on the fly from the gathered r and p_in (the single-instance kernel's FMA order).
template <int SPW>
__device__ __forceinline__ void rows_dir(const SellView<float>& A, const float* r,
                                         const float* pin, float beta, const int (&s)[SPW],
                                         int lane, float (&sum)[SPW]) {
  long long base[SPW];
  int len[SPW], lmax = 0;
#pragma unroll
  for (int u = 0; u < SPW; ++u) {
    sum[u] = 0.f;
    base[u] = 0;
    len[u] = 0;
    if (s[u] < A.nslices) {
      slice_range(A, s[u], base[u], len[u]);
    }
    lmax = max(lmax, len[u]);
  }
  constexpr int CH = 4 / SPW;
  for (int j0 = 0; j0 < lmax; j0 += CH) {
    int c[SPW][CH];
    float v[SPW][CH], xv[SPW][CH];
#pragma unroll
    for (int u = 0; u < SPW; ++u)
#pragma unroll
      for (int t = 0; t < CH; ++t) {
        const bool in = j0 + t < len[u];
        c[u][t] = in ? ld_stream(A.col + base[u] + 32LL * (j0 + t) + lane) : -1;
        v[u][t] = in ? ld_stream(A.val + base[u] + 32LL * (j0 + t) + lane) : 0.f;
      }
#pragma unroll
    for (int u = 0; u < SPW; ++u)
#pragma unroll
      for (int t = 0; t < CH; ++t)
        xv[u][t] = (c[u][t] >= 0) ? fmaf(beta, __ldcg(pin + c[u][t]), __ldcg(r + c[u][t])) : 0.f;
#pragma unroll
    for (int u = 0; u < SPW; ++u)
#pragma unroll
      for (int t = 0; t < CH; ++t) sum[u] = fmaf(xv[u][t], v[u][t], sum[u]);
  }
}

// One slice's rows of the packed FP32 operator times p = r + beta p_in, in the FMA order
// of the single-instance packed kernel (all eight slots: an unused eighth slot adds
// x * 0.0f, which leaves the sum unchanged); slices stored plain use the sliced layout.
template <int NIB>
__device__ __forceinline__ float row_dir_packed(const BatchSolve& B, const float* tab,
                                                const float* r, const float* pin, float beta,
                                                int s, int lane) {
  PackedWords w;
  packed_words<NIB>(B.pk_delta, B.pk_idx, B.pk_plain, s, lane, w);
  int c[8];
  packed_cols(B.pk_base, s, w.d, c);
  if (w.plain) {
    const int ss[1] = {s};
    float sm[1];
    rows_dir<1>(B.A, r, pin, beta, ss, lane, sm);
    return sm[0];
  }
  float xv[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) xv[j] = fmaf(beta, __ldcg(pin + c[j]), __ldcg(r + c[j]));
  float sum = 0.f;
#pragma unroll
  for (int j = 0; j < 8; ++j) sum = fmaf(xv[j], tab[packed_index<NIB>(w, j)], sum);
  return sum;
}

__device__ __forceinline__ float pick(const float4& a, int k) {
  return k == 0 ? a.x : k == 1 ? a.y : k == 2 ? a.z : a.w;
}

// The solve's scalars, in shared memory: thread 0 updates them from the group sums (which
// every CTA of the group holds identically), the other threads read them after a barrier.
struct SolveState {
  double rz, beta, alpha, pAp, bb, rr, maxr2, trig, kappa_c, kappa;
  int total, outer, status, done, upd;
};

// r = b - L x rows (FP64), r^ = S r (FP32); first: p = r^, y = 0.  acc: r.r, r^.r^, b.b,
// sum(r), the pinned row's r^ (exact through the sums of zeros).
template <int SPW>
__device__ __forceinline__ void residual_rows(const BatchSolve& B, int first, int gw, int nw,
                                              double (&acc)[5]) {
  const int lane = threadIdx.x & 31;
  for (int s0 = gw; s0 < B.L.nslices; s0 += SPW * nw) {
    int s[SPW];
#pragma unroll
    for (int u = 0; u < SPW; ++u) s[u] = s0 + u * nw;
    double sum[SPW];
    rows_l<SPW>(B.L, B.x, s, lane, sum);
#pragma unroll
    for (int u = 0; u < SPW; ++u) {
      const int i = s[u] * 32 + lane;
      if (s[u] < B.L.nslices && i < B.n) {
        const double bi = B.b[i];
        const double ri = bi - sum[u];
        const float rh = (float)(ri * B.scale[i]);
        B.r[i] = rh;
        if (first) {
          B.p[0][i] = rh;
          B.y[i] = 0.f;
        }
        acc[0] += ri * ri;
        acc[1] += (double)rh * (double)rh;
        acc[2] += bi * bi;
        acc[3] += ri;
        if (i == B.pin_row) acc[4] = rh;
      }
    }
  }
}

// Thread 0: the residual's scalars (the single-instance engine's residual finish) and the
// pinned entry's adjustment.
__device__ __forceinline__ void residual_finish(const BatchSolve& B, SolveState& T, int first,
                                                int rank, const double (&t)[5]) {
  if (first) T.bb = t[2];
  T.rr = t[0];
  double rzl = t[1];
  T.kappa_c = 0.0;
  const int pin = B.pin_row;
  if (pin >= 0) {
    const float old = (float)t[4];
    const float nwv = (float)((double)old - B.scale[pin] * t[3]);
    if (rank == 0) {
      B.r[pin] = nwv;
      if (first) B.p[0][pin] = nwv;
    }
    rzl = rzl - (double)old * (double)old + (double)nwv * (double)nwv;
    T.kappa_c = t[3] / B.pin_val;
  }
  if (!first) {
    T.beta = rzl / T.rz;  // continue the direction with the replaced residual
    T.outer += 1;
  }
  T.rz = rzl;
  T.maxr2 = rzl;
  const double goal = 0.5 * B.tol * sqrt(T.bb);
  T.trig = (t[0] > 0.0) ? rzl * (goal * goal) / t[0] : 0.0;
  const bool finite = isfinite(t[0]) && isfinite(T.bb);
  const bool conv = finite && !(sqrt(t[0]) > B.tol * sqrt(T.bb));
  if (conv || !finite || T.total >= B.maxit || T.outer >= B.max_outer) {
    if (!conv) T.status = finite ? GIPB200_ERR_NOT_CONVERGED : GIPB200_ERR_BREAKDOWN;
    T.done = 1;
  }
}

template <int BS, int SPW, int OCC>
__global__ void __launch_bounds__(BS, OCC / BS) k_batch_pcg(const BatchSolve* __restrict__ inst,
                                                             const int* __restrict__ owner,
                                                             int* __restrict__ err) {
  __shared__ BatchSolve B;
  __shared__ SolveState T;
  __shared__ double sh[kBatchWidth][32];
  __shared__ float tab[256];  // the packed operator's value table
  __shared__ int s_ok;
  const int g = owner[blockIdx.x];
  if (g < 0) return;  // an idle CTA (the groups do not fill the grid)
  if (threadIdx.x == 0) {
    B = inst[g];
    T = SolveState{};
    T.status = GIPB200_OK;
  }
  __syncthreads();
  if (B.pk_nib)
    for (int t = threadIdx.x; t < (1 << B.pk_nib); t += BS) tab[t] = B.pk_table[t];
  Group G{B.bar, B.part, (int)blockIdx.x - B.cta0, B.ncta, 0u, 0};
  const int lane = threadIdx.x & 31;
  const int gw = G.rank * (BS / 32) + (threadIdx.x >> 5), nw = G.ncta * (BS / 32);
  const int gt = G.rank * BS + threadIdx.x, nt = G.ncta * BS;
  const bool lead = threadIdx.x == 0;

  // r = b - L x with the pin split; false when a barrier gave up
  auto residual = [&](int first) -> bool {
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    residual_rows<1>(B, first, gw, nw, acc);  // rare (replacements): one slice a pass
    if (!group_sum<5>(acc, G, sh, &s_ok)) return false;
    if (lead) residual_finish(B, T, first, G.rank, acc);
    __syncthreads();
    // the adjusted pinned entry is written before any CTA gathers it
    if (B.pin_row >= 0 && !group_sync(G, &s_ok)) return false;
    return true;
  };

  bool ok = true;
  if (B.x != B.x0)
    for (int i = gt; i < B.n_all; i += nt) B.x[i] = __ldg(B.x0 + i);
  ok = group_sync(G, &s_ok) && residual(1);
  for (int k = 0; ok && !T.done; ++k) {
    const float* pin_v = B.p[k & 1];
    float* pout = B.p[(k & 1) ^ 1];
    // Ap = A^ p, p = r^ + beta p_in, p.Ap  -> alpha
    {
      const float bf = (float)T.beta;
      double acc[1] = {0.0};
      const int nib = B.pk_nib;
      for (int s0 = gw; s0 < B.A.nslices; s0 += SPW * nw) {
        int s[SPW];
#pragma unroll
        for (int u = 0; u < SPW; ++u) s[u] = s0 + u * nw;
        float sum[SPW];
        if (nib == 4) {
#pragma unroll
          for (int u = 0; u < SPW; ++u)
            sum[u] = s[u] < B.A.nslices ? row_dir_packed<4>(B, tab, B.r, pin_v, bf, s[u], lane) : 0.f;
        } else if (nib == 8) {
#pragma unroll
          for (int u = 0; u < SPW; ++u)
            sum[u] = s[u] < B.A.nslices ? row_dir_packed<8>(B, tab, B.r, pin_v, bf, s[u], lane) : 0.f;
        } else {
          rows_dir<SPW>(B.A, B.r, pin_v, bf, s, lane, sum);
        }
#pragma unroll
        for (int u = 0; u < SPW; ++u) {
          const int i = s[u] * 32 + lane;
          if (s[u] < B.A.nslices && i < B.n) {
            const float pi = fmaf(bf, __ldcg(pin_v + i), __ldcg(B.r + i));
            pout[i] = pi;
            B.Ap[i] = sum[u];
            acc[0] += (double)pi * (double)sum[u];
          }
        }
      }
      if (!(ok = group_sum<1>(acc, G, sh, &s_ok))) break;
      if (lead) {
        T.pAp = acc[0];
        T.alpha = T.rz / acc[0];
        if (!(acc[0] > 0.0) || !isfinite(T.alpha)) T.alpha = 0.0;  // direction lost: replace
      }
      __syncthreads();
    }
    // y += alpha p, r^ -= alpha Ap, r^.r^  -> beta or a replacement
    {
      const float af = (float)T.alpha;
      const int n = B.n, pin = B.pin_row;
      double acc[2] = {0.0, 0.0};
      const int n4 = n >> 2;
      float4* y4 = reinterpret_cast<float4*>(B.y);
      float4* r4 = reinterpret_cast<float4*>(B.r);
      const float4* p4 = reinterpret_cast<const float4*>(pout);
      const float4* a4 = reinterpret_cast<const float4*>(B.Ap);
      for (int q = gt; q < n4; q += nt) {
        float4 yv = __ldcg(y4 + q), rv = __ldcg(r4 + q);
        const float4 pv = __ldcg(p4 + q), av = __ldcg(a4 + q);
        yv.x = fmaf(af, pv.x, yv.x);
        yv.y = fmaf(af, pv.y, yv.y);
        yv.z = fmaf(af, pv.z, yv.z);
        yv.w = fmaf(af, pv.w, yv.w);
        rv.x = fmaf(-af, av.x, rv.x);
        rv.y = fmaf(-af, av.y, rv.y);
        rv.z = fmaf(-af, av.z, rv.z);
        rv.w = fmaf(-af, av.w, rv.w);
        y4[q] = yv;
        r4[q] = rv;
        acc[0] += (double)rv.x * (double)rv.x + (double)rv.y * (double)rv.y +
                  (double)rv.z * (double)rv.z + (double)rv.w * (double)rv.w;
        if ((unsigned)(pin - 4 * q) < 4u) acc[1] = pick(yv, pin - 4 * q);
      }
      for (int i = 4 * n4 + gt; i < n; i += nt) {
        const float yi = fmaf(af, __ldcg(pout + i), __ldcg(B.y + i));
        const float ri = fmaf(-af, __ldcg(B.Ap + i), __ldcg(B.r + i));
        B.y[i] = yi;
        B.r[i] = ri;
        acc[0] += (double)ri * (double)ri;
        if (i == pin) acc[1] = yi;
      }
      if (!(ok = group_sum<2>(acc, G, sh, &s_ok))) break;
      if (lead) {
        T.total += 1;
        const double rzn = acc[0];
        if (rzn > T.maxr2) T.maxr2 = rzn;
        T.upd = !(rzn > T.trig) || !(rzn > B.delta * B.delta * T.maxr2) || T.alpha == 0.0 ||
                T.total >= B.maxit || !isfinite(rzn);
        if (T.upd) {
          T.kappa = (pin >= 0) ? T.kappa_c - B.scale[pin] * acc[1] : 0.0;
        } else {
          T.beta = rzn / T.rz;
          T.rz = rzn;
        }
      }
      __syncthreads();
    }
    if (!T.upd) continue;
    // replacement: x += S y + kappa, y = 0, then the FP64 true residual
    {
      const double kappa = T.kappa;
      for (int i = gt; i < B.n; i += nt) {
        B.x[i] = __ldcg(B.x + i) + (B.scale[i] * (double)__ldcg(B.y + i) + kappa);
        B.y[i] = 0.f;
      }
    }
    if (!(ok = group_sync(G, &s_ok))) break;
    ok = residual(0);
  }
  if (!ok && lead) {
    T.status = GIPB200_ERR_TIMEOUT;
    atomicExch(err, 1);
  }
  if (G.rank == 0 && lead) {
    PcgScalars* S = B.S;
    S->rz = T.rz;
    S->pAp = T.pAp;
    S->alpha = T.alpha;
    S->beta = T.beta;
    S->rr = T.rr;
    S->bb = T.bb;
    S->iter = T.total;
    S->done = 1;
    S->inner_done = 1;
    S->status = T.status;
    S->outer = T.outer;
    S->total_inner = T.total;
    S->kernels = B.count_launch;
    S->kappa_c = T.kappa_c;
    S->kappa = T.kappa;
    S->maxr2 = T.maxr2;
    S->trig = T.trig;
    S->upd = 0;
  }
}

template <int BS, int SPW, int OCC>
int launch_variant(int grid, const BatchSolve* inst, const int* owner, int* err, cudaStream_t s,
                   int* capacity) {
  auto kern = k_batch_pcg<BS, SPW, OCC>;
  if (capacity) {
    DeviceInfo di;
    GIPB_TRY(device_info(&di));
    int per_sm = 0;
    GIPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BS, 0));
    *capacity = per_sm * di.nsm;
    return GIPB200_OK;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(BS);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  GIPB_CUDA(cudaLaunchKernelEx(&cfg, kern, inst, owner, err));
  return GIPB200_OK;
}

int dispatch(const BatchShape& sh, int grid, const BatchSolve* inst, const int* owner, int* err,
             cudaStream_t s, int* capacity) {
  const int spw = sh.rows_per_warp / 32;
  const int key = (sh.threads_per_sm == 1536 ? 100000 : 0) + sh.block * 4 + spw;
#define GIPB_BP(BS, SPW, OCC) \
  case (OCC == 1536 ? 100000 : 0) + BS * 4 + SPW: \
    return launch_variant<BS, SPW, OCC>(grid, inst, owner, err, s, capacity)
  switch (key) {
    GIPB_BP(128, 1, 1024);
    GIPB_BP(128, 2, 1024);
    GIPB_BP(256, 1, 1024);
    GIPB_BP(256, 2, 1024);
    GIPB_BP(512, 1, 1024);
    GIPB_BP(512, 2, 1024);
    GIPB_BP(128, 1, 1536);
    GIPB_BP(128, 2, 1536);
    GIPB_BP(256, 1, 1536);
    GIPB_BP(256, 2, 1536);
    GIPB_BP(512, 1, 1536);
    GIPB_BP(512, 2, 1536);
    default:
      return fail(GIPB200_ERR_ARG,
                  "unsupported batch shape: block %d, rows per warp %d, threads per SM %d",
                  sh.block, sh.rows_per_warp, sh.threads_per_sm);
  }
#undef GIPB_BP
}

}  // namespace

// One CTA whose group claims two: its first barrier waits for a CTA that does not exist and
// gives up after the bounded spin.
int batch_pcg_check_timeout(cudaStream_t s, int* h_status) {
  DevBuf<BatchSolve> inst;
  DevBuf<int> owner, err;
  DevBuf<unsigned> bar;
  DevBuf<double> part;
  DevBuf<PcgScalars> sc;
  GIPB_TRY(inst.alloc(1));
  GIPB_TRY(owner.alloc(1));
  GIPB_TRY(err.alloc(1));
  GIPB_TRY(bar.alloc(1));
  GIPB_TRY(part.alloc((size_t)2 * kBatchWidth * kBatchGroupMax));
  GIPB_TRY(sc.alloc(1));
  GIPB_TRY(err.zero(s));
  GIPB_TRY(bar.zero(s));
  GIPB_TRY(sc.zero(s));
  BatchSolve h{};
  h.S = sc.p;
  h.part = part.p;
  h.bar = bar.p;
  h.pin_row = -1;
  h.cta0 = 0;
  h.ncta = 2;
  const int o = 0;
  GIPB_CUDA(cudaMemcpyAsync(inst.p, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  GIPB_CUDA(cudaMemcpyAsync(owner.p, &o, sizeof(int), cudaMemcpyHostToDevice, s));
  BatchShape sh;
  GIPB_TRY(batch_pcg_launch(sh, 1, inst.p, owner.p, err.p, s));
  int e = 0;
  PcgScalars r{};
  GIPB_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaMemcpyAsync(&r, sc.p, sizeof(r), cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaStreamSynchronize(s));
  *h_status = (e != 0 && r.status == GIPB200_ERR_TIMEOUT) ? GIPB200_ERR_TIMEOUT : GIPB200_OK;
  return GIPB200_OK;
}

bool batch_shape_valid(const BatchShape& sh) {
  return (sh.block == 128 || sh.block == 256 || sh.block == 512) &&
         (sh.rows_per_warp == 32 || sh.rows_per_warp == 64) &&
         (sh.threads_per_sm == 1024 || sh.threads_per_sm == 1536);
}

int batch_pcg_capacity(const BatchShape& sh, int* ctas) {
  return dispatch(sh, 0, nullptr, nullptr, nullptr, nullptr, ctas);
}

int batch_pcg_launch(const BatchShape& sh, int grid, const BatchSolve* inst, const int* owner,
                     int* err, cudaStream_t s) {
  if (grid <= 0) return fail(GIPB200_ERR_ARG, "empty persistent grid");
  return dispatch(sh, grid, inst, owner, err, s, nullptr);
}

}  // namespace gipb200
