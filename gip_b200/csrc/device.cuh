// Device-side building blocks: exact FP64 arithmetic, warp/block/grid reductions and
// the sliced-ELL row kernel.
#pragma once

#include <cuda_runtime.h>

#include "internal.cuh"

namespace gipb200 {

// GIP's CPU loops round every product and every sum (no FMA contraction); these keep the
// same IEEE operations on the device.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// Start of a kernel that may be launched dependent on its predecessor: wait for the
// predecessor's completion (a no-op for an ordinary launch), then let the next kernel in
// the stream be scheduled.
__device__ __forceinline__ void dep_begin() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename T>
__device__ __forceinline__ T ld_stream(const T* p) {
  return __ldcs(p);
}

// Asynchronous prefetch of `bytes` (a multiple of 16, 16-byte aligned) into L2.
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

struct SumOp {
  __device__ static double identity() { return 0.0; }
  __device__ static double apply(double a, double b) { return dadd(a, b); }
};
struct MaxOp {  // of non-negative values (infinity norm)
  __device__ static double identity() { return 0.0; }
  __device__ static double apply(double a, double b) { return (b > a) ? b : a; }
};
struct MinOp {
  __device__ static double identity() { return 1e20; }
  __device__ static double apply(double a, double b) { return (b < a) ? b : a; }
};

template <class Op>
__device__ __forceinline__ double warp_reduce(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = Op::apply(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Reduces K values per thread over the grid.  Every block writes its K partials; the
// last block to finish reduces them in block order and calls fin(total[]) on thread 0.
// Returns true in the block that ran fin (all its threads).
template <class Op, int K, class Fin>
__device__ __forceinline__ bool grid_reduce(const double (&v)[K], ReduceScratch rs, Fin fin) {
  __shared__ double sh[K][32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double w = warp_reduce<Op>(v[k]);
    if (lane == 0) sh[k][warp] = w;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double w = (lane < nwarps) ? sh[k][lane] : Op::identity();
      w = warp_reduce<Op>(w);
      if (lane == 0) rs.partials[k * kMaxReduceBlocks + blockIdx.x] = w;
    }
  }
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned t = atomicAdd(rs.ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double tot[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double a = Op::identity();
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
      a = Op::apply(a, __ldcg(&rs.partials[k * kMaxReduceBlocks + b]));
    a = warp_reduce<Op>(a);
    if (lane == 0) sh[k][warp] = a;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double a = Op::identity();
      for (int w = 0; w < nwarps; ++w) a = Op::apply(a, sh[k][w]);
      tot[k] = a;
    }
    fin(tot);
    *rs.ticket = 0u;
    __threadfence();
  }
  return true;
}

// ------------------------------------------------------------------ packed FP32 rows
// The mixed form's compressed operator: per row one 16-byte word of eight 16-bit column
// deltas from per-(slice, slot) int32 bases, and eight value-table indices (4 or 8 bits).
// (Loading a slice's words one slice ahead of their use measured slower at the 32
// registers these kernels keep for full occupancy: 147.7 against 138.6 us per CG SpMV-dot
// on the 256^3 cavity.)
struct PackedWords {
  uint4 d;          // column deltas
  unsigned w0, w1;  // value-table indices
  int plain;        // the slice is stored in the plain sliced layout instead
};

// The words are loaded whatever the slice's plain flag (every row has them), so the flag,
// the words and the slot bases are one round trip, not two.
template <int NIB>
__device__ __forceinline__ void packed_words(const uint4* __restrict__ delta,
                                             const void* __restrict__ idx,
                                             const unsigned char* __restrict__ plain, int s,
                                             int lane, PackedWords& o) {
  const int i = s * 32 + lane;
  o.plain = __ldg(plain + s);
  o.d = ld_stream(delta + i);
  if (NIB == 4) {
    o.w0 = ld_stream(static_cast<const unsigned*>(idx) + i);
    o.w1 = 0u;
  } else {
    const uint2 w = ld_stream(static_cast<const uint2*>(idx) + i);
    o.w0 = w.x;
    o.w1 = w.y;
  }
}

// The row's eight columns: the slice's slot bases plus the row's deltas.
__device__ __forceinline__ void packed_cols(const int* __restrict__ base, int s, const uint4& d,
                                            int (&c)[8]) {
  const int4 b0 = __ldg(reinterpret_cast<const int4*>(base) + 2 * s);
  const int4 b1 = __ldg(reinterpret_cast<const int4*>(base) + 2 * s + 1);
  c[0] = b0.x + (int)(d.x & 0xffffu);
  c[1] = b0.y + (int)(d.x >> 16);
  c[2] = b0.z + (int)(d.y & 0xffffu);
  c[3] = b0.w + (int)(d.y >> 16);
  c[4] = b1.x + (int)(d.z & 0xffffu);
  c[5] = b1.y + (int)(d.z >> 16);
  c[6] = b1.z + (int)(d.w & 0xffffu);
  c[7] = b1.w + (int)(d.w >> 16);
}

// Value-table index of slot j.
template <int NIB>
__device__ __forceinline__ unsigned packed_index(const PackedWords& w, int j) {
  return (NIB == 4) ? (w.w0 >> (4 * j)) & 15u : ((j < 4 ? w.w0 : w.w1) >> (8 * (j & 3))) & 255u;
}

// Stored value of slot k: through the operator's value table (TAB: one byte per slot into
// vtab, the same doubles) or read directly.  A compile-time choice, like every switch in a
// gather loop.
template <bool TAB, typename V>
__device__ __forceinline__ V sell_value(const SellView<V>& A, long long k) {
  if constexpr (TAB)
    return __ldg(A.vtab + ld_stream(A.vidx + k));
  else
    return ld_stream(A.val + k);
}

// One row of a SELL-32 matrix, summed slot by slot in CSR order with GIP's rounding.
// `any` reports whether the row has at least one stored nonzero.
template <typename V, typename X, int CH = 8, bool TAB = false>
__device__ __forceinline__ void sell_row_f64(const SellView<V>& A, const X* __restrict__ x,
                                             int s, int lane, double& sum, bool& any) {
  long long base;
  int len;
  slice_range(A, s, base, len);
  const int* cp = A.col + base + lane;
  for (int j0 = 0; j0 < len; j0 += CH) {
    int c[CH];
    V v[CH];
#pragma unroll
    for (int t = 0; t < CH; ++t) {
      if (j0 + t < len) {
        c[t] = ld_stream(cp + (size_t)(j0 + t) * 32);
        v[t] = sell_value<TAB>(A, base + (long long)(j0 + t) * 32 + lane);
      } else {
        c[t] = -1;
        v[t] = V(0);
      }
    }
    double xv[CH];
#pragma unroll
    for (int t = 0; t < CH; ++t) xv[t] = (c[t] >= 0) ? (double)__ldg(x + c[t]) : 0.0;
#pragma unroll
    for (int t = 0; t < CH; ++t)
      if (c[t] >= 0) {
        sum = dadd(sum, dmul(xv[t], (double)v[t]));
        any = true;
      }
  }
}

// Two rows products of one operator row with two vectors (sum1 = row.x1, sum2 = row.x2),
// each summed slot by slot with GIP's rounding: the same results as two sell_row_f64
// calls, with the row's columns and values streamed once.
template <typename V, int CH = 4>
__device__ __forceinline__ void sell_row_f64_pair(const SellView<V>& A, const double* __restrict__ x1,
                                                  const double* __restrict__ x2, int s, int lane,
                                                  double& sum1, double& sum2, bool& any) {
  long long base;
  int len;
  slice_range(A, s, base, len);
  const int* cp = A.col + base + lane;
  const V* vp = A.val + base + lane;
  for (int j0 = 0; j0 < len; j0 += CH) {
    int c[CH];
    V v[CH];
#pragma unroll
    for (int t = 0; t < CH; ++t) {
      if (j0 + t < len) {
        c[t] = ld_stream(cp + (size_t)(j0 + t) * 32);
        v[t] = ld_stream(vp + (size_t)(j0 + t) * 32);
      } else {
        c[t] = -1;
        v[t] = V(0);
      }
    }
    double a[CH], b[CH];
#pragma unroll
    for (int t = 0; t < CH; ++t) {
      a[t] = (c[t] >= 0) ? __ldg(x1 + c[t]) : 0.0;
      b[t] = (c[t] >= 0) ? __ldg(x2 + c[t]) : 0.0;
    }
#pragma unroll
    for (int t = 0; t < CH; ++t)
      if (c[t] >= 0) {
        sum1 = dadd(sum1, dmul(a[t], (double)v[t]));
        sum2 = dadd(sum2, dmul(b[t], (double)v[t]));
        any = true;
      }
  }
}

// Three sliced operators' rows walked together (sum_k = row s of M_k . x_k, each summed slot
// by slot with GIP's rounding, any_k = the row has a stored nonzero): the slot loads of all
// three and then their gathers are in flight at once, three dependent round trips per row
// instead of nine.  The same results as three sell_row_f64 calls.
template <bool TAB = false>
__device__ __forceinline__ void sell_rows3_f64(const SellView<double> (&M)[3],
                                               const double* const (&x)[3], int s, int lane,
                                               double (&sum)[3], bool (&any)[3]) {
  long long base[3];
  int len[3], len_max = 0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    base[k] = 0;
    len[k] = 0;
    if (s < M[k].nslices) {
      slice_range(M[k], s, base[k], len[k]);
    }
    len_max = max(len_max, len[k]);
  }
  for (int j0 = 0; j0 < len_max; j0 += 2) {
    int c[3][2];
    double v[3][2], xv[3][2];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int j = j0 + t;
        c[k][t] = (j < len[k]) ? ld_stream(M[k].col + base[k] + 32LL * j + lane) : -1;
        v[k][t] = (j < len[k]) ? sell_value<TAB>(M[k], base[k] + 32LL * j + lane) : 0.0;
      }
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int t = 0; t < 2; ++t) xv[k][t] = (c[k][t] >= 0) ? __ldg(x[k] + c[k][t]) : 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int t = 0; t < 2; ++t)
        if (c[k][t] >= 0) {
          sum[k] = dadd(sum[k], dmul(xv[k][t], v[k][t]));
          any[k] = true;
        }
  }
}

// FP32 row: FP32 storage and FP32 accumulation (the inner solver of the mixed form).
template <int CH = 8>
__device__ __forceinline__ float sell_row_f32(const SellView<float>& A, const float* __restrict__ x,
                                              int s, int lane) {
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
    for (int t = 0; t < CH; ++t) xv[t] = (c[t] >= 0) ? __ldg(x + c[t]) : 0.f;
#pragma unroll
    for (int t = 0; t < CH; ++t) sum = fmaf(xv[t], v[t], sum);
  }
  return sum;
}

}  // namespace gipb200
