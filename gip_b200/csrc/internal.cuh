// Internal declarations shared by the gipb200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gipb200.h"

namespace gipb200 {

// ------------------------------------------------------------------ errors
int fail(int status, const char* fmt, ...);
void clear_error();

#define GIPB_CUDA(call)                                                                    \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return ::gipb200::fail(GIPB200_ERR_CUDA, "%s failed: %s (%s:%d)", #call,             \
                             cudaGetErrorString(e_), __FILE__, __LINE__);                  \
  } while (0)

#define GIPB_TRY(expr)                   \
  do {                                   \
    int s_ = (expr);                     \
    if (s_ != GIPB200_OK) return s_;     \
  } while (0)

#define GIPB_LAUNCH_CHECK()                                                                \
  do {                                                                                     \
    cudaError_t e_ = cudaGetLastError();                                                   \
    if (e_ != cudaSuccess)                                                                 \
      return ::gipb200::fail(GIPB200_ERR_CUDA, "kernel launch failed: %s (%s:%d)",         \
                             cudaGetErrorString(e_), __FILE__, __LINE__);                  \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ------------------------------------------------------------------ device info
struct DeviceInfo {
  int device = -1;
  int nsm = 0;
  int l2_bytes = 0;
};
int device_info(DeviceInfo* out);  // of the current device, cached per device

// ------------------------------------------------------------------ owning device buffer
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  int alloc(size_t count) {
    release();
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      return fail(GIPB200_ERR_NOMEM, "cudaMalloc(%zu bytes): %s", count * sizeof(T),
                  cudaGetErrorString(e));
    }
    n = count;
    return GIPB200_OK;
  }
  int upload(const T* h, size_t count, cudaStream_t s = 0) {
    GIPB_TRY(alloc(count));
    if (count) GIPB_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    return GIPB200_OK;
  }
  int zero(cudaStream_t s = 0) {
    GIPB_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
    return GIPB200_OK;
  }
};

// ------------------------------------------------------------------ reduction scratch
// Block partials plus a ticket counter for single-pass grid reductions.  The last
// block to arrive sums the partials in block order, so the result depends only on the
// launch shape, never on scheduling.
constexpr int kMaxReduceBlocks = 8192;
constexpr int kMaxReduceWidth = 4;
struct ReduceScratch {
  double* partials;   // [kMaxReduceWidth][kMaxReduceBlocks]
  unsigned* ticket;   // one counter, zero between launches
};
// `blocks` lowered to the number of 256-thread blocks of `kernel` that are resident at
// once on the device (grid-stride kernels then run in one wave, without a tail).
template <class K>
int one_wave(K kernel, int blocks, int* out) {
  DeviceInfo di;
  GIPB_TRY(device_info(&di));
  int per_sm = 0;
  GIPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0));
  *out = std::max(1, std::min(blocks, std::max(per_sm, 1) * di.nsm));
  return GIPB200_OK;
}

int reduce_scratch_alloc(DevBuf<double>* partials, DevBuf<unsigned>* ticket, ReduceScratch* out);

// ------------------------------------------------------------------ setup trace
// GIPB200_SETUP_TRACE=1: prints `what` with the wall time since the previous mark (and
// restarts the clock) on stderr; otherwise does nothing.
void setup_mark(const char* what);

// ------------------------------------------------------------------ dependent launches
// Programmatic dependent launch (GIPB200_PDL=1): a kernel of the PCG loop is scheduled
// while its predecessor in the stream is still running, so launch latency overlaps the
// predecessor's tail.  Every such kernel waits for its predecessor's completion
// (griddepcontrol.wait) before its first memory access, so results are unchanged.
bool pdl_enabled();
template <typename... KArgs, typename... Args>
void launch_dep(void (*kernel)(KArgs...), int grid, int block, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  (void)cudaLaunchKernelEx(&cfg, kernel, args...);  // failures surface in GIPB_LAUNCH_CHECK
}

// ------------------------------------------------------------------ sliced ELL (SELL-32)
// Rows are grouped in slices of 32; slice s stores its rows' nonzeros column-major
// (slot j of lane l at sptr[s] + 32*j + l), padded to the slice's longest row with
// col = -1.  Each row keeps its CSR nonzero order, so a lane summing slot by slot
// adds in exactly the CSR order.
template <typename V>
struct SellView {
  int nrows;
  int nslices;
  const long long* __restrict__ sptr;
  const int* __restrict__ col;
  const V* __restrict__ val;
  int uslots;  // > 0: every slice has this many slots (slice s starts at 32 * uslots * s)
  // optional value table (operators with at most 256 distinct stored values): slot k holds
  // vtab[vidx[k]], the same double as val[k], in one byte instead of eight
  const unsigned char* __restrict__ vidx = nullptr;
  const V* __restrict__ vtab = nullptr;
};

// Slot range of slice s: computed when the slices are uniform, else read from sptr.
template <typename V>
__host__ __device__ __forceinline__ void slice_range(const SellView<V>& A, int s, long long& base,
                                                     int& len) {
  if (A.uslots > 0) {
    base = 32LL * A.uslots * s;
    len = A.uslots;
  } else {
    base = A.sptr[s];
    len = (int)((A.sptr[s + 1] - base) >> 5);
  }
}

struct Sell {
  int nrows = 0, ncols = 0, nnz = 0, nslices = 0;
  long long nslots = 0;
  bool rows_nonempty = true;  // no empty row
  int uslots = 0;             // > 0: every slice has this many slots
  DevBuf<long long> sptr;
  DevBuf<int> col;
  DevBuf<double> val;
  DevBuf<float> val32;        // optional FP32 copy
  DevBuf<int> pos;            // CSR nonzero k -> slot index (value-target writes)
  DevBuf<int> rowptr;         // device CSR copy
  DevBuf<int> csr_col;
  DevBuf<double> csr_val;
  std::vector<int> h_rowptr, h_col;  // host CSR structure (setup only)
  // value table (sell_add_value_table): ntab > 0 distinct stored values, vidx per slot
  int ntab = 0;
  DevBuf<unsigned char> vidx;
  DevBuf<double> vtab;
  SellView<double> view() const {
    return {nrows, nslices, sptr.p, col.p, val.p, uslots, ntab ? vidx.p : nullptr,
            ntab ? vtab.p : nullptr};
  }
  SellView<double> view_vals(const double* v) const {
    return {nrows, nslices, sptr.p, col.p, v, uslots};
  }
  SellView<float> view32() const { return {nrows, nslices, sptr.p, col.p, val32.p, uslots}; }
};

// Builds SELL-32 from host CSR arrays, keeping what `keep` asks for: a device CSR copy
// (rowptr, csr_col, csr_val), the CSR -> slot position map (pos) and the host CSR structure
// (h_rowptr, h_col).
enum : unsigned { kKeepDeviceCsr = 1u, kKeepPos = 2u, kKeepHost = 4u, kKeepAll = 7u };
int sell_build(Sell* S, int nrows, int ncols, int nnz, const int* h_rowptr, const int* h_col,
               const double* h_val, cudaStream_t stream, unsigned keep = kKeepAll);
// Only the device CSR copy (operators read row by row, never sliced).
int csr_build(Sell* S, int nrows, int ncols, int nnz, const int* h_rowptr, const int* h_col,
              const double* h_val, cudaStream_t stream);
// Adds an FP32 value copy.
int sell_add_fp32(Sell* S, cudaStream_t stream);
// Adds a value table when the operator's stored values (h_val, its nnz CSR values) take at
// most 256 distinct doubles (bitwise); else leaves ntab = 0.  Lossless: the table holds
// the values themselves.
int sell_add_value_table(Sell* S, const double* h_val, long long nnz, cudaStream_t stream);
// The table of the distinct doubles (bitwise, sorted by bit pattern) among v[0..n), or
// false when there are more than `cap`.
bool value_table(const double* v, long long n, int cap, std::vector<double>* tab);
int validate_csr(int nrows, int ncols, int nnz, const int* rowptr, const int* col,
                 int col_bound, const char* name);

// Generic launches used by several translation units.
int launch_sell_spmv(const Sell& A, const double* vals, const double* x, double* y, double alpha,
                     double beta, int mode, cudaStream_t s);
int launch_csr_spmv(int nrows, const int* rowptr, const int* col, const double* val,
                    const double* x, double* y, const int* ypos, double alpha, double beta,
                    int mode, cudaStream_t s);
// The same product with the values read through a value table (vtab[vidx[j]]).
int launch_csr_spmv_tab(int nrows, const int* rowptr, const int* col, const unsigned char* vidx,
                        const double* vtab, const double* x, double* y, const int* ypos,
                        double alpha, double beta, int mode, cudaStream_t s);
int grid_blocks(int threads, int work_items, int per_thread, int max_blocks, int* blocks);

}  // namespace gipb200

struct gipb200_matrix_s {
  gipb200::Sell S;
  // reduction scratch of the fused operations called on this handle (spmv_dot,
  // cg_update_dot): calls that share a handle must be ordered on one stream
  gipb200::DevBuf<double> partials;
  gipb200::DevBuf<unsigned> ticket;
  gipb200::ReduceScratch rs{};
};
