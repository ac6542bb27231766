// Library plumbing, raw-pointer kernels (the counterparts of GIP's libgpu.cu routines),
// sliced-ELL construction and matrix handles.
#include <cuda_runtime.h>
#include <stdio.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <mutex>

#include "device.cuh"
#include "internal.cuh"

namespace gipb200 {

// ------------------------------------------------------------------ errors
static thread_local std::string g_last_error;

int fail(int status, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return status;
}
void clear_error() { g_last_error.clear(); }

void setup_mark(const char* what) {
  static thread_local std::chrono::steady_clock::time_point last = std::chrono::steady_clock::now();
  if (!getenv("GIPB200_SETUP_TRACE")) return;
  const auto now = std::chrono::steady_clock::now();
  fprintf(stderr, "gipb200 setup: %-28s %8.3f s\n", what,
          std::chrono::duration<double>(now - last).count());
  last = now;
}

bool pdl_enabled() {
  const char* e = getenv("GIPB200_PDL");  // read at each launch (captured graphs keep it)
  return e && e[0] == '1';
}

// ------------------------------------------------------------------ device info
int device_info(DeviceInfo* out) {
  static std::mutex mu;
  static DeviceInfo cache[64];
  int dev = 0;
  GIPB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(GIPB200_ERR_ARG, "device index %d out of range", dev);
  std::lock_guard<std::mutex> lk(mu);
  if (cache[dev].device != dev) {
    DeviceInfo d;
    d.device = dev;
    GIPB_CUDA(cudaDeviceGetAttribute(&d.nsm, cudaDevAttrMultiProcessorCount, dev));
    GIPB_CUDA(cudaDeviceGetAttribute(&d.l2_bytes, cudaDevAttrL2CacheSize, dev));
    cache[dev] = d;
  }
  *out = cache[dev];
  return GIPB200_OK;
}

int grid_blocks(int threads, int work_items, int per_thread, int max_blocks, int* blocks) {
  DeviceInfo di;
  GIPB_TRY(device_info(&di));
  long long need = ((long long)work_items + (long long)threads * per_thread - 1) /
                   ((long long)threads * per_thread);
  long long cap = (long long)di.nsm * (2048 / threads);
  if (max_blocks > 0) cap = std::min<long long>(cap, max_blocks);
  long long b = std::max<long long>(1, std::min(need, cap));
  *blocks = (int)b;
  return GIPB200_OK;
}

int reduce_scratch_alloc(DevBuf<double>* partials, DevBuf<unsigned>* ticket, ReduceScratch* out) {
  GIPB_TRY(partials->alloc((size_t)kMaxReduceWidth * kMaxReduceBlocks));
  GIPB_TRY(ticket->alloc(1));
  GIPB_CUDA(cudaMemset(ticket->p, 0, sizeof(unsigned)));
  out->partials = partials->p;
  out->ticket = ticket->p;
  return GIPB200_OK;
}

// ------------------------------------------------------------------ validation
int validate_csr(int nrows, int ncols, int nnz, const int* rowptr, const int* col, int col_bound,
                 const char* name) {
  if (nrows < 0 || ncols < 0 || nnz < 0)
    return fail(GIPB200_ERR_ARG, "%s: negative size", name);
  if (nrows > 0 && !rowptr) return fail(GIPB200_ERR_ARG, "%s: null rowptr", name);
  if (nnz > 0 && !col) return fail(GIPB200_ERR_ARG, "%s: null col", name);
  if (nrows > 0 && rowptr[0] != 0) return fail(GIPB200_ERR_ARG, "%s: rowptr[0] != 0", name);
  for (int i = 0; i < nrows; ++i)
    if (rowptr[i + 1] < rowptr[i]) return fail(GIPB200_ERR_ARG, "%s: rowptr decreases at %d", name, i);
  if (nrows > 0 && rowptr[nrows] != nnz)
    return fail(GIPB200_ERR_ARG, "%s: rowptr[nrows]=%d != nnz=%d", name, rowptr[nrows], nnz);
  for (int k = 0; k < nnz; ++k)
    if (col[k] < 0 || (col_bound >= 0 && col[k] >= col_bound))
      return fail(GIPB200_ERR_ARG, "%s: column %d at nonzero %d out of [0,%d)", name, col[k], k,
                  col_bound);
  return GIPB200_OK;
}

// ------------------------------------------------------------------ SELL-32 build
int sell_build(Sell* S, int nrows, int ncols, int nnz, const int* rp, const int* col,
               const double* val, cudaStream_t stream, unsigned keep) {
  // every gather must stay inside an x of ncols entries
  GIPB_TRY(validate_csr(nrows, ncols, nnz, rp, col, ncols, "matrix"));
  S->nrows = nrows;
  S->ncols = ncols;
  S->nnz = nnz;
  S->nslices = (nrows + 31) / 32;
  std::vector<long long> sptr((size_t)S->nslices + 1, 0);
  bool nonempty = true;
  for (int s = 0; s < S->nslices; ++s) {
    int len = 0;
    for (int r = s * 32; r < std::min(nrows, s * 32 + 32); ++r) {
      len = std::max(len, rp[r + 1] - rp[r]);
      nonempty = nonempty && (rp[r + 1] > rp[r]);
    }
    sptr[s + 1] = sptr[s] + 32LL * len;
  }
  S->rows_nonempty = nonempty;
  S->nslots = sptr[S->nslices];
  S->uslots = 0;
  if (S->nslices > 0 && S->nslots > 0 && !getenv("GIPB200_NO_UNIFORM")) {
    const long long l0 = sptr[1] - sptr[0];
    bool uniform = true;
    for (int s = 1; s < S->nslices && uniform; ++s) uniform = sptr[s + 1] - sptr[s] == l0;
    if (uniform) S->uslots = (int)(l0 / 32);
  }
  std::vector<int> scol((size_t)std::max<long long>(S->nslots, 1), -1);
  std::vector<double> sval((size_t)std::max<long long>(S->nslots, 1), 0.0);
  if (S->nslots > 0x7fffffffLL)
    return fail(GIPB200_ERR_ARG, "matrix too large for 32-bit slot indices");
  const bool want_pos = (keep & kKeepPos) != 0;
  std::vector<int> pos(want_pos ? (size_t)std::max(nnz, 1) : 0, 0);
#pragma omp parallel for schedule(static)
  for (int r = 0; r < nrows; ++r) {
    int s = r >> 5, lane = r & 31;
    for (int k = rp[r]; k < rp[r + 1]; ++k) {
      long long slot = sptr[s] + 32LL * (k - rp[r]) + lane;
      scol[slot] = col[k];
      sval[slot] = val ? val[k] : 0.0;
      if (want_pos) pos[k] = (int)slot;
    }
  }
  GIPB_TRY(S->sptr.upload(sptr.data(), sptr.size(), stream));
  GIPB_TRY(S->col.upload(scol.data(), scol.size(), stream));
  GIPB_TRY(S->val.upload(sval.data(), sval.size(), stream));
  if (want_pos) GIPB_TRY(S->pos.upload(pos.data(), pos.size(), stream));
  if (keep & kKeepDeviceCsr) {
    GIPB_TRY(S->rowptr.upload(rp, (size_t)nrows + 1, stream));
    GIPB_TRY(S->csr_col.upload(col, (size_t)std::max(nnz, 1), stream));
    if (val) {
      GIPB_TRY(S->csr_val.upload(val, (size_t)std::max(nnz, 1), stream));
    } else {
      GIPB_TRY(S->csr_val.alloc((size_t)std::max(nnz, 1)));
      GIPB_TRY(S->csr_val.zero(stream));
    }
  }
  if (keep & kKeepHost) {
    S->h_rowptr.assign(rp, rp + nrows + 1);
    S->h_col.assign(col, col + nnz);
  }
  GIPB_CUDA(cudaStreamSynchronize(stream));  // host staging vectors go out of scope
  return GIPB200_OK;
}

int csr_build(Sell* S, int nrows, int ncols, int nnz, const int* rp, const int* col,
              const double* val, cudaStream_t stream) {
  GIPB_TRY(validate_csr(nrows, ncols, nnz, rp, col, ncols, "matrix"));
  S->nrows = nrows;
  S->ncols = ncols;
  S->nnz = nnz;
  S->nslices = 0;
  S->nslots = 0;
  GIPB_TRY(S->rowptr.upload(rp, (size_t)nrows + 1, stream));
  GIPB_TRY(S->csr_col.upload(col, (size_t)std::max(nnz, 1), stream));
  if (val) {
    GIPB_TRY(S->csr_val.upload(val, (size_t)std::max(nnz, 1), stream));
  } else {
    GIPB_TRY(S->csr_val.alloc((size_t)std::max(nnz, 1)));
    GIPB_TRY(S->csr_val.zero(stream));
  }
  GIPB_CUDA(cudaStreamSynchronize(stream));
  return GIPB200_OK;
}

__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

int sell_add_fp32(Sell* S, cudaStream_t stream) {
  GIPB_TRY(S->val32.alloc((size_t)std::max<long long>(S->nslots, 1)));
  int blocks;
  GIPB_TRY(grid_blocks(256, (int)std::min<long long>(S->nslots, 1 << 30), 1, 0, &blocks));
  k_to_f32<<<blocks, 256, 0, stream>>>(S->val.p, S->val32.p, S->nslots);
  GIPB_LAUNCH_CHECK();
  return GIPB200_OK;
}

// ------------------------------------------------------------------ value tables
bool value_table(const double* v, long long n, int cap, std::vector<double>* tab) {
  std::vector<unsigned long long> keys;
  bool ok = true;
#pragma omp parallel
  {
    std::vector<unsigned long long> loc;
    bool lok = true;
    unsigned long long last = 0;
    bool have_last = false;
#pragma omp for schedule(static) nowait
    for (long long k = 0; k < n; ++k) {
      if (!lok) continue;
      unsigned long long b;
      memcpy(&b, v + k, 8);
      if (have_last && b == last) continue;
      if (std::find(loc.begin(), loc.end(), b) == loc.end()) {
        if ((int)loc.size() >= cap) {
          lok = false;
          continue;
        }
        loc.push_back(b);
      }
      last = b;
      have_last = true;
    }
#pragma omp critical
    {
      if (!lok) ok = false;
      for (unsigned long long b : loc)
        if (std::find(keys.begin(), keys.end(), b) == keys.end()) keys.push_back(b);
    }
  }
  if (!ok || (int)keys.size() > cap) return false;
  std::sort(keys.begin(), keys.end());
  tab->resize(keys.size());
  for (size_t t = 0; t < keys.size(); ++t) memcpy(&(*tab)[t], &keys[t], 8);
  return true;
}

// idx[k] = position of val[k]'s bit pattern in the sorted keys (padding slots: 0); miss
// counts stored slots whose value the table does not hold.
__global__ void k_value_index(long long nslots, const double* __restrict__ val,
                              const int* __restrict__ col, const unsigned long long* __restrict__ keys,
                              int nkeys, unsigned char* __restrict__ idx, unsigned* miss) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nslots;
       k += (long long)gridDim.x * blockDim.x) {
    int t = 0;
    if (col[k] >= 0) {
      const unsigned long long b = (unsigned long long)__double_as_longlong(val[k]);
      int lo = 0, hi = nkeys - 1;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (keys[mid] < b) lo = mid + 1;
        else hi = mid;
      }
      if (keys[lo] != b) atomicAdd(miss, 1u);
      t = lo;
    }
    idx[k] = (unsigned char)t;
  }
}

int sell_add_value_table(Sell* S, const double* h_val, long long nnz, cudaStream_t stream) {
  S->ntab = 0;
  if (S->nslots == 0 || nnz <= 0 || !h_val || getenv("GIPB200_NO_VALUE_TABLE")) return GIPB200_OK;
  std::vector<double> tab;
  if (!value_table(h_val, nnz, 256, &tab) || tab.empty()) return GIPB200_OK;
  std::vector<unsigned long long> keys(tab.size());
  for (size_t t = 0; t < tab.size(); ++t) memcpy(&keys[t], &tab[t], 8);
  DevBuf<unsigned long long> dkeys;
  DevBuf<unsigned> miss;
  GIPB_TRY(dkeys.upload(keys.data(), keys.size(), stream));
  GIPB_TRY(miss.alloc(1));
  GIPB_TRY(miss.zero(stream));
  GIPB_TRY(S->vidx.alloc((size_t)S->nslots));
  int blocks;
  GIPB_TRY(grid_blocks(256, (int)std::min<long long>(S->nslots, 1 << 30), 1, 0, &blocks));
  k_value_index<<<blocks, 256, 0, stream>>>(S->nslots, S->val.p, S->col.p, dkeys.p,
                                            (int)keys.size(), S->vidx.p, miss.p);
  GIPB_LAUNCH_CHECK();
  unsigned h_miss = 0;
  GIPB_CUDA(cudaMemcpyAsync(&h_miss, miss.p, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
  GIPB_CUDA(cudaStreamSynchronize(stream));
  if (h_miss) {  // slot values that are not the CSR values: keep the direct layout only
    S->vidx.release();
    return GIPB200_OK;
  }
  GIPB_TRY(S->vtab.upload(tab.data(), tab.size(), stream));
  GIPB_CUDA(cudaStreamSynchronize(stream));
  S->ntab = (int)tab.size();
  return GIPB200_OK;
}

// ------------------------------------------------------------------ SpMV kernels
// mode 0: y = Ax; mode 1: y = alpha Ax + beta y.  Rows without nonzeros keep y.
__global__ void __launch_bounds__(256) k_sell_spmv(SellView<double> A, const double* __restrict__ x,
                                                   double* __restrict__ y, double alpha,
                                                   double beta, int mode) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int s = gw; s < A.nslices; s += nw) {
    double sum = 0.0;
    bool any = false;
    sell_row_f64(A, x, s, lane, sum, any);
    const int row = s * 32 + lane;
    if (row < A.nrows && any) y[row] = mode ? dadd(dmul(alpha, sum), dmul(beta, y[row])) : sum;
  }
}

// Thread-per-row CSR for raw device pointers and for operators whose rows vary too much
// in length for slicing (Ec).  `ypos` (optional) scatters row k to y[ypos[k]].
__global__ void __launch_bounds__(256) k_csr_spmv(int nrows, const int* __restrict__ rp,
                                                  const int* __restrict__ col,
                                                  const double* __restrict__ val,
                                                  const double* __restrict__ x, double* y,
                                                  const int* __restrict__ ypos, double alpha,
                                                  double beta, int mode) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += gridDim.x * blockDim.x) {
    const int jb = rp[r], je = rp[r + 1];
    if (jb == je) continue;
    double sum = 0.0;
    for (int j = jb; j < je; ++j) sum = dadd(sum, dmul(__ldg(x + col[j]), val[j]));
    const int o = ypos ? ypos[r] : r;
    y[o] = mode ? dadd(dmul(alpha, sum), dmul(beta, y[o])) : sum;
  }
}

// k_csr_spmv with the stored values read through a value table (vidx, vtab)
__global__ void __launch_bounds__(256) k_csr_spmv_tab(int nrows, const int* __restrict__ rp,
                                                      const int* __restrict__ col,
                                                      const unsigned char* __restrict__ vidx,
                                                      const double* __restrict__ vtab,
                                                      const double* __restrict__ x, double* y,
                                                      const int* __restrict__ ypos, double alpha,
                                                      double beta, int mode) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += gridDim.x * blockDim.x) {
    const int jb = rp[r], je = rp[r + 1];
    if (jb == je) continue;
    double sum = 0.0;
    for (int j = jb; j < je; ++j) sum = dadd(sum, dmul(__ldg(x + col[j]), __ldg(vtab + vidx[j])));
    const int o = ypos ? ypos[r] : r;
    y[o] = mode ? dadd(dmul(alpha, sum), dmul(beta, y[o])) : sum;
  }
}

int launch_csr_spmv_tab(int nrows, const int* rowptr, const int* col, const unsigned char* vidx,
                        const double* vtab, const double* x, double* y, const int* ypos,
                        double alpha, double beta, int mode, cudaStream_t s) {
  if (nrows == 0) return GIPB200_OK;
  int blocks;
  GIPB_TRY(grid_blocks(256, nrows, 1, 0, &blocks));
  k_csr_spmv_tab<<<blocks, 256, 0, s>>>(nrows, rowptr, col, vidx, vtab, x, y, ypos, alpha, beta,
                                        mode);
  GIPB_LAUNCH_CHECK();
  return GIPB200_OK;
}

int launch_sell_spmv(const Sell& A, const double* vals, const double* x, double* y, double alpha,
                     double beta, int mode, cudaStream_t s) {
  if (A.nrows == 0) return GIPB200_OK;
  int blocks;
  GIPB_TRY(grid_blocks(256, A.nslices * 32, 1, 0, &blocks));
  k_sell_spmv<<<blocks, 256, 0, s>>>(A.view_vals(vals), x, y, alpha, beta, mode);
  GIPB_LAUNCH_CHECK();
  return GIPB200_OK;
}

int launch_csr_spmv(int nrows, const int* rowptr, const int* col, const double* val,
                    const double* x, double* y, const int* ypos, double alpha, double beta,
                    int mode, cudaStream_t s) {
  if (nrows == 0) return GIPB200_OK;
  int blocks;
  GIPB_TRY(grid_blocks(256, nrows, 1, 0, &blocks));
  k_csr_spmv<<<blocks, 256, 0, s>>>(nrows, rowptr, col, val, x, y, ypos, alpha, beta, mode);
  GIPB_LAUNCH_CHECK();
  return GIPB200_OK;
}

// ------------------------------------------------------------------ vector kernels
__global__ void k_axpy(int n, double* __restrict__ y, const double* __restrict__ x, double a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = dadd(y[i], dmul(a, x[i]));
}
__global__ void k_axpby(int n, double* __restrict__ y, const double* __restrict__ x, double a,
                        double b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = dadd(dmul(a, x[i]), dmul(b, y[i]));
}
// GIP_Topo::pack / unpack (GIP_Topo.cpp:109-122) kept in device memory
__global__ void k_gather(int n, const int* __restrict__ idx, const double* __restrict__ x,
                         double* __restrict__ buf) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    buf[k] = x[idx[k]];
}
__global__ void k_scatter(int n, const int* __restrict__ idx, const double* __restrict__ buf,
                          double* __restrict__ x) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    x[idx[k]] = buf[k];
}
__global__ void k_fill(int n, double* __restrict__ y, double v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = v;
}

struct StoreResult {
  double* out;
  __device__ void operator()(const double* t) const { *out = t[0]; }
};

__global__ void __launch_bounds__(256) k_dot(int n, const double* __restrict__ x,
                                             const double* __restrict__ y, ReduceScratch rs,
                                             double* out) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    acc[0] = dadd(acc[0], dmul(x[i], y[i]));
  grid_reduce<SumOp, 1>(acc, rs, StoreResult{out});
}

__global__ void __launch_bounds__(256) k_norminf(int n, const double* __restrict__ x,
                                                 ReduceScratch rs, double* out) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double a = fabs(x[i]);
    if (a > acc[0]) acc[0] = a;
  }
  grid_reduce<MaxOp, 1>(acc, rs, StoreResult{out});
}

// Per-cell CFL candidate with GIP's CPU expression order (GIP_NonLinearMulticore.cpp:20-35).
__device__ __forceinline__ double cfl_cell(double ut, double vt, double wt, double dx,
                                           double gamma, double rho, double dt) {
  const double convCoef = 0.25;
  double normit = (fabs(ut) > fabs(vt)) ? fabs(ut) : fabs(vt);
  if (normit < fabs(wt)) normit = fabs(wt);
  if (!(ddiv(dx, normit) < 1e-17)) {
    double c = ddiv(dmul(convCoef, dx), normit);
    if (dt > c) dt = c;
  }
  double d2 = ddiv(dmul(dmul(dmul(dx, dx), rho), 1.0), gamma);  // dx*dx*rho/gamma
  if (!(d2 < 1e-17)) {
    double c = ddiv(dmul(dmul(dmul(0.2, dx), dx), rho), gamma);
    if (dt > c) dt = c;
  }
  return dt;
}

struct CflFinish {
  double* out;
  __device__ void operator()(const double* t) const {
    const double fin = t[0];
    *out = (dmul(0.8, fin) > 1e-1) ? 1e-1 : dmul(0.8, fin);
  }
};

__global__ void __launch_bounds__(256) k_cfl(int n, const double* __restrict__ u,
                                             const double* __restrict__ v,
                                             const double* __restrict__ w,
                                             const double* __restrict__ dxs, double gamma,
                                             double rho, ReduceScratch rs, double* out) {
  double acc[1] = {1e20};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    acc[0] = cfl_cell(u[i], v[i], w[i], dxs[i], gamma, rho, acc[0]);
  grid_reduce<MinOp, 1>(acc, rs, CflFinish{out});
}

// Shared scratch for the blocking raw-pointer reductions: one per device, serialised.
struct RawScratch {
  std::mutex mu;
  DevBuf<double> partials, result;
  DevBuf<unsigned> ticket;
  ReduceScratch rs{};
  double* h_result = nullptr;
  bool ready = false;
};
static RawScratch g_raw[64];

static int raw_scratch(RawScratch** out) {
  DeviceInfo di;
  GIPB_TRY(device_info(&di));
  RawScratch* r = &g_raw[di.device];
  if (!r->ready) {
    GIPB_TRY(reduce_scratch_alloc(&r->partials, &r->ticket, &r->rs));
    GIPB_TRY(r->result.alloc(1));
    GIPB_CUDA(cudaMallocHost(reinterpret_cast<void**>(&r->h_result), sizeof(double)));
    r->ready = true;
  }
  *out = r;
  return GIPB200_OK;
}

}  // namespace gipb200

using namespace gipb200;

// ====================================================================== C ABI
extern "C" {

int gipb200_version(void) { return 100; }

const char* gipb200_status_string(int s) {
  switch (s) {
    case GIPB200_OK: return "ok";
    case GIPB200_ERR_ARG: return "invalid argument";
    case GIPB200_ERR_CUDA: return "CUDA error";
    case GIPB200_ERR_BREAKDOWN: return "PCG breakdown";
    case GIPB200_ERR_TIMEOUT: return "device wait timed out";
    case GIPB200_ERR_NOMEM: return "out of memory";
    case GIPB200_ERR_NOT_CONVERGED: return "not converged";
    case GIPB200_ERR_STATE: return "invalid state";
    default: return "unknown status";
  }
}

const char* gipb200_last_error(void) { return g_last_error.c_str(); }

int gipb200_set_device(int device) {
  GIPB_CUDA(cudaSetDevice(device));
  return GIPB200_OK;
}
int gipb200_malloc(void** d_ptr, size_t bytes) {
  if (!d_ptr) return fail(GIPB200_ERR_ARG, "null output pointer");
  cudaError_t e = cudaMalloc(d_ptr, bytes ? bytes : 1);
  if (e != cudaSuccess) return fail(GIPB200_ERR_NOMEM, "cudaMalloc: %s", cudaGetErrorString(e));
  return GIPB200_OK;
}
int gipb200_free(void* d_ptr) {
  GIPB_CUDA(cudaFree(d_ptr));
  return GIPB200_OK;
}
int gipb200_memcpy_h2d(void* d, const void* h, size_t bytes, void* stream) {
  GIPB_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, as_stream(stream)));
  return GIPB200_OK;
}
int gipb200_memcpy_d2h(void* h, const void* d, size_t bytes, void* stream) {
  GIPB_CUDA(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, as_stream(stream)));
  GIPB_CUDA(cudaStreamSynchronize(as_stream(stream)));
  return GIPB200_OK;
}
int gipb200_memcpy_d2h_async(void* h, const void* d, size_t bytes, void* stream) {
  GIPB_CUDA(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, as_stream(stream)));
  return GIPB200_OK;
}
int gipb200_dcopy(int n, double* d_dst, const double* d_src, void* stream) {
  if (n < 0) return fail(GIPB200_ERR_ARG, "negative size");
  if (n == 0) return GIPB200_OK;
  GIPB_CUDA(cudaMemcpyAsync(d_dst, d_src, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice,
                            as_stream(stream)));
  return GIPB200_OK;
}
int gipb200_stream_sync(void* stream) {
  GIPB_CUDA(cudaStreamSynchronize(as_stream(stream)));
  return GIPB200_OK;
}

int gipb200_event_create(void** ev) {
  if (!ev) return fail(GIPB200_ERR_ARG, "null output");
  cudaEvent_t e;
  GIPB_CUDA(cudaEventCreate(&e));
  *ev = (void*)e;
  return GIPB200_OK;
}
int gipb200_event_record(void* ev, void* stream) {
  GIPB_CUDA(cudaEventRecord((cudaEvent_t)ev, as_stream(stream)));
  return GIPB200_OK;
}
int gipb200_event_elapsed_ms(void* a, void* b, float* ms) {
  if (!ms) return fail(GIPB200_ERR_ARG, "null output");
  GIPB_CUDA(cudaEventSynchronize((cudaEvent_t)b));
  GIPB_CUDA(cudaEventElapsedTime(ms, (cudaEvent_t)a, (cudaEvent_t)b));
  return GIPB200_OK;
}
int gipb200_event_destroy(void* ev) {
  GIPB_CUDA(cudaEventDestroy((cudaEvent_t)ev));
  return GIPB200_OK;
}

int gipb200_dcsr_spmv(int nrows, const int* d_rowptr, const int* d_col, const double* d_val,
                      const double* d_x, double* d_y, double alpha, double beta, int mode,
                      void* stream) {
  if (nrows < 0 || (mode != 0 && mode != 1)) return fail(GIPB200_ERR_ARG, "bad nrows/mode");
  if (nrows > 0 && (!d_rowptr || !d_x || !d_y))
    return fail(GIPB200_ERR_ARG, "null device pointer");
  return launch_csr_spmv(nrows, d_rowptr, d_col, d_val, d_x, d_y, nullptr, alpha, beta, mode,
                         as_stream(stream));
}

int gipb200_daxpy(int n, double* y, const double* x, double a, void* stream) {
  if (n < 0) return fail(GIPB200_ERR_ARG, "negative size");
  if (n == 0) return GIPB200_OK;
  int b;
  GIPB_TRY(grid_blocks(256, n, 4, 0, &b));
  k_axpy<<<b, 256, 0, as_stream(stream)>>>(n, y, x, a);
  GIPB_LAUNCH_CHECK();
  return GIPB200_OK;
}
int gipb200_daxpby(int n, double* y, const double* x, double a, double bt, void* stream) {
  if (n < 0) return fail(GIPB200_ERR_ARG, "negative size");
  if (n == 0) return GIPB200_OK;
  int b;
  GIPB_TRY(grid_blocks(256, n, 4, 0, &b));
  k_axpby<<<b, 256, 0, as_stream(stream)>>>(n, y, x, a, bt);
  GIPB_LAUNCH_CHECK();
  return GIPB200_OK;
}
int gipb200_dfill(int n, double* y, double v, void* stream) {
  if (n < 0) return fail(GIPB200_ERR_ARG, "negative size");
  if (n == 0) return GIPB200_OK;
  int b;
  GIPB_TRY(grid_blocks(256, n, 4, 0, &b));
  k_fill<<<b, 256, 0, as_stream(stream)>>>(n, y, v);
  GIPB_LAUNCH_CHECK();
  return GIPB200_OK;
}

int gipb200_gather(int n, const int* d_idx, const double* d_x, double* d_buf, void* stream) {
  if (n < 0 || (n > 0 && (!d_idx || !d_x || !d_buf)))
    return fail(GIPB200_ERR_ARG, "gather: bad size or null pointer");
  if (n == 0) return GIPB200_OK;
  int b;
  GIPB_TRY(grid_blocks(256, n, 4, 0, &b));
  k_gather<<<b, 256, 0, as_stream(stream)>>>(n, d_idx, d_x, d_buf);
  GIPB_LAUNCH_CHECK();
  return GIPB200_OK;
}

int gipb200_scatter(int n, const int* d_idx, const double* d_buf, double* d_x, void* stream) {
  if (n < 0 || (n > 0 && (!d_idx || !d_x || !d_buf)))
    return fail(GIPB200_ERR_ARG, "scatter: bad size or null pointer");
  if (n == 0) return GIPB200_OK;
  int b;
  GIPB_TRY(grid_blocks(256, n, 4, 0, &b));
  k_scatter<<<b, 256, 0, as_stream(stream)>>>(n, d_idx, d_buf, d_x);
  GIPB_LAUNCH_CHECK();
  return GIPB200_OK;
}

static int raw_reduce_finish(RawScratch* r, cudaStream_t s, double* h_result) {
  GIPB_CUDA(cudaMemcpyAsync(r->h_result, r->result.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaStreamSynchronize(s));
  *h_result = *r->h_result;
  return GIPB200_OK;
}

int gipb200_ddot(int n, const double* x, const double* y, double* h_result, void* stream) {
  if (n < 0 || !h_result) return fail(GIPB200_ERR_ARG, "bad size or null result");
  if (n == 0) {
    *h_result = 0.0;
    return GIPB200_OK;
  }
  RawScratch* r;
  GIPB_TRY(raw_scratch(&r));
  std::lock_guard<std::mutex> lk(r->mu);
  int b;
  GIPB_TRY(grid_blocks(256, n, 4, kMaxReduceBlocks, &b));
  k_dot<<<b, 256, 0, as_stream(stream)>>>(n, x, y, r->rs, r->result.p);
  GIPB_LAUNCH_CHECK();
  return raw_reduce_finish(r, as_stream(stream), h_result);
}

int gipb200_dnorminf(int n, const double* x, double* h_result, void* stream) {
  if (n < 0 || !h_result) return fail(GIPB200_ERR_ARG, "bad size or null result");
  if (n == 0) {
    *h_result = 0.0;
    return GIPB200_OK;
  }
  RawScratch* r;
  GIPB_TRY(raw_scratch(&r));
  std::lock_guard<std::mutex> lk(r->mu);
  int b;
  GIPB_TRY(grid_blocks(256, n, 4, kMaxReduceBlocks, &b));
  k_norminf<<<b, 256, 0, as_stream(stream)>>>(n, x, r->rs, r->result.p);
  GIPB_LAUNCH_CHECK();
  return raw_reduce_finish(r, as_stream(stream), h_result);
}

int gipb200_cfl(int n, const double* u, const double* v, const double* w, const double* dxs,
                double gamma, double rho, double* h_dt, void* stream) {
  if (n < 0 || !h_dt) return fail(GIPB200_ERR_ARG, "bad size or null result");
  RawScratch* r;
  GIPB_TRY(raw_scratch(&r));
  std::lock_guard<std::mutex> lk(r->mu);
  int b;
  GIPB_TRY(grid_blocks(256, std::max(n, 1), 4, kMaxReduceBlocks, &b));
  k_cfl<<<b, 256, 0, as_stream(stream)>>>(n, u, v, w, dxs, gamma, rho, r->rs, r->result.p);
  GIPB_LAUNCH_CHECK();
  return raw_reduce_finish(r, as_stream(stream), h_dt);
}

// ------------------------------------------------------------------ matrix handles
int gipb200_matrix_create(int nrows, int ncols, int nnz, const int* rp, const int* col,
                          const double* val, gipb200_matrix* out) {
  if (!out) return fail(GIPB200_ERR_ARG, "null output handle");
  *out = nullptr;
  gipb200_matrix A = new (std::nothrow) gipb200_matrix_s();
  if (!A) return fail(GIPB200_ERR_NOMEM, "host allocation failed");
  int st = sell_build(&A->S, nrows, ncols, nnz, rp, col, val, 0);
  if (st == GIPB200_OK) st = reduce_scratch_alloc(&A->partials, &A->ticket, &A->rs);
  if (st != GIPB200_OK) {
    delete A;
    return st;
  }
  *out = A;
  return GIPB200_OK;
}

int gipb200_matrix_destroy(gipb200_matrix A) {
  delete A;
  return GIPB200_OK;
}

int gipb200_matrix_info(gipb200_matrix A, int* nrows, int* ncols, int* nnz, int64_t* slots) {
  if (!A) return fail(GIPB200_ERR_ARG, "null matrix");
  if (nrows) *nrows = A->S.nrows;
  if (ncols) *ncols = A->S.ncols;
  if (nnz) *nnz = A->S.nnz;
  if (slots) *slots = A->S.nslots;
  return GIPB200_OK;
}

int gipb200_matrix_spmv(gipb200_matrix A, const double* x, double* y, double alpha, double beta,
                        int mode, void* stream) {
  if (!A || (mode != 0 && mode != 1)) return fail(GIPB200_ERR_ARG, "null matrix or bad mode");
  return launch_sell_spmv(A->S, A->S.val.p, x, y, alpha, beta, mode, as_stream(stream));
}

__global__ void k_scatter_vals(int nnz, const int* __restrict__ pos, const double* __restrict__ csr,
                               double* __restrict__ sell) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x)
    sell[pos[k]] = csr[k];
}

int gipb200_matrix_spmv_values(gipb200_matrix A, const double* x, gipb200_matrix T, double alpha,
                               double beta, int mode, void* stream) {
  if (!A || !T || (mode != 0 && mode != 1)) return fail(GIPB200_ERR_ARG, "bad arguments");
  if (A->S.nrows != T->S.nnz)
    return fail(GIPB200_ERR_ARG, "operator has %d rows but target has %d values", A->S.nrows,
                T->S.nnz);
  cudaStream_t s = as_stream(stream);
  // the target keeps its CSR values authoritative; the sliced copy follows
  GIPB_TRY(launch_csr_spmv(A->S.nrows, A->S.rowptr.p, A->S.csr_col.p, A->S.csr_val.p, x,
                           T->S.csr_val.p, nullptr, alpha, beta, mode, s));
  if (T->S.nnz > 0) {
    int b;
    GIPB_TRY(grid_blocks(256, T->S.nnz, 4, 0, &b));
    k_scatter_vals<<<b, 256, 0, s>>>(T->S.nnz, T->S.pos.p, T->S.csr_val.p, T->S.val.p);
    GIPB_LAUNCH_CHECK();
  }
  return GIPB200_OK;
}

int gipb200_matrix_get_values(gipb200_matrix A, double* h_val) {
  if (!A || (!h_val && A->S.nnz)) return fail(GIPB200_ERR_ARG, "bad arguments");
  if (A->S.nnz)
    GIPB_CUDA(cudaMemcpy(h_val, A->S.csr_val.p, (size_t)A->S.nnz * sizeof(double),
                         cudaMemcpyDeviceToHost));
  return GIPB200_OK;
}

__global__ void k_inv_diag(int nrows, const int* __restrict__ rp, const int* __restrict__ col,
                           const double* __restrict__ val, double* __restrict__ dinv,
                           int* missing) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrows; i += gridDim.x * blockDim.x) {
    double d = 0.0;
    bool found = false;
    for (int j = rp[i]; j < rp[i + 1]; ++j)
      if (col[j] == i) {
        d = ddiv(1.0, val[j]);  // the last diagonal entry wins, as in GIP's loop
        found = true;
      }
    dinv[i] = d;
    if (!found) atomicAdd(missing, 1);
  }
}

int gipb200_matrix_inverse_diagonal(gipb200_matrix A, double* d_dinv, int* missing) {
  if (!A || !d_dinv) return fail(GIPB200_ERR_ARG, "bad arguments");
  DevBuf<int> m;
  GIPB_TRY(m.alloc(1));
  GIPB_TRY(m.zero());
  if (A->S.nrows > 0) {
    int b;
    GIPB_TRY(grid_blocks(256, A->S.nrows, 1, 0, &b));
    k_inv_diag<<<b, 256>>>(A->S.nrows, A->S.rowptr.p, A->S.csr_col.p, A->S.csr_val.p, d_dinv, m.p);
    GIPB_LAUNCH_CHECK();
  }
  int h = 0;
  GIPB_CUDA(cudaMemcpy(&h, m.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (missing) *missing = h;
  return GIPB200_OK;
}

}  // extern "C"
