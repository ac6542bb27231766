// Smoothed-aggregation algebraic multigrid: an FP32 V-cycle used as the preconditioner of
// the mixed form's inner CG (an addition beyond GIP, whose solver is Jacobi-PCG).
#pragma once

#include <cstdlib>

#include <cuda_fp16.h>

#include <memory>
#include <vector>

#include "internal.cuh"

namespace gipb200 {

struct PcgScalars;

// An AMG operator in one precision: sliced (SELL-32, a thread per row) when its rows are
// short, CSR with `lanes` threads per row when they are long (restrictions, coarse
// Galerkin operators), where a thread per row would walk dozens of padded slots alone.
template <typename T>
struct SellT {
  int nrows = 0, ncols = 0, nslices = 0;
  long long nslots = 0, nnz = 0;
  DevBuf<long long> sptr;
  DevBuf<int> col;
  DevBuf<T> val;
  int lanes = 0;               // > 0: CSR form (rp, col, val) with this many threads per row
  DevBuf<int> rp;
  bool half = false;           // values stored in FP16 (hval) instead of T (val)
  DevBuf<__half> hval;
  // 16-bit columns: column = cbase[row] + dcol[k], cbase the row's smallest column (every
  // row's columns span at most 65536; in the sliced form 0xffff marks padding slots)
  int pipe = 0;                // sliced FP32 form: 1 = software-pipelined product (k_amg_spmv_pf)
  bool short_cols = false;
  DevBuf<unsigned short> dcol;
  DevBuf<int> cbase;
  SellView<T> view() const { return {nrows, nslices, sptr.p, col.p, val.p}; }
  SellView<__half> hview() const { return {nrows, nslices, sptr.p, col.p, hval.p}; }
};

// One product of the FP32 cycle's small levels as the coarse-tail kernel runs it.
enum {
  kTailDense = 0,
  kTailSellResid,
  kTailSellSmooth,
  kTailSellRestrict,
  kTailSellProlong,
  kTailCsrResid,
  kTailCsrSmooth,
  kTailCsrRestrict,
  kTailCsrProlong
};
struct TailOp {
  int form;        // kTail*
  int lanes;       // CSR threads per row
  int nrows, nslices;
  const long long* sptr;
  const int* rp;
  const int* col;
  const void* val;  // float or __half (dense: float)
  const float* x;
  const float* b;
  const float* dinv;
  const float* xs;
  float* y;
  int level, kind;  // cycle position (profiling)
  double bytes;
};

// The mixed form's packed FP32 operator (see CompressedOp), for the V-cycle's level-0
// products.  on = false: use the plain sliced view.
struct PackedView {
  bool on = false;
  int nib = 4, slots = 8;
  const uint4* delta = nullptr;
  const void* idx = nullptr;
  const int* base = nullptr;
  const unsigned char* plain = nullptr;
  const float* table = nullptr;
};

// Per-kernel timing of V-cycles (profiling only): an event is recorded before every
// kernel and one after the last, and each kernel is tagged with its level, its kind
// (GIPB200_CYCLE_*) and its algorithmic bytes.
struct CycleTrace {
  std::vector<cudaEvent_t> ev;
  std::vector<int> level, kind, form;
  std::vector<double> bytes;
  bool captured = false;  // record into a graph being captured (external event nodes)
  int mark(cudaStream_t s, int lvl, int knd, double by, int frm);  // before a kernel
  int close(cudaStream_t s);                              // after the last one
  ~CycleTrace();
};

template <typename T>
struct AmgLevel {
  int n = 0;
  SellT<T> A;             // the level's operator (level 0: the solver's own operator)
  SellT<T> P, R;          // prolongation (n x n_next) and restriction (n_next x n)
  DevBuf<T> dinv;         // omega / a_ii of the Jacobi smoother
  DevBuf<T> b, x, t;      // right-hand side (levels >= 1), iterate, work / smoothed iterate
};

// T = float: preconditioner of the mixed form's FP32 CG; T = double: of the FP64 CG.
template <typename T>
struct AmgT {
  std::vector<std::unique_ptr<AmgLevel<T>>> lv;
  int nc = 0;             // coarsest size: solved with a dense (pseudo-)inverse
  DevBuf<T> cinv;         // nc x nc, row-major
  double op_complexity = 0.0, setup_s = 0.0;
  // Level 0 has a unit diagonal (the Jacobi-scaled operator, to within 10%): its smoother
  // is the constant weight omega0 = w, so the cycle never forms x0 = omega0 r (the residual
  // gathers r and scales the product) and reads no diagonal.  A fixed symmetric smoother
  // like the per-row one, so the cycle stays a symmetric positive definite operator.
  bool unit0 = false;
  // Levels >= 1 of at most kFoldRows unknowns fold their Jacobi start x = D^-1 b into the
  // kernels that gather it (GIPB200_AMG_NO_FOLD=1: a separate kernel forms it everywhere).
  // On small levels the saved launch wins; on a level of millions of unknowns the second
  // gather per nonzero costs more than the separate pass (24 against 10 us on the 2.1M
  // unknowns of the 256^3 cavity's level 1).
  static constexpr int kFoldRows = 1 << 19;
  bool fold_coarse = getenv("GIPB200_AMG_NO_FOLD") == nullptr;
  bool folds(int l) const { return l > 0 && fold_coarse && lv[l]->n <= kFoldRows; }
  double omega0 = 0.0;
  // Level 0's residual position in aggregate order (empty: written in row order); the
  // level-0 restriction's columns are numbered in that order.
  DevBuf<int> perm0;
  // Coarse tail (FP32 cycle, GIPB200_AMG_TAIL=<CTAs per SM>): levels tail_from.. (at most
  // kTailRows unknowns each, all folding their Jacobi starts) run as one cooperative launch
  // of tail_grid CTAs; tail_from < 0: one kernel per product (the default).
  static constexpr int kTailRows = 1 << 19;
  int tail_from = -1, tail_grid = 0, tail_nops = 0;
  DevBuf<TailOp> tail_ops;
  DevBuf<unsigned> tail_bar;
  double tail_bytes = 0.0;
  int build_tail(cudaStream_t s);
  int reset_tail(cudaStream_t s) const;

  // Hierarchy of the n x n operator (host CSR, FP64 values; columns < n), near-null
  // vector z.  singular: the operator annihilates z (pinned-Neumann inner system), so the
  // coarsest level is inverted on the complement of z.  x0_len: length of level 0's
  // iterate, at least the number of columns the level-0 operator given to enqueue gathers
  // from (its entries past n stay zero).
  int build(int n, const int* rp, const int* ci, const double* v, const double* z, bool singular,
            int x0_len, cudaStream_t s);
  // z0 = M r with the level-0 operator A0; the last kernel reduces r.z and sets the CG's
  // beta = (r.z) / (previous r.z) (0 when `first` or when no previous r.z is stored) and
  // stores r.z in S.
  int enqueue(SellView<T> A0, const T* r, T* z0, PcgScalars* S, ReduceScratch rs, int first,
              cudaStream_t s, const PackedView* pk = nullptr, CycleTrace* tr = nullptr,
              double a0_stream_bytes = 0.0) const;
  // Algorithmic bytes of one V-cycle: every operator's stored words once per use and every
  // vector read or written once per kernel; level 0's operator stream is given (packed or
  // plain, the caller's operator).
  double cycle_bytes(double a0_stream_bytes) const;
};

// Stored bytes one product streams from an AMG operator.
// The kernel form of a product with operator M (GIPB200_FORM_*).
template <typename T>
int product_form(const SellT<T>& M) {
  if (M.lanes > 0) return GIPB200_FORM_CSR;
  return (M.pipe && !M.short_cols) ? GIPB200_FORM_PIPELINED : GIPB200_FORM_SLICED;
}

template <typename T>
double stream_bytes(const SellT<T>& M) {
  const double w = M.half ? 2.0 : (double)sizeof(T);
  if (M.lanes > 0)
    return (double)M.nnz * ((M.short_cols ? 2.0 : 4.0) + w) + (M.nrows + 1.0) * 4.0 +
           (M.short_cols ? 4.0 * M.nrows : 0.0);
  return (double)M.nslots * ((M.short_cols ? 2.0 : 4.0) + w) + (M.nslices + 1.0) * 8.0 +
         (M.short_cols ? 4.0 * M.nrows : 0.0);
}

using Amg = AmgT<float>;
using Amg64 = AmgT<double>;

}  // namespace gipb200
