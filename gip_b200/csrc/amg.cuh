// Smoothed-aggregation algebraic multigrid: an FP32 V-cycle used as the preconditioner of
// the mixed form's inner CG (an addition beyond GIP, whose solver is Jacobi-PCG).
#pragma once

#include <memory>
#include <vector>

#include "internal.cuh"

namespace gipb200 {

struct PcgScalars;

// FP32 sliced operator without the extra copies a Sell keeps (no FP64 values, no CSR).
struct Sell32 {
  int nrows = 0, ncols = 0, nslices = 0;
  long long nslots = 0, nnz = 0;
  DevBuf<long long> sptr;
  DevBuf<int> col;
  DevBuf<float> val;
  SellView<float> view() const { return {nrows, nslices, sptr.p, col.p, val.p}; }
};

struct AmgLevel {
  int n = 0;
  Sell32 A;               // the level's operator (level 0: the solver's own FP32 operator)
  Sell32 P, R;            // prolongation (n x n_next) and restriction (n_next x n)
  DevBuf<float> dinv;     // omega / a_ii of the Jacobi smoother
  DevBuf<float> b, x, t;  // right-hand side (levels >= 1), iterate, work / smoothed iterate
};

struct Amg {
  std::vector<std::unique_ptr<AmgLevel>> lv;
  int nc = 0;             // coarsest size: solved with a dense (pseudo-)inverse
  DevBuf<float> cinv;     // nc x nc, row-major
  double op_complexity = 0.0, setup_s = 0.0;
  int blocks = 1;
  long long kernels_per_cycle = 0;

  // Hierarchy of the n x n operator (host CSR, FP64 values; columns < n), near-null
  // vector z.  singular: the operator annihilates z (pinned-Neumann inner system), so the
  // coarsest level is inverted on the complement of z.
  int build(int n, const int* rp, const int* ci, const double* v, const double* z, bool singular,
            cudaStream_t s);
  // z0 = M r with the level-0 operator A0; the last kernel reduces r.z and sets the CG's
  // beta = (r.z) / (previous r.z) (0 on the first cycle of a solve) and r.z in S.
  int enqueue(SellView<float> A0, const float* r, float* z0, PcgScalars* S, ReduceScratch rs,
              cudaStream_t s) const;
};

}  // namespace gipb200
