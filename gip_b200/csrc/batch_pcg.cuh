// Persistent batched pressure solve: one cooperative launch runs the mixed Jacobi-PCG of
// every instance of a batch (batch_pcg.cu).
#pragma once

#include "pcg.cuh"

namespace gipb200 {

constexpr int kBatchGroupMax = 1024;  // CTAs of one instance's group
constexpr int kBatchWidth = 8;        // partial sums per group reduction (slots)

// One instance's solve as the persistent kernel reads it (device copy, one per instance).
// The arrays are the instance's own mixed-form solver buffers (Pcg), so the history and
// result kernels of the instance read the outcome where the single-instance solve leaves
// it.
struct BatchSolve {
  SellView<double> L;   // FP64 operator of the true residual
  SellView<float> A;    // FP32 Jacobi-scaled operator S L S (pin removed), plain sliced
  const double* scale;  // S = 1/sqrt(L_ii)
  const double* b;
  double* x;
  const double* x0;
  float* r;             // scaled FP32 residual
  float* p[2];          // direction buffers: iteration k reads p[k&1], writes the other
  float* Ap;
  float* y;             // FP32 correction, folded into x at each replacement
  PcgScalars* S;        // written once, by the group's first CTA, when the solve ends
  double* part;         // group partial sums: [2 parities][kBatchWidth][kBatchGroupMax]
  unsigned* bar;        // group barrier arrivals (zero at launch)
  double tol, delta, pin_val;
  int n, n_all, maxit, max_outer, pin_row;
  int cta0, ncta;       // the instance's CTAs: [cta0, cta0 + ncta)
  int count_launch;     // 1 on the instance whose step history counts the launch
  // the packed FP32 operator (pk_nib = 4 or 8; 0: the plain sliced layout only)
  int pk_nib;
  const uint4* pk_delta;
  const void* pk_idx;
  const int* pk_base;
  const unsigned char* pk_plain;
  const float* pk_table;
};

// Launch shape of the persistent kernel: threads per CTA (128, 256 or 512), rows per
// warp pass (32: one slice of 32 rows per warp; 64: two slices in flight) and resident
// threads per SM it is compiled for (1024: 64 registers a thread; 1536: 40, a few spilled).
struct BatchShape {
  int block = 256;
  int rows_per_warp = 32;
  int threads_per_sm = 1024;
};

bool batch_shape_valid(const BatchShape& sh);
// CTAs of shape `sh` that are resident at once on the current device (the cooperative
// launch's grid limit).
int batch_pcg_capacity(const BatchShape& sh, int* ctas);
// One cooperative launch of `grid` CTAs; owner[c] = the instance of CTA c (-1: idle).
// *err becomes nonzero when a group barrier gave up waiting.
int batch_pcg_launch(const BatchShape& sh, int grid, const BatchSolve* inst, const int* owner,
                     int* err, cudaStream_t s);

// Runs one persistent launch whose group barrier can never complete and reports
// GIPB200_ERR_TIMEOUT in *h_status when the bounded wait gave up as designed.
int batch_pcg_check_timeout(cudaStream_t s, int* h_status);

}  // namespace gipb200
