// Device-resident Jacobi-PCG shared by the PCG handle and the timestep engine.
#pragma once

#include <memory>

#include "amg.cuh"
#include "internal.cuh"

namespace gipb200 {

// Scalars of one solve, in device memory (kernels read and write them; the host only
// reads them after the solve).
struct PcgScalars {
  double rz;        // r.z (FP64 modes) / scaled r.r (inner solve of MIXED)
  double pAp;
  double alpha, beta;
  double rr;        // r.r (FP64 modes: recursive residual; MIXED: true residual)
  double bb;        // b.b
  double rz_target; // MIXED: inner stop level
  int iter;         // iterations of the current (inner) solve
  int done;         // FP64 modes: solve finished; MIXED: outer loop finished
  int inner_done;   // MIXED: current inner solve finished
  int status;       // GIPB200_OK or GIPB200_ERR_BREAKDOWN / NOT_CONVERGED
  int outer;        // MIXED: refinement cycles done
  int total_inner;  // MIXED: inner iterations summed over cycles
  int kernels;      // MIXED: PCG kernel launches of this solve, early exits included
  int pad1;
  double rsum;      // MIXED: sum of the FP64 residual (pinned-Neumann deflation)
  double kappa_c;   // MIXED: sum(r)/pin of the current segment
  double kappa;     // MIXED: constant added to x at the next replacement
  double maxr2;     // MIXED: largest FP32 r^.r^ since the last replacement
  double trig;      // MIXED: FP32 r^.r^ level that predicts convergence
  int upd;          // MIXED: replace the FP32 residual by the FP64 one now
  int pad2;
};

// The FP32 operator of the mixed form, compressed without loss.  Each row's nonzeros
// are sorted by column (the FP32 operator only: L keeps GIP's order for the FP64
// residual).  A slice of 32 rows whose rows have at most 8 slots and whose column spread
// per slot fits 16 bits is packed per row: eight 16-bit column deltas (one 16-byte load)
// from a per-(slice, slot) base, and eight value-table indices (4 bits when the operator
// has at most 15 distinct nonzero values, else 8 bits; index 0 = 0.0f, padding and
// stored zeros).  Other slices stay in the plain sliced layout.
struct CompressedOp {
  bool enabled = false;
  int index_bits = 0;            // 4 or 8
  int slots = 8;                 // 7: no packed row uses the eighth slot
  DevBuf<uint4> delta;           // per row (nslices * 32)
  DevBuf<unsigned> idx4;         // per row, 8 x 4 bits
  DevBuf<uint2> idx8;            // per row, 8 x 8 bits
  DevBuf<int> base;              // per slice, 8 slots
  DevBuf<unsigned char> plain;   // per slice
  DevBuf<float> table;           // 16 or 256 entries
  int ntable = 0;
  double compressed_fraction = 0.0;  // share of L's slots in packed slices
  double bytes_per_launch = 0.0;     // stored bytes the kernel streams (+ vectors)
};

struct Pcg {
  const Sell* L = nullptr;   // not owned
  int n = 0;                 // unknowns = L rows (GIP's inner range)
  int n_all = 0;             // vector length (inner + ghost cells)
  gipb200_pcg_params prm{};
  DevBuf<double> dinv, p, Ap, r;
  // MIXED
  DevBuf<float> lhat;        // S L S values in L's slice structure, rows sorted by column
  DevBuf<int> col32;         // their columns (-1: padding and dropped ghost columns)
  DevBuf<double> scale;      // S = 1/sqrt(L_ii)
  DevBuf<float> p32, Ap32, r32, y32;
  DevBuf<float> p32b;        // second direction buffer: each SpMV reads one, writes the other
  // AMG path: A p by the recurrence A z + beta A p_in (one gather per nonzero); the two
  // product buffers alternate like the direction buffers
  bool rec = false;
  DevBuf<float> Ap32b;
  CompressedOp cop;
  // AMG preconditioner of the FP32 inner CG (MIXED with GIPB200_PRECOND_AMG)
  std::unique_ptr<Amg> amg;
  DevBuf<float> z32;         // preconditioned residual
  int build_amg(cudaStream_t s);
  // AMG preconditioner of the FP64 CG (TOL with GIPB200_PRECOND_AMG)
  std::unique_ptr<Amg64> amg64;
  DevBuf<double> z64;
  int build_amg64(cudaStream_t s);
  // Algorithmic bytes of one PCG iteration (CG products and updates, plus the V-cycle with
  // AMG) and of one MIXED residual replacement (FP64 residual and the fold of y into x).
  double iteration_bytes() const;
  double replacement_bytes() const;
  int sort_fp32_rows(cudaStream_t s);
  // Packed FP64 residual of the mixed form (r = b - L x from the packed operator's columns
  // and a table of L's values): L's inner values in the sorted slot order and its ghost
  // entries (host, set-up only), then on the device the value indices, the table, the
  // ghost rows and the right-hand side less the ghost part (constant during a solve).
  std::vector<double> lval_sorted;
  std::vector<int> ghost_rows, ghost_rp, ghost_col;
  std::vector<double> ghost_val;
  bool lpacked = false;
  DevBuf<unsigned> lidx4;      // per row, 8 x 4 bits into ltable
  DevBuf<double> ltable;       // 16 entries, index 0 = 0.0
  DevBuf<int> d_ghost_rows, d_ghost_rp, d_ghost_col;
  DevBuf<double> d_ghost_val;
  DevBuf<double> bprime;       // b - L_ghost x_ghost
  void launch_pcg_update(double* x, cudaStream_t s);
  int build_compressed(cudaStream_t s);
  SellView<float> a32() const {
    return {L->nrows, L->nslices, L->sptr.p, col32.p, lhat.p, L->uslots};
  }
  PackedView packed() const {
    PackedView v;
    v.on = cop.enabled;
    v.nib = cop.index_bits;
    v.slots = cop.slots;
    v.delta = cop.delta.p;
    v.idx = cop.index_bits == 4 ? (const void*)cop.idx4.p : (const void*)cop.idx8.p;
    v.base = cop.base.p;
    v.plain = cop.plain.p;
    v.table = cop.table.p;
    return v;
  }
  // Pinned-Neumann structure of L (every row sums to zero except one pinned row p with
  // sum pin > 0): the FP32 inner solve then runs on the pure-Neumann part and the
  // constant mode is restored exactly from the pin equation.
  int pin_row = -1;
  double pin_val = 0.0;
  // scalars and reduction scratch
  DevBuf<PcgScalars> sc;
  DevBuf<double> partials;
  DevBuf<unsigned> ticket;
  ReduceScratch rs{};
  PcgScalars* h_sc = nullptr;  // pinned
  int blocks_spmv = 1, blocks_vec = 1;
  // launch shape overrides (autotuning): 0 = default grid
  int set_launch(int spmv_blocks, int vec_blocks);
  long long launches = 0;      // kernels enqueued by this solver (host count)
  // streams that capture the bodies of the conditional while-nodes
  cudaStream_t body_stream[2] = {nullptr, nullptr};

  ~Pcg();
  int init(const Sell* L, int n_all, const gipb200_pcg_params& prm, cudaStream_t s);
  // Enqueues a whole solve.  FIXED mode never synchronises the host.  TOL and MIXED
  // poll the device's stop flag every `poll` iterations when host_sync is true; with
  // host_sync false they run exactly their iteration caps (masked after convergence).
  int enqueue(const double* b, double* x, const double* x0, cudaStream_t s, bool host_sync);
  int result(cudaStream_t s, gipb200_pcg_result* out);
  // Times `reps` launches of the SpMV+dot kernel of the current mode on scratch scalars.
  int time_spmv(int mixed, int reps, cudaStream_t s, double* avg_ms, double* bytes);
  // Times `reps` launches of the mixed form's FP32 update kernel (scratch scalars, alpha 0).
  int time_update(int reps, cudaStream_t s, double* avg_ms, double* bytes);
  // Per-kernel profile of `reps` V-cycles on the current residual (scratch scalars).
  int profile_vcycle(int reps, cudaStream_t s, int cap, int* n_kernels, int* level, int* kind,
                     double* ms, double* bytes);
  std::vector<int> cycle_forms;  // kernel forms of the last profiled cycle (GIPB200_FORM_*)
  int vcycle_forms(int cap, int* n_kernels, int* h_form) const;

 private:
  int enqueue_fp64(const double* b, double* x, const double* x0, cudaStream_t s, bool host_sync);
  int enqueue_mixed(const double* b, double* x, const double* x0, cudaStream_t s, bool host_sync);
  int read_flag(cudaStream_t s, int which, int* v);
  int enqueue_fp64_graph(const double* b, double* x, const double* x0, cudaStream_t s);
  int enqueue_mixed_graph(const double* b, double* x, const double* x0, cudaStream_t s);
  int launch_mixed_residual(const double* b, const double* x, int first, cudaStream_t s,
                            int use_cond, cudaGraphConditionalHandle h);
};

}  // namespace gipb200

struct gipb200_pcg_s {
  gipb200::Pcg P;
};
