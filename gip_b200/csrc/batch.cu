// Batched cavities: one CUDA graph per timestep.  By default each instance's whole step is
// a parallel branch (fork/join events) with its own conditional PCG loops (pcg.cu), so
// instances converge independently inside the same launch.  With the persistent solver the
// branches stop before the pressure solve, one cooperative launch (batch_pcg.cu) solves
// every instance's pressure system with a CTA group per instance, and a second set of
// branches finishes the steps.
#include <algorithm>
#include <cmath>
#include <vector>

#include "batch_pcg.cuh"
#include "dns.cuh"

namespace gipb200 {

struct Batch {
  std::vector<gipb200_dns> inst;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> joins;
  cudaEvent_t fork = nullptr, fork2 = nullptr;
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // persistent pressure solve
  bool persistent = false;
  BatchShape shape;
  int grid = 0;                   // CTAs of the launch (all resident at once)
  std::vector<int> ncta;          // per instance
  std::vector<double> weights;    // per instance: expected work
  DevBuf<BatchSolve> d_inst;
  DevBuf<int> d_owner;
  DevBuf<unsigned> d_bar;
  DevBuf<double> d_part;
  DevBuf<int> d_err;
  ~Batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto s : streams) cudaStreamDestroy(s);
    for (auto e : joins) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (fork2) cudaEventDestroy(fork2);
    if (cap) cudaStreamDestroy(cap);
    for (auto d : inst) gipb200_dns_destroy(d);
  }
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  int branches(cudaEvent_t from, int part, int* st);
  int capture();
  int layout(cudaStream_t s);
};

// Every instance's step (part 0) or part of it as a branch from event `from`, joined back
// into the capture stream.
int Batch::branches(cudaEvent_t from, int part, int* st) {
  GIPB_CUDA(cudaEventRecord(from, cap));
  for (size_t i = 0; i < inst.size(); ++i) {
    GIPB_CUDA(cudaStreamWaitEvent(streams[i], from, 0));
    Dns& E = inst[i]->E;
    const long long before = E.launches;
    *st = E.enqueue_step(streams[i], false, part);
    E.graph_kernels += E.launches - before;
    E.launches = before;
    if (*st != GIPB200_OK) return *st;
    GIPB_CUDA(cudaEventRecord(joins[i], streams[i]));
    GIPB_CUDA(cudaStreamWaitEvent(cap, joins[i], 0));
  }
  return GIPB200_OK;
}

int Batch::capture() {
  for (auto d : inst) d->E.graph_kernels = 0;
  GIPB_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
  int st = GIPB200_OK;
  int rc = [&]() -> int {
    if (!persistent) return branches(fork, 0, &st);
    GIPB_TRY(branches(fork, 1, &st));
    GIPB_CUDA(cudaMemsetAsync(d_bar.p, 0, inst.size() * sizeof(unsigned), cap));
    GIPB_TRY(batch_pcg_launch(shape, grid, d_inst.p, d_owner.p, d_err.p, cap));
    inst[0]->E.graph_kernels += 1;
    return branches(fork2, 2, &st);
  }();
  cudaGraph_t g = nullptr;
  cudaError_t ce = cudaStreamEndCapture(cap, &g);
  if (rc != GIPB200_OK || st != GIPB200_OK) {
    if (g) cudaGraphDestroy(g);
    return rc != GIPB200_OK ? rc : st;
  }
  if (ce != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(GIPB200_ERR_CUDA, "batch capture failed: %s", cudaGetErrorString(ce));
  }
  graph = g;
  GIPB_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  return GIPB200_OK;
}

// CTA groups of the persistent solve: the grid is every CTA resident at once; instance i
// gets a share proportional to weights[i], at least one CTA and no more than it has slices
// for (nor kBatchGroupMax).  Writes the owner table and the per-instance descriptors.
int Batch::layout(cudaStream_t s) {
  const int ni = (int)inst.size();
  int capacity = 0;
  GIPB_TRY(batch_pcg_capacity(shape, &capacity));
  if (capacity < ni)
    return fail(GIPB200_ERR_ARG, "%d instances but only %d resident CTAs", ni, capacity);
  grid = capacity;
  const int warps = shape.block / 32, spw = shape.rows_per_warp / 32;
  std::vector<int> cap_i(ni);
  double wsum = 0.0;
  for (int i = 0; i < ni; ++i) {
    const Pcg& P = inst[i]->E.pcg;
    const int slices = std::max(P.L->nslices, 1);
    cap_i[i] = std::max(1, std::min(kBatchGroupMax, (slices + warps * spw - 1) / (warps * spw)));
    wsum += std::max(weights[i], 0.0);
  }
  ncta.assign(ni, 1);
  int used = ni;
  if (wsum > 0.0) {
    used = 0;
    for (int i = 0; i < ni; ++i) {
      const double share = (double)grid * std::max(weights[i], 0.0) / wsum;
      ncta[i] = std::max(1, std::min(cap_i[i], (int)std::floor(share)));
      used += ncta[i];
    }
    while (used > grid) {  // rounding up to one CTA each can overshoot: trim the largest
      int k = (int)(std::max_element(ncta.begin(), ncta.end()) - ncta.begin());
      ncta[k] -= 1;
      used -= 1;
    }
  }
  std::vector<int> owner(grid, -1);
  std::vector<BatchSolve> h(ni);
  int c = 0;
  for (int i = 0; i < ni; ++i) {
    Dns& E = inst[i]->E;
    Pcg& P = E.pcg;
    BatchSolve& d = h[i];
    d.L = P.L->view();
    d.A = P.a32();
    d.scale = P.scale.p;
    d.b = E.rhs.p;
    d.x = E.p.p;
    d.x0 = E.p0.p;
    d.r = P.r32.p;
    d.p[0] = P.p32.p;
    d.p[1] = P.p32b.p;
    d.Ap = P.Ap32.p;
    d.y = P.y32.p;
    d.S = P.sc.p;
    d.part = d_part.p + (size_t)i * 2 * kBatchWidth * kBatchGroupMax;
    d.bar = d_bar.p + i;
    d.tol = P.prm.tol;
    d.delta = P.prm.inner_tol;
    d.pin_val = P.pin_val;
    d.n = P.n;
    d.n_all = P.n_all;
    d.maxit = P.prm.maxit;
    d.max_outer = P.prm.max_outer;
    d.pin_row = P.pin_row;
    d.cta0 = c;
    d.ncta = ncta[i];
    d.count_launch = (i == 0) ? 1 : 0;
    const PackedView pk = P.packed();
    d.pk_nib = pk.on ? pk.nib : 0;
    d.pk_delta = pk.delta;
    d.pk_idx = pk.idx;
    d.pk_base = pk.base;
    d.pk_plain = pk.plain;
    d.pk_table = pk.table;
    for (int k = 0; k < ncta[i]; ++k) owner[c + k] = i;
    c += ncta[i];
  }
  if (d_owner.n != (size_t)grid) GIPB_TRY(d_owner.alloc(grid));
  GIPB_CUDA(cudaMemcpyAsync(d_owner.p, owner.data(), (size_t)grid * sizeof(int),
                            cudaMemcpyHostToDevice, s));
  GIPB_CUDA(cudaMemcpyAsync(d_inst.p, h.data(), (size_t)ni * sizeof(BatchSolve),
                            cudaMemcpyHostToDevice, s));
  GIPB_CUDA(cudaStreamSynchronize(s));
  return GIPB200_OK;
}

}  // namespace gipb200

using namespace gipb200;

struct gipb200_batch_s {
  gipb200::Batch B;
};

extern "C" {

int gipb200_batch_create(int n, const gipb200_dns_ops* const* ops, const double* const* h_u,
                         const double* const* h_v, const double* const* h_w,
                         const double* const* h_dxs, const gipb200_dns_params* params,
                         gipb200_batch* out) {
  if (n <= 0 || !ops || !h_u || !h_v || !h_w || !h_dxs || !params || !out)
    return fail(GIPB200_ERR_ARG, "null argument or empty batch");
  *out = nullptr;
  gipb200_batch H = new (std::nothrow) gipb200_batch_s();
  if (!H) return fail(GIPB200_ERR_NOMEM, "host allocation failed");
  int st = [&]() -> int {
    Batch& B = H->B;
    for (int i = 0; i < n; ++i) {
      gipb200_dns d = nullptr;
      GIPB_TRY(gipb200_dns_create(ops[i], h_u[i], h_v[i], h_w[i], h_dxs[i], &params[i], &d));
      B.inst.push_back(d);
      cudaStream_t s;
      GIPB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      B.streams.push_back(s);
      cudaEvent_t e;
      GIPB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      B.joins.push_back(e);
    }
    GIPB_CUDA(cudaEventCreateWithFlags(&B.fork, cudaEventDisableTiming));
    GIPB_CUDA(cudaEventCreateWithFlags(&B.fork2, cudaEventDisableTiming));
    GIPB_CUDA(cudaStreamCreateWithFlags(&B.cap, cudaStreamNonBlocking));
    return GIPB200_OK;
  }();
  if (st != GIPB200_OK) {
    delete H;
    return st;
  }
  *out = H;
  return GIPB200_OK;
}

int gipb200_batch_destroy(gipb200_batch H) {
  delete H;
  return GIPB200_OK;
}

int gipb200_batch_instance(gipb200_batch H, int i, gipb200_dns* out) {
  if (!H || !out || i < 0 || i >= (int)H->B.inst.size()) return fail(GIPB200_ERR_ARG, "bad index");
  *out = H->B.inst[i];
  return GIPB200_OK;
}

int gipb200_batch_advance(gipb200_batch H, int nsteps, void* stream) {
  if (!H || nsteps < 0) return fail(GIPB200_ERR_ARG, "bad arguments");
  Batch& B = H->B;
  cudaStream_t s = as_stream(stream);
  // host-side preparation of every instance: history room, initial dt
  bool recapture = false;
  for (auto d : B.inst) {
    Dns& E = d->E;
    const int cap_before = E.capacity;
    GIPB_TRY(E.grow_history(E.steps_enqueued + nsteps, s));
    recapture = recapture || E.capacity != cap_before;
    if (!E.started) {
      GIPB_TRY(E.enqueue_initial_dt(s));
      E.started = true;
    }
  }
  if (recapture) B.drop_graph();
  if (!B.exec) {
    GIPB_CUDA(cudaStreamSynchronize(s));
    GIPB_TRY(B.capture());
  }
  for (int k = 0; k < nsteps; ++k) {
    GIPB_CUDA(cudaGraphLaunch(B.exec, s));
    for (auto d : B.inst) {
      d->E.launches += d->E.graph_kernels;
      d->E.steps_enqueued += 1;
    }
  }
  return GIPB200_OK;
}

int gipb200_batch_set_solver(gipb200_batch H, int persistent, int block, int rows_per_warp,
                             int threads_per_sm) {
  if (!H) return fail(GIPB200_ERR_ARG, "null batch");
  Batch& B = H->B;
  if (!persistent) {
    B.persistent = false;
    B.drop_graph();
    return GIPB200_OK;
  }
  BatchShape sh;
  sh.block = block;
  sh.rows_per_warp = rows_per_warp;
  sh.threads_per_sm = threads_per_sm > 0 ? threads_per_sm : 1024;
  if (!batch_shape_valid(sh))
    return fail(GIPB200_ERR_ARG,
                "block must be 128, 256 or 512, rows_per_warp 32 or 64, threads_per_sm 1024 "
                "or 1536");
  for (size_t i = 0; i < B.inst.size(); ++i) {
    const Pcg& P = B.inst[i]->E.pcg;
    if (P.prm.mode != GIPB200_PCG_MIXED || P.prm.precond != GIPB200_PRECOND_JACOBI)
      return fail(GIPB200_ERR_ARG,
                  "instance %zu: the persistent solve runs the mixed form with Jacobi only", i);
    if (P.n <= 0) return fail(GIPB200_ERR_ARG, "instance %zu has no unknowns", i);
  }
  const int ni = (int)B.inst.size();
  if (B.weights.size() != B.inst.size()) {
    B.weights.resize(ni);
    for (int i = 0; i < ni; ++i) {
      const double rows = B.inst[i]->E.pcg.n;
      B.weights[i] = rows * std::cbrt(rows);  // Jacobi-PCG iterations grow with the edge
    }
  }
  if (!B.d_inst.p) {
    GIPB_TRY(B.d_inst.alloc(ni));
    GIPB_TRY(B.d_bar.alloc(ni));
    GIPB_TRY(B.d_part.alloc((size_t)ni * 2 * kBatchWidth * kBatchGroupMax));
    GIPB_TRY(B.d_err.alloc(1));
    GIPB_TRY(B.d_err.zero(B.cap));
  }
  B.shape = sh;
  B.persistent = true;
  GIPB_TRY(B.layout(B.cap));
  B.drop_graph();  // the grid size is part of the captured launch
  return GIPB200_OK;
}

int gipb200_batch_balance(gipb200_batch H, const double* weights) {
  if (!H) return fail(GIPB200_ERR_ARG, "null batch");
  Batch& B = H->B;
  const int ni = (int)B.inst.size();
  if (weights) {
    for (int i = 0; i < ni; ++i)
      if (!(weights[i] >= 0.0) || !std::isfinite(weights[i]))
        return fail(GIPB200_ERR_ARG, "weight %d is negative or not finite", i);
    B.weights.assign(weights, weights + ni);
  } else {
    B.weights.clear();
  }
  if (!B.persistent) return GIPB200_OK;
  if (B.weights.empty()) {
    B.weights.resize(ni);
    for (int i = 0; i < ni; ++i) {
      const double rows = B.inst[i]->E.pcg.n;
      B.weights[i] = rows * std::cbrt(rows);
    }
  }
  // same grid and buffers: a captured graph reads the new tables at its next launch (none
  // may be running while they are rewritten)
  GIPB_CUDA(cudaDeviceSynchronize());
  return B.layout(B.cap);
}

int gipb200_batch_layout(gipb200_batch H, int* grid, int* h_ncta) {
  if (!H || !grid) return fail(GIPB200_ERR_ARG, "null argument");
  Batch& B = H->B;
  *grid = B.persistent ? B.grid : 0;
  if (h_ncta)
    for (size_t i = 0; i < B.inst.size(); ++i) h_ncta[i] = B.persistent ? B.ncta[i] : 0;
  return GIPB200_OK;
}

int gipb200_batch_solver_status(gipb200_batch H, void* stream, int* h_err) {
  if (!H || !h_err) return fail(GIPB200_ERR_ARG, "null argument");
  Batch& B = H->B;
  *h_err = 0;
  if (!B.d_err.p) return GIPB200_OK;
  cudaStream_t s = as_stream(stream);
  GIPB_CUDA(cudaMemcpyAsync(h_err, B.d_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  GIPB_CUDA(cudaStreamSynchronize(s));
  GIPB_CUDA(cudaMemsetAsync(B.d_err.p, 0, sizeof(int), s));
  return GIPB200_OK;
}

int gipb200_batch_check_bounded_wait(void* stream, int* h_status) {
  if (!h_status) return fail(GIPB200_ERR_ARG, "null status");
  return batch_pcg_check_timeout(as_stream(stream), h_status);
}

}  // extern "C"
