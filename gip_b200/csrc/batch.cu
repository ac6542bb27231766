// Batched cavities: one CUDA graph per timestep with one parallel branch per instance.
// Each branch is that instance's fused step (dns.cu) with its own conditional PCG loops
// (pcg.cu), so instances converge independently inside the same launch.
#include <vector>

#include "dns.cuh"

namespace gipb200 {

struct Batch {
  std::vector<gipb200_dns> inst;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> joins;
  cudaEvent_t fork = nullptr;
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~Batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto s : streams) cudaStreamDestroy(s);
    for (auto e : joins) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (cap) cudaStreamDestroy(cap);
    for (auto d : inst) gipb200_dns_destroy(d);
  }
  int capture();
};

int Batch::capture() {
  GIPB_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
  int st = GIPB200_OK;
  cudaError_t e = cudaEventRecord(fork, cap);
  for (size_t i = 0; i < inst.size() && st == GIPB200_OK && e == cudaSuccess; ++i) {
    e = cudaStreamWaitEvent(streams[i], fork, 0);
    if (e != cudaSuccess) break;
    Dns& E = inst[i]->E;
    const long long before = E.launches;
    st = E.enqueue_step(streams[i], false);
    E.graph_kernels = E.launches - before;
    E.launches = before;
    if (st != GIPB200_OK) break;
    e = cudaEventRecord(joins[i], streams[i]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(cap, joins[i], 0);
  }
  cudaGraph_t g = nullptr;
  cudaError_t ce = cudaStreamEndCapture(cap, &g);
  if (st != GIPB200_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (e != cudaSuccess || ce != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(GIPB200_ERR_CUDA, "batch capture failed: %s",
                cudaGetErrorString(e != cudaSuccess ? e : ce));
  }
  graph = g;
  GIPB_CUDA(cudaGraphInstantiate(&exec, graph, 0));
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
    recapture = recapture || E.capacity != cap_before || (E.exec == nullptr && E.graph == nullptr &&
                                                          false);
    if (!E.started) {
      GIPB_TRY(E.enqueue_initial_dt(s));
      E.started = true;
    }
  }
  if (recapture && B.exec) {
    cudaGraphExecDestroy(B.exec);
    cudaGraphDestroy(B.graph);
    B.exec = nullptr;
    B.graph = nullptr;
  }
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

}  // extern "C"
