// The fused timestep engine shared by the C ABI (dns.cu) and the adjoint (adjoint.cu).
#pragma once

#include <string>
#include <vector>

#include "pcg.cuh"

namespace gipb200 {

struct DnsScalars {
  double dt, sigma, time;
  int step;
  int started;
};

struct DnsHistory {
  double* time;
  double* dt;
  double* massr;
  int* iters;
  double* rr;
  int* outer;
  int* kernels;  // kernels the step launched (early exits included)
  unsigned long long* stamps;  // kPhaseMarks device times per step (phase stamps on)
  int capacity;
  int stamp_kernels;  // phase-stamp kernels each step adds (0 when stamps are off)
};

// Device timestamps at the step's 8 phase boundaries (kPhaseMarks per step, ns).
constexpr int kPhaseMarks = 8;

// SFx, SFy and SFz merged row by row for the mass-flux kernel: a face row holds its SFx
// entries, then its SFy entries, then its SFz entries (each in stored order), with the
// three counts per face.  A face of a structured grid has entries in one of the three
// only, so the merged slices have no padding where three separate ones are two-thirds
// padding.  Each operator's row sum keeps its own order, so results are unchanged.
struct FaceOps3 {
  bool on = false;
  bool single = false;               // every face's entries belong to one operator only
  Sell S;                            // merged rows (NF rows)
  DevBuf<unsigned short> cnt;        // per face: cx | cy << 4 | cz << 8
};

struct Dns {
  int N = 0, NO = 0, NF = 0;
  gipb200_dns_params prm{};
  Sell D, Ec, L, Lb, Mx, My, Mz, Mres, Gx, Gy, Gz, SFx, SFy, SFz, SO;
  FaceOps3 SF3;
  double setup_s[4] = {0, 0, 0, 0};  // create time: renumbering, operators, solver, total
  // Ec with its rows in C's slot order (row t = the Ec row of the nonzero stored in slot t
  // of D's sliced layout; padding slots are empty rows), so C's values are written
  // contiguously instead of through D's position map.
  bool ec_slot = false;
  int ec_rows = 0;
  DevBuf<int> ec_rp, ec_col;
  DevBuf<double> ec_val;         // (empty when the value table is used)
  int ec_ntab = 0;               // > 0: values through ec_vtab[ec_vidx[e]]
  DevBuf<unsigned char> ec_vidx;
  DevBuf<double> ec_vtab;
  // the phase kernels' operators all tabled (each kernel reads its operators one way)
  bool tab_d() const { return D.ntab > 0; }
  bool tab_m() const { return Mx.ntab > 0 && My.ntab > 0 && Mz.ntab > 0; }
  int value_tables() const {
    return (tab_d() ? 1 : 0) + (tab_m() ? 1 : 0) + (Mres.ntab > 0 ? 1 : 0) + (ec_ntab > 0 ? 1 : 0);
  }
  DevBuf<double> cval;
  DevBuf<double> u, v, w, dxs, ax, ay, az, ax0, ay0, az0, rhs, p, p0, gpx, gpy, gpz, temp, mf;
  Pcg pcg;
  DevBuf<DnsScalars> sc;
  DevBuf<double> h_time, h_dt, h_massr, h_rr;
  DevBuf<int> h_iters, h_outer, h_kernels;
  DevBuf<unsigned long long> h_stamps;  // capacity x kPhaseMarks, 0 = not recorded
  bool stamps_on = false;               // stamp the phase boundaries on the device
  int capacity = 0;
  DevBuf<double> partials;
  DevBuf<unsigned> ticket;
  ReduceScratch rs{};
  int steps_enqueued = 0;
  bool started = false;
  cudaStream_t cap_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int blocks_cells = 1, blocks_faces = 1, blocks_owned = 1, blocks_vec = 1;
  // per-kernel grids: the shared sizes above lowered to what stays resident in one wave
  struct {
    int convdiff = 1, ab2 = 1, rhs = 1, gradcorr = 1, massflux = 1, massr = 1, cfl = 1;
  } grid;
  // internal renumbering (reorder): external index e lives at internal perm[e]
  bool reordered = false;
  DevBuf<int> perm_c, perm_f;
  DevBuf<double> staging;
  long long launches = 0;        // kernels launched (graph launches count their kernels)
  long long graph_kernels = 0;   // kernels in the captured step graph
  cudaEvent_t* phase_events = nullptr;  // when set: recorded at the step's phase boundaries
  // device-side snapshot of the whole timestep state (checkpoint / resume)
  std::vector<DevBuf<double>*> snap;
  DevBuf<DnsScalars> snap_sc;
  int snap_steps = -1;
  // prescribed time steps (adjoint runs): dt of step k is dt_seq[min(k, len-1)]
  DevBuf<double> dt_seq;
  int dt_seq_len = 0;

  ~Dns() {
    for (auto* b : snap) delete b;
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (cap_stream) cudaStreamDestroy(cap_stream);
  }
  DnsHistory history() const {
    return {h_time.p,    h_dt.p,     h_massr.p, h_iters.p,
            h_rr.p,      h_outer.p,  h_kernels.p, h_stamps.p,
            capacity,    stamps_on ? kPhaseMarks : 0};
  }
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  int grow_history(int need, cudaStream_t s);
  // Algorithmic bytes of each phase of one timestep, in gipb200_dns_step_phases order
  // (the PCG entry is 0: its bytes are iterations x iteration_bytes + replacements).
  void phase_bytes(double out[7]) const;
  // part 0: the whole step; 1: the phases before the pressure solve; 2: those after it
  // (a batch runs the solves of all its instances in between).
  int enqueue_step(cudaStream_t s, bool host_sync, int part = 0);
  int enqueue_initial_dt(cudaStream_t s);
  double* field(const std::string& name, int* n);
};

int dns_init(Dns& E, const gipb200_dns_ops* ops, const double* h_u, const double* h_v,
             const double* h_w, const double* h_dxs, const gipb200_dns_params* prm);
int dns_advance(Dns& E, int nsteps, cudaStream_t s);
int check_dns_ops(const gipb200_dns_ops* ops);

}  // namespace gipb200

struct gipb200_dns_s {
  gipb200::Dns E;
};
