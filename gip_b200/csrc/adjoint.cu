// FP64 discrete adjoint of the fractional-step timestep (GIP_DNS.h:309-391) with the
// time steps frozen (the CFL step size is not differentiated).
//
// Objective: J = 1/2 sum_i vol_i (u_i^2 + v_i^2 + w_i^2) over the inner cells after the
// last step.  Parameters: the lid's ghost velocities (u on the given ghost cells) and the
// viscosity nu = s * nu0 (D = s * D_given).
//
// Forward step n (dt, sigma = 1/dt), as the engine runs it:
//   C = Ec mf;  a = D u - C u;  u* = u + 1.5dt a + (-0.5dt) a0;  a0' = a
//   rhs = sigma (Mx u* + My v* + Mz w*);  p = L^-1 rhs;  p_full = [p ; Lb p]
//   gp = G p_full;  u' = u* - dt/rho gp;  mf' = -dt SO p_full + dt SF gp + rho SF u'
// The backward applies the transposed chain with transposed operators built once on
// the host (CSR transposes), one adjoint Poisson solve per step with the same PCG
// (L is symmetric), and the convective adjoint dJ/dmf = -Ec^T z with
// z_k = sum_d abar_d[row k] u_d[col k] over D's nonzeros.
// Forward states are checkpointed every `checkpoint_every` steps and recomputed per
// segment during the backward sweep.
#include <math.h>

#include <algorithm>
#include <vector>

#include "device.cuh"
#include "dns.cuh"

namespace gipb200 {
namespace {

struct HostT {
  int nrows = 0, ncols = 0;
  std::vector<int> rp, col, map;  // map: source nonzero index of each entry
  std::vector<double> val;
};

// CSR transpose (counting sort); entries of a transposed row in ascending source row.
void transpose(const gipb200_host_csr& m, int ncols, HostT* t) {
  t->nrows = ncols;
  t->ncols = m.nrows;
  t->rp.assign((size_t)ncols + 1, 0);
  for (int k = 0; k < m.nnz; ++k) t->rp[m.col[k] + 1]++;
  for (int j = 0; j < ncols; ++j) t->rp[j + 1] += t->rp[j];
  t->col.resize((size_t)m.nnz);
  t->val.resize((size_t)m.nnz);
  t->map.resize((size_t)m.nnz);
  std::vector<int> pos(t->rp.begin(), t->rp.end() - 1);
  for (int i = 0; i < m.nrows; ++i)
    for (int k = m.rowptr[i]; k < m.rowptr[i + 1]; ++k) {
      const int o = pos[m.col[k]]++;
      t->col[o] = i;
      t->val[o] = m.val ? m.val[k] : 0.0;
      t->map[o] = k;
    }
}

int upload_t(const HostT& t, Sell* S) {
  return sell_build(S, t.nrows, t.ncols, (int)t.col.size(), t.rp.data(), t.col.data(),
                    t.val.data(), 0);
}

// ---------------------------------------------------------------------- kernels
__global__ void k_scale_copy(long long n, const double* __restrict__ a, double s,
                             double* __restrict__ b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = a[i] * s;
}

__global__ void k_scatter_idx(int n, const int* __restrict__ idx, const double* __restrict__ v,
                              double* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    out[idx[k]] = v[k];
}
__global__ void k_gather_idx(int n, const int* __restrict__ idx, const double* __restrict__ in,
                             double* __restrict__ v) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    v[k] = in[idx[k]];
}

struct AddTo {
  double* out;
  __device__ void operator()(const double* t) const { *out += t[0]; }
};

// J = 1/2 sum vol (u^2 + v^2 + w^2) over [0,n)
__global__ void __launch_bounds__(256) k_kinetic(int n, const double* __restrict__ vol,
                                                 const double* __restrict__ u,
                                                 const double* __restrict__ v,
                                                 const double* __restrict__ w, ReduceScratch rs,
                                                 double* out) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    acc[0] += 0.5 * vol[i] * (u[i] * u[i] + v[i] * v[i] + w[i] * w[i]);
  grid_reduce<SumOp, 1>(acc, rs, AddTo{out});
}

// seed: ub = vol * u (inner), 0 elsewhere
__global__ void k_seed(int n, int n_all, const double* __restrict__ vol, const double* __restrict__ u,
                       double* __restrict__ ub) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_all; i += gridDim.x * blockDim.x)
    ub[i] = (i < n) ? vol[i] * u[i] : 0.0;
}

// gpb(inner) += fact * ub(inner)
__global__ void k_axpy_inner(int n, double* __restrict__ y, const double* __restrict__ x, double a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] += a * x[i];
}

// ab = a1 * ub + a0b ; a0b = a2 * ub   (inner)
__global__ void k_ab(int n, const double* __restrict__ ub, double* __restrict__ a0b,
                     double* __restrict__ ab, double a1, double a2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double x = ub[i];
    ab[i] = a1 * x + a0b[i];
    a0b[i] = a2 * x;
  }
}

// y_j += alpha * sum_t cval[map[t]] * x[col[t]]  over the transposed pattern of D (C^T x)
__global__ void k_ct_spmv(int nrows, const int* __restrict__ rp, const int* __restrict__ col,
                          const int* __restrict__ map, const double* __restrict__ cval,
                          const double* __restrict__ x, double* __restrict__ y, double alpha) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nrows; j += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int t = rp[j]; t < rp[j + 1]; ++t) s += cval[map[t]] * x[col[t]];
    if (rp[j] != rp[j + 1]) y[j] += alpha * s;
  }
}

// z_k = sum_d ab_d[row k] * u_d[col k] over D's nonzeros
__global__ void k_zvec(int nnz, const int* __restrict__ rowidx, const int* __restrict__ col,
                       const double* __restrict__ abx, const double* __restrict__ aby,
                       const double* __restrict__ abz, const double* __restrict__ u,
                       const double* __restrict__ v, const double* __restrict__ w,
                       double* __restrict__ z) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x) {
    const int i = rowidx[k], c = col[k];
    z[k] = abx[i] * u[c] + aby[i] * v[c] + abz[i] * w[c];
  }
}

__global__ void k_mask_mul(int n, double* __restrict__ y, const unsigned char* __restrict__ keep) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (!keep[i]) y[i] = 0.0;
}

// gnu += sum_i ab_i * (Dg u)_i
__global__ void __launch_bounds__(256) k_dot_acc(int n, const double* __restrict__ a,
                                                 const double* __restrict__ b, ReduceScratch rs,
                                                 double* out) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    acc[0] += a[i] * b[i];
  grid_reduce<SumOp, 1>(acc, rs, AddTo{out});
}

}  // namespace

// ---------------------------------------------------------------------- the object
struct Adjoint {
  Dns E;
  gipb200_adjoint_params prm{};
  int N = 0, NO = 0, NF = 0, nnzD = 0, n_lid = 0;
  std::vector<double> u0, v0, w0;          // initial fields (host)
  DevBuf<double> dval0;                    // D_given in D's sliced layout
  DevBuf<double> dtab0;                    // D_given's value table (when D has one)
  DevBuf<double> cval0;                    // C's initial values (= D_given, CSR order)
  DevBuf<double> vol;
  DevBuf<int> lid;
  Sell SOt, SFt[3], Gt[3], Mt[3], Dt, Lbt, Ect;
  DevBuf<int> dt_rp, dt_col, dt_map, rowidx;  // transposed pattern of D with source map
  DevBuf<unsigned char> so_empty;             // faces whose SO row is empty (mf carried)
  // state
  int nsteps = 0;
  double s_nu = 1.0;
  std::vector<double> dts;
  std::vector<double> lid_vals;
  struct Ckpt {
    int step;
    DevBuf<double> u, v, w, mf, ax0, ay0, az0, p0;
  };
  std::vector<Ckpt*> ckpts;
  DevBuf<double> lid_dev;                     // the lid values of the current forward
  DevBuf<double> seg_u, seg_mf;               // per-step u,v,w (3*NO) and mf (NF)
  int seg_cap = 0;
  // adjoint vectors
  DevBuf<double> ub[3], gpb[3], a0b[3], ab[3], mfb, pfb, pb, lam, tmp, tmpN, z, cval, dgu;
  DevBuf<double> acc;                         // [0] J, [1] dJ/ds
  DevBuf<double> partials;
  DevBuf<unsigned> ticket;
  ReduceScratch rs{};
  Pcg adj;                                    // adjoint Poisson solve
  ~Adjoint() {
    for (auto* c : ckpts) delete c;
  }
  int reset_state(cudaStream_t s);
  int save(Ckpt* c, cudaStream_t s);
  int restore(const Ckpt* c, cudaStream_t s);
  int run_forward(int n0, int n1, bool store, cudaStream_t s);
  int adjoint_step(int n, int seg_slot, cudaStream_t s);
};

static int blocks_for(int n, int* b) { return grid_blocks(256, std::max(n, 1), 4, kMaxReduceBlocks, b); }

// The engine's prescribed dt sequence: copied into its buffer, which grows only when a run
// is longer than any before (no allocation per forward or backward call).
static int put_dt_seq(Dns& E, const double* h, int n) {
  if (!E.dt_seq.p || E.dt_seq.n < (size_t)n) GIPB_TRY(E.dt_seq.alloc((size_t)n));
  GIPB_CUDA(cudaMemcpy(E.dt_seq.p, h, (size_t)n * 8, cudaMemcpyHostToDevice));
  E.dt_seq_len = n;
  return GIPB200_OK;
}

int Adjoint::reset_state(cudaStream_t s) {
  // the engine restarts from the initial fields with the lid values applied
  std::vector<double> uu(u0);
  GIPB_CUDA(cudaMemcpyAsync(E.u.p, uu.data(), (size_t)NO * 8, cudaMemcpyHostToDevice, s));
  GIPB_CUDA(cudaMemcpyAsync(E.v.p, v0.data(), (size_t)NO * 8, cudaMemcpyHostToDevice, s));
  GIPB_CUDA(cudaMemcpyAsync(E.w.p, w0.data(), (size_t)NO * 8, cudaMemcpyHostToDevice, s));
  if (n_lid) {
    if (!lid_dev.p) GIPB_TRY(lid_dev.alloc((size_t)n_lid));
    GIPB_CUDA(cudaMemcpyAsync(lid_dev.p, lid_vals.data(), (size_t)n_lid * 8,
                              cudaMemcpyHostToDevice, s));
    int b;
    GIPB_TRY(blocks_for(n_lid, &b));
    k_scatter_idx<<<b, 256, 0, s>>>(n_lid, lid.p, lid_dev.p, E.u.p);
    GIPB_LAUNCH_CHECK();
    GIPB_CUDA(cudaStreamSynchronize(s));
  }
  DevBuf<double>* zero[] = {&E.ax, &E.ay, &E.az, &E.ax0, &E.ay0, &E.az0, &E.rhs, &E.p,
                            &E.p0, &E.gpx, &E.gpy, &E.gpz, &E.temp, &E.mf};
  for (auto* z : zero) GIPB_TRY(z->zero(s));
  GIPB_CUDA(cudaMemcpyAsync(E.cval.p, E.D.val.p, E.cval.n * 8, cudaMemcpyDeviceToDevice, s));
  // C starts from the D file's values, not the scaled D
  {
    int b;
    GIPB_TRY(blocks_for(nnzD, &b));
    k_scatter_idx<<<b, 256, 0, s>>>(nnzD, E.D.pos.p, cval0.p, E.cval.p);
    GIPB_LAUNCH_CHECK();
  }
  GIPB_TRY(E.sc.zero(s));
  E.started = false;
  E.steps_enqueued = 0;
  return GIPB200_OK;
}

int Adjoint::save(Ckpt* c, cudaStream_t s) {
  DevBuf<double>* src[] = {&E.u, &E.v, &E.w, &E.mf, &E.ax0, &E.ay0, &E.az0, &E.p0};
  DevBuf<double>* dst[] = {&c->u, &c->v, &c->w, &c->mf, &c->ax0, &c->ay0, &c->az0, &c->p0};
  for (int k = 0; k < 8; ++k) {
    if (!dst[k]->p) GIPB_TRY(dst[k]->alloc(src[k]->n));
    GIPB_CUDA(cudaMemcpyAsync(dst[k]->p, src[k]->p, src[k]->n * 8, cudaMemcpyDeviceToDevice, s));
  }
  return GIPB200_OK;
}

int Adjoint::restore(const Ckpt* c, cudaStream_t s) {
  const DevBuf<double>* src[] = {&c->u, &c->v, &c->w, &c->mf, &c->ax0, &c->ay0, &c->az0, &c->p0};
  DevBuf<double>* dst[] = {&E.u, &E.v, &E.w, &E.mf, &E.ax0, &E.ay0, &E.az0, &E.p0};
  for (int k = 0; k < 8; ++k)
    GIPB_CUDA(cudaMemcpyAsync(dst[k]->p, src[k]->p, src[k]->n * 8, cudaMemcpyDeviceToDevice, s));
  // engine scalars at the checkpoint's step: dt of that step, step counter
  DnsScalars S;
  S.dt = dts[c->step];
  S.sigma = 1.0 / S.dt;
  S.time = 0.0;
  S.step = c->step;
  S.started = 1;
  GIPB_CUDA(cudaMemcpyAsync(E.sc.p, &S, sizeof(S), cudaMemcpyHostToDevice, s));
  GIPB_CUDA(cudaStreamSynchronize(s));
  E.started = true;
  return GIPB200_OK;
}

// steps [n0, n1); with `store`, the state entering each step goes to the segment buffers
int Adjoint::run_forward(int n0, int n1, bool store, cudaStream_t s) {
  for (int n = n0; n < n1; ++n) {
    if (store) {
      const int k = n - n0;
      GIPB_CUDA(cudaMemcpyAsync(seg_u.p + (size_t)(3 * k + 0) * NO, E.u.p, (size_t)NO * 8, cudaMemcpyDeviceToDevice, s));
      GIPB_CUDA(cudaMemcpyAsync(seg_u.p + (size_t)(3 * k + 1) * NO, E.v.p, (size_t)NO * 8, cudaMemcpyDeviceToDevice, s));
      GIPB_CUDA(cudaMemcpyAsync(seg_u.p + (size_t)(3 * k + 2) * NO, E.w.p, (size_t)NO * 8, cudaMemcpyDeviceToDevice, s));
      GIPB_CUDA(cudaMemcpyAsync(seg_mf.p + (size_t)k * NF, E.mf.p, (size_t)NF * 8, cudaMemcpyDeviceToDevice, s));
    }
    GIPB_TRY(dns_advance(E, 1, s));
  }
  return GIPB200_OK;
}

int Adjoint::adjoint_step(int n, int k, cudaStream_t s) {
  const double dt = dts[n];
  const double sigma = 1.0 / dt;
  const double fact1 = -1.0 / sigma, fact2 = 1.0 / sigma, fact = -1.0 / (prm.rho * sigma);
  const double a1 = 1.5 * dt, a2 = -0.5 * dt;
  const double* un[3] = {seg_u.p + (size_t)(3 * k) * NO, seg_u.p + (size_t)(3 * k + 1) * NO,
                         seg_u.p + (size_t)(3 * k + 2) * NO};
  const double* mfn = seg_mf.p + (size_t)k * NF;
  int bN, bO, bF, bZ;
  GIPB_TRY(blocks_for(N, &bN));
  GIPB_TRY(blocks_for(NO, &bO));
  GIPB_TRY(blocks_for(NF, &bF));
  GIPB_TRY(blocks_for(nnzD, &bZ));
  // A1: mass fluxes
  GIPB_TRY(pfb.zero(s));
  GIPB_TRY(launch_sell_spmv(SOt, SOt.val.p, mfb.p, pfb.p, fact1, 1.0, 1, s));
  for (int d = 0; d < 3; ++d) {
    GIPB_TRY(gpb[d].zero(s));
    GIPB_TRY(launch_sell_spmv(SFt[d], SFt[d].val.p, mfb.p, gpb[d].p, fact2, 1.0, 1, s));
    GIPB_TRY(launch_sell_spmv(SFt[d], SFt[d].val.p, mfb.p, ub[d].p, prm.rho, 1.0, 1, s));
  }
  // A2: velocity correction
  for (int d = 0; d < 3; ++d) {
    k_axpy_inner<<<bN, 256, 0, s>>>(N, gpb[d].p, ub[d].p, fact);
    GIPB_LAUNCH_CHECK();
  }
  // A3: gradients
  for (int d = 0; d < 3; ++d) GIPB_TRY(launch_sell_spmv(Gt[d], Gt[d].val.p, gpb[d].p, pfb.p, 1.0, 1.0, 1, s));
  // A4: ghost copy p_ghost = Lb p
  GIPB_CUDA(cudaMemcpyAsync(pb.p, pfb.p, (size_t)NO * 8, cudaMemcpyDeviceToDevice, s));
  GIPB_TRY(launch_sell_spmv(Lbt, Lbt.val.p, pfb.p, pb.p, 1.0, 1.0, 1, s));
  // A5: adjoint Poisson solve  L lam = pbar
  GIPB_TRY(tmp.zero(s));
  GIPB_TRY(adj.enqueue(pb.p, lam.p, tmp.p, s, true));
  // A6: divergence
  for (int d = 0; d < 3; ++d) GIPB_TRY(launch_sell_spmv(Mt[d], Mt[d].val.p, lam.p, ub[d].p, sigma, 1.0, 1, s));
  // A7: Adams-Bashforth
  for (int d = 0; d < 3; ++d) {
    k_ab<<<bN, 256, 0, s>>>(N, ub[d].p, a0b[d].p, ab[d].p, a1, a2);
    GIPB_LAUNCH_CHECK();
  }
  // C of this step (C = Ec mf^n) in D's CSR order
  GIPB_TRY(launch_csr_spmv(E.Ec.nrows, E.Ec.rowptr.p, E.Ec.csr_col.p, E.Ec.csr_val.p, mfn, cval.p,
                           nullptr, 0.0, 0.0, 0, s));
  // A8: u += s D^T ab - C^T ab ; dJ/ds += ab . (Dg u)
  for (int d = 0; d < 3; ++d) {
    GIPB_TRY(launch_sell_spmv(Dt, Dt.val.p, ab[d].p, ub[d].p, s_nu, 1.0, 1, s));
    k_ct_spmv<<<bO, 256, 0, s>>>(NO, dt_rp.p, dt_col.p, dt_map.p, cval.p, ab[d].p, ub[d].p, -1.0);
    GIPB_LAUNCH_CHECK();
    GIPB_TRY(dgu.zero(s));
    GIPB_TRY(launch_sell_spmv(E.D, dval0.p, un[d], dgu.p, 0.0, 0.0, 0, s));
    k_dot_acc<<<bN, 256, 0, s>>>(N, ab[d].p, dgu.p, rs, acc.p + 1);
    GIPB_LAUNCH_CHECK();
  }
  // A9: mass-flux adjoint through C:  mfb = mfb * [SO row empty] - Ec^T z
  k_zvec<<<bZ, 256, 0, s>>>(nnzD, rowidx.p, E.D.csr_col.p, ab[0].p, ab[1].p, ab[2].p, un[0], un[1],
                            un[2], z.p);
  k_mask_mul<<<bF, 256, 0, s>>>(NF, mfb.p, so_empty.p);
  GIPB_LAUNCH_CHECK();
  GIPB_TRY(launch_sell_spmv(Ect, Ect.val.p, z.p, mfb.p, -1.0, 1.0, 1, s));
  return GIPB200_OK;
}

}  // namespace gipb200

using namespace gipb200;

struct gipb200_adjoint_s {
  gipb200::Adjoint A;
};

extern "C" {

int gipb200_adjoint_create(const gipb200_dns_ops* ops, const double* h_u0, const double* h_v0,
                           const double* h_w0, const double* h_dxs, const double* h_volume,
                           const int* h_lid_cells, int n_lid, const gipb200_adjoint_params* prm,
                           gipb200_adjoint* out) {
  if (!ops || !h_u0 || !h_v0 || !h_w0 || !h_dxs || !h_volume || !prm || !out ||
      (n_lid > 0 && !h_lid_cells) || n_lid < 0)
    return fail(GIPB200_ERR_ARG, "null argument");
  if (!(prm->tol > 0) || prm->maxit <= 0 || prm->checkpoint_every <= 0 || !(prm->nu0 > 0))
    return fail(GIPB200_ERR_ARG, "adjoint: tol, maxit, checkpoint_every and nu0 must be positive");
  *out = nullptr;
  GIPB_TRY(check_dns_ops(ops));
  const int N = ops->n_inner, NO = ops->n_owned, NF = ops->n_faces;
  for (int k = 0; k < n_lid; ++k)
    if (h_lid_cells[k] < 0 || h_lid_cells[k] >= NO)
      return fail(GIPB200_ERR_ARG, "lid cell %d out of range", h_lid_cells[k]);
  if (ops->D.nrows != N || ops->Lb.nrows > NO || ops->SO.nrows != NF)
    return fail(GIPB200_ERR_ARG, "adjoint: D needs n_inner rows and SO n_faces rows");
  gipb200_adjoint H = new (std::nothrow) gipb200_adjoint_s();
  if (!H) return fail(GIPB200_ERR_NOMEM, "host allocation failed");
  Adjoint& A = H->A;
  int st = [&]() -> int {
    A.prm = *prm;
    A.N = N;
    A.NO = NO;
    A.NF = NF;
    A.nnzD = ops->D.nnz;
    A.n_lid = n_lid;
    gipb200_dns_params dp;
    memset(&dp, 0, sizeof(dp));
    dp.rho = prm->rho;
    dp.gamma = prm->gamma;
    dp.pcg.mode = GIPB200_PCG_TOL;
    dp.pcg.maxit = prm->maxit;
    dp.pcg.tol = prm->tol;
    dp.pcg.precond = prm->precond;
    dp.use_graph = 1;
    dp.reorder = 0;
    GIPB_TRY(dns_init(A.E, ops, h_u0, h_v0, h_w0, h_dxs, &dp));
    A.u0.assign(h_u0, h_u0 + NO);
    A.v0.assign(h_v0, h_v0 + NO);
    A.w0.assign(h_w0, h_w0 + NO);
    GIPB_TRY(A.dval0.alloc(A.E.D.val.n));
    GIPB_CUDA(cudaMemcpy(A.dval0.p, A.E.D.val.p, A.E.D.val.n * 8, cudaMemcpyDeviceToDevice));
    if (A.E.D.ntab) {  // the forward kernels read D through its table: scaled with it
      GIPB_TRY(A.dtab0.alloc((size_t)A.E.D.ntab));
      GIPB_CUDA(cudaMemcpy(A.dtab0.p, A.E.D.vtab.p, (size_t)A.E.D.ntab * 8,
                           cudaMemcpyDeviceToDevice));
    }
    GIPB_TRY(A.cval0.upload(ops->D.val, std::max(ops->D.nnz, 1)));
    GIPB_TRY(A.vol.upload(h_volume, N));
    GIPB_TRY(A.lid.upload(h_lid_cells, std::max(n_lid, 1)));
    // transposed operators
    HostT t;
    transpose(ops->SO, NO, &t);
    GIPB_TRY(upload_t(t, &A.SOt));
    const gipb200_host_csr* sf[3] = {&ops->SFx, &ops->SFy, &ops->SFz};
    const gipb200_host_csr* g[3] = {&ops->Gx, &ops->Gy, &ops->Gz};
    const gipb200_host_csr* m[3] = {&ops->Mx, &ops->My, &ops->Mz};
    for (int d = 0; d < 3; ++d) {
      transpose(*sf[d], NO, &t);
      GIPB_TRY(upload_t(t, &A.SFt[d]));
      transpose(*g[d], NO, &t);
      GIPB_TRY(upload_t(t, &A.Gt[d]));
      transpose(*m[d], NO, &t);
      GIPB_TRY(upload_t(t, &A.Mt[d]));
    }
    transpose(ops->Lb, NO, &t);
    GIPB_TRY(upload_t(t, &A.Lbt));
    transpose(ops->D, NO, &t);
    GIPB_TRY(upload_t(t, &A.Dt));
    GIPB_TRY(A.dt_rp.upload(t.rp.data(), t.rp.size()));
    GIPB_TRY(A.dt_col.upload(t.col.data(), std::max<size_t>(t.col.size(), 1)));
    GIPB_TRY(A.dt_map.upload(t.map.data(), std::max<size_t>(t.map.size(), 1)));
    transpose(ops->Ec, NF, &t);
    GIPB_TRY(upload_t(t, &A.Ect));
    std::vector<int> rowidx((size_t)std::max(ops->D.nnz, 1));
    for (int i = 0; i < ops->D.nrows; ++i)
      for (int k = ops->D.rowptr[i]; k < ops->D.rowptr[i + 1]; ++k) rowidx[k] = i;
    GIPB_TRY(A.rowidx.upload(rowidx.data(), rowidx.size()));
    std::vector<unsigned char> se((size_t)std::max(NF, 1), 0);
    for (int f = 0; f < ops->SO.nrows; ++f) se[f] = ops->SO.rowptr[f] == ops->SO.rowptr[f + 1];
    GIPB_TRY(A.so_empty.upload(se.data(), se.size()));
    for (int d = 0; d < 3; ++d) {
      GIPB_TRY(A.ub[d].alloc(NO));
      GIPB_TRY(A.gpb[d].alloc(NO));
      GIPB_TRY(A.a0b[d].alloc(N));
      GIPB_TRY(A.ab[d].alloc(N));
    }
    GIPB_TRY(A.mfb.alloc(std::max(NF, 1)));
    GIPB_TRY(A.pfb.alloc(NO));
    GIPB_TRY(A.pb.alloc(NO));
    GIPB_TRY(A.lam.alloc(NO));
    GIPB_TRY(A.tmp.alloc(NO));
    GIPB_TRY(A.dgu.alloc(N));
    GIPB_TRY(A.z.alloc(std::max(ops->D.nnz, 1)));
    GIPB_TRY(A.cval.upload(ops->D.val, std::max(ops->D.nnz, 1)));
    GIPB_TRY(A.acc.alloc(2));
    GIPB_TRY(reduce_scratch_alloc(&A.partials, &A.ticket, &A.rs));
    gipb200_pcg_params pp;
    memset(&pp, 0, sizeof(pp));
    pp.mode = GIPB200_PCG_TOL;
    pp.maxit = prm->maxit;
    pp.tol = prm->tol;
    pp.precond = prm->precond;
    GIPB_TRY(A.adj.init(&A.E.L, NO, pp, 0));
    GIPB_CUDA(cudaDeviceSynchronize());
    return GIPB200_OK;
  }();
  if (st != GIPB200_OK) {
    delete H;
    return st;
  }
  *out = H;
  return GIPB200_OK;
}

int gipb200_adjoint_destroy(gipb200_adjoint H) {
  delete H;
  return GIPB200_OK;
}

int gipb200_adjoint_forward(gipb200_adjoint H, const double* h_lid, double nu_scale, int nsteps,
                            double* h_dt, int dt_given, double* h_J) {
  if (!H || nsteps <= 0 || !h_J || (H->A.n_lid > 0 && !h_lid) || (dt_given && !h_dt))
    return fail(GIPB200_ERR_ARG, "bad arguments");
  if (!(nu_scale > 0)) return fail(GIPB200_ERR_ARG, "nu_scale must be positive");
  Adjoint& A = H->A;
  cudaStream_t s = 0;
  A.nsteps = nsteps;
  A.s_nu = nu_scale;
  A.lid_vals.assign(h_lid, h_lid + A.n_lid);
  // D = s * D_given
  {
    int b;
    GIPB_TRY(grid_blocks(256, (int)std::min<size_t>(A.dval0.n, 1u << 30), 4, 0, &b));
    k_scale_copy<<<b, 256, 0, s>>>((long long)A.dval0.n, A.dval0.p, nu_scale, A.E.D.val.p);
    GIPB_LAUNCH_CHECK();
    // the same product of the same doubles: every slot's table value equals its scaled value
    if (A.E.D.ntab) {
      k_scale_copy<<<1, 256, 0, s>>>((long long)A.E.D.ntab, A.dtab0.p, nu_scale, A.E.D.vtab.p);
      GIPB_LAUNCH_CHECK();
    }
  }
  if (dt_given) {
    GIPB_TRY(put_dt_seq(A.E, h_dt, nsteps));
  } else {
    A.E.dt_seq_len = 0;  // dt from the CFL condition (the buffer is kept for the backward)
  }
  // a new dt source changes the captured step: capture again
  if (A.E.exec) {
    cudaGraphExecDestroy(A.E.exec);
    A.E.exec = nullptr;
  }
  if (A.E.graph) {
    cudaGraphDestroy(A.E.graph);
    A.E.graph = nullptr;
  }
  GIPB_TRY(A.reset_state(s));
  // the checkpoints are kept from call to call (their device buffers are reused: a forward
  // allocates only when it needs more segments than the last one)
  const int K = A.prm.checkpoint_every;
  const int nck = (nsteps + K - 1) / K;
  while ((int)A.ckpts.size() > nck) {
    delete A.ckpts.back();
    A.ckpts.pop_back();
  }
  while ((int)A.ckpts.size() < nck) A.ckpts.push_back(new Adjoint::Ckpt());
  for (int n0 = 0, ci = 0; n0 < nsteps; n0 += K, ++ci) {
    Adjoint::Ckpt* c = A.ckpts[(size_t)ci];
    c->step = n0;
    if (n0 == 0) {
      // the first step's dt comes from the initial CFL (or the prescribed list)
      GIPB_TRY(A.E.grow_history(nsteps, s));
      GIPB_TRY(A.E.enqueue_initial_dt(s));
      A.E.started = true;
    }
    GIPB_TRY(A.save(c, s));
    GIPB_TRY(A.run_forward(n0, std::min(nsteps, n0 + K), false, s));
  }
  // record the dt sequence used
  A.dts.assign(nsteps, 0.0);
  GIPB_CUDA(cudaDeviceSynchronize());
  GIPB_CUDA(cudaMemcpy(A.dts.data(), A.E.h_dt.p, (size_t)nsteps * 8, cudaMemcpyDeviceToHost));
  if (!dt_given && h_dt) memcpy(h_dt, A.dts.data(), (size_t)nsteps * 8);
  GIPB_TRY(A.acc.zero(s));
  int b;
  GIPB_TRY(blocks_for(A.N, &b));
  k_kinetic<<<b, 256, 0, s>>>(A.N, A.vol.p, A.E.u.p, A.E.v.p, A.E.w.p, A.rs, A.acc.p);
  GIPB_LAUNCH_CHECK();
  GIPB_CUDA(cudaMemcpy(h_J, A.acc.p, sizeof(double), cudaMemcpyDeviceToHost));
  // the engine's final velocity seeds the backward sweep
  for (int d = 0; d < 3; ++d) {
    const double* uf = d == 0 ? A.E.u.p : (d == 1 ? A.E.v.p : A.E.w.p);
    k_seed<<<b, 256, 0, s>>>(A.N, A.NO, A.vol.p, uf, A.ub[d].p);
    GIPB_LAUNCH_CHECK();
  }
  GIPB_CUDA(cudaDeviceSynchronize());
  return GIPB200_OK;
}

int gipb200_adjoint_backward(gipb200_adjoint H, double* h_grad_lid, double* h_grad_nu) {
  if (!H || (!h_grad_lid && H->A.n_lid) || !h_grad_nu) return fail(GIPB200_ERR_ARG, "bad arguments");
  Adjoint& A = H->A;
  if (A.nsteps <= 0 || A.ckpts.empty()) return fail(GIPB200_ERR_STATE, "run the forward first");
  cudaStream_t s = 0;
  const int K = A.prm.checkpoint_every;
  if (A.seg_cap < K) {
    GIPB_TRY(A.seg_u.alloc((size_t)3 * K * A.NO));
    GIPB_TRY(A.seg_mf.alloc((size_t)K * std::max(A.NF, 1)));
    A.seg_cap = K;
  }
  // the backward replays each segment with the recorded steps
  GIPB_TRY(put_dt_seq(A.E, A.dts.data(), A.nsteps));
  if (A.E.exec) {
    cudaGraphExecDestroy(A.E.exec);
    A.E.exec = nullptr;
  }
  if (A.E.graph) {
    cudaGraphDestroy(A.E.graph);
    A.E.graph = nullptr;
  }
  // adjoint state after the last step (ub seeded by the forward)
  GIPB_TRY(A.mfb.zero(s));
  for (int d = 0; d < 3; ++d) GIPB_TRY(A.a0b[d].zero(s));
  double zero2[2] = {0.0, 0.0};
  GIPB_CUDA(cudaMemcpyAsync(A.acc.p, zero2, sizeof(zero2), cudaMemcpyHostToDevice, s));
  for (int c = (int)A.ckpts.size() - 1; c >= 0; --c) {
    const int n0 = A.ckpts[c]->step, n1 = std::min(A.nsteps, n0 + K);
    GIPB_TRY(A.restore(A.ckpts[c], s));
    GIPB_TRY(A.run_forward(n0, n1, true, s));
    for (int n = n1 - 1; n >= n0; --n) GIPB_TRY(A.adjoint_step(n, n - n0, s));
  }
  GIPB_CUDA(cudaDeviceSynchronize());
  if (A.n_lid) {
    DevBuf<double> g;
    GIPB_TRY(g.alloc(A.n_lid));
    int b;
    GIPB_TRY(blocks_for(A.n_lid, &b));
    k_gather_idx<<<b, 256>>>(A.n_lid, A.lid.p, A.ub[0].p, g.p);
    GIPB_LAUNCH_CHECK();
    GIPB_CUDA(cudaMemcpy(h_grad_lid, g.p, (size_t)A.n_lid * 8, cudaMemcpyDeviceToHost));
  }
  double ds = 0.0;
  GIPB_CUDA(cudaMemcpy(&ds, A.acc.p + 1, sizeof(double), cudaMemcpyDeviceToHost));
  *h_grad_nu = ds / A.prm.nu0;  // D = (nu/nu0) D_given
  return GIPB200_OK;
}

}  // extern "C"
