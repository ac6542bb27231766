// Device-resident fractional-step timestep: GIP_DNS::integrate (src/Algorithms/GIP_DNS.h:
// 99-113) with its five phases fused into a handful of kernels, dt/sigma/time and the
// per-step history kept on the device, and each step capturable in one CUDA graph.
//
// Every output element is produced with the IEEE operations and the order of GIP's CPU
// code (GIP_DNS.h:309-414 over GIP_MatrixMulticore / GIP_VectorMulticore), including
// GIP's rule that an empty CSR row leaves its output untouched; only the reductions of
// the PCG dot products are ordered differently.
#include <math.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "device.cuh"
#include "dns.cuh"

namespace gipb200 {

// ------------------------------------------------------------------ row helpers
// D and C share D's sparsity (GIP loads C from D's file, GIP_DNS.h:150-151): one pass
// over the slots yields D u, D v, D w, C u, C v, C w, each summed in CSR order.
template <bool TAB>
__device__ __forceinline__ void dc_row(const SellView<double>& D, const double* __restrict__ cval,
                                       const double* __restrict__ u, const double* __restrict__ v,
                                       const double* __restrict__ w, int s, int lane,
                                       double (&sd)[3], double (&sc)[3], bool& any) {
  long long base;
  int len;
  slice_range(D, s, base, len);
  // four slots at a time: their columns and values, then their twelve gathers, are in
  // flight together (two dependent round trips per group instead of two per slot; 76
  // registers and 3 CTAs per SM, against 62 and 4 with two slots: the predictor phase of
  // the 256^3 cavity 1.52 against 1.60 ms)
  for (int j0 = 0; j0 < len; j0 += 4) {
    int c[4];
    double dv[4], cv[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const bool in = j0 + t < len;
      const long long k = base + 32LL * (j0 + t) + lane;
      c[t] = in ? ld_stream(D.col + k) : -1;
      dv[t] = in ? sell_value<TAB>(D, k) : 0.0;
      cv[t] = in ? ld_stream(cval + k) : 0.0;
    }
    double xu[4], xv[4], xw[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      xu[t] = c[t] >= 0 ? __ldg(u + c[t]) : 0.0;
      xv[t] = c[t] >= 0 ? __ldg(v + c[t]) : 0.0;
      xw[t] = c[t] >= 0 ? __ldg(w + c[t]) : 0.0;
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      if (c[t] < 0) continue;
      sd[0] = dadd(sd[0], dmul(xu[t], dv[t]));
      sd[1] = dadd(sd[1], dmul(xv[t], dv[t]));
      sd[2] = dadd(sd[2], dmul(xw[t], dv[t]));
      sc[0] = dadd(sc[0], dmul(xu[t], cv[t]));
      sc[1] = dadd(sc[1], dmul(xv[t], cv[t]));
      sc[2] = dadd(sc[2], dmul(xw[t], cv[t]));
      any = true;
    }
  }
}

// y = alpha*sum + beta*y as GIP_MatrixMulticore::spmv(x,b,alpha,beta) (:85-103)
__device__ __forceinline__ double axpby_row(double alpha, double sum, double beta, double y) {
  return dadd(dmul(alpha, sum), dmul(beta, y));
}

// ------------------------------------------------------------------ PredictorVelocity
// ax = D u; ax = -C u + ax  (and v, w)   -- GIP_DNS.h:313-318
template <bool TAB>
__global__ void __launch_bounds__(256) k_dns_convdiff(SellView<double> D,
                                                      const double* __restrict__ cval,
                                                      const double* __restrict__ u,
                                                      const double* __restrict__ v,
                                                      const double* __restrict__ w,
                                                      double* __restrict__ ax, double* __restrict__ ay,
                                                      double* __restrict__ az) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int s = gw; s < D.nslices; s += nw) {
    double sd[3] = {0.0, 0.0, 0.0}, sc[3] = {0.0, 0.0, 0.0};
    bool any = false;
    dc_row<TAB>(D, cval, u, v, w, s, lane, sd, sc, any);
    const int i = s * 32 + lane;
    if (i < D.nrows && any) {
      ax[i] = axpby_row(-1.0, sc[0], 1.0, sd[0]);
      ay[i] = axpby_row(-1.0, sc[1], 1.0, sd[1]);
      az[i] = axpby_row(-1.0, sc[2], 1.0, sd[2]);
    }
  }
}

// u += 1.5dt ax; u += -0.5dt ax0; ax0 = ax (and v, w) over the inner cells -- :320-336
__global__ void __launch_bounds__(256) k_dns_ab2(int n, double* __restrict__ u, double* __restrict__ v,
                                                 double* __restrict__ w, const double* __restrict__ ax,
                                                 const double* __restrict__ ay,
                                                 const double* __restrict__ az,
                                                 double* __restrict__ ax0, double* __restrict__ ay0,
                                                 double* __restrict__ az0, const DnsScalars* S) {
  const double dt = S->dt;
  const double a1 = dmul(1.5, dt);
  const double a2 = dmul(-0.5, dt);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double x = ax[i], y = ay[i], z = az[i];
    u[i] = dadd(dadd(u[i], dmul(a1, x)), dmul(a2, ax0[i]));
    v[i] = dadd(dadd(v[i], dmul(a1, y)), dmul(a2, ay0[i]));
    w[i] = dadd(dadd(w[i], dmul(a1, z)), dmul(a2, az0[i]));
    ax0[i] = x;
    ay0[i] = y;
    az0[i] = z;
  }
}

// ------------------------------------------------------------------ PoissonEquation rhs
// rhs = Mx u; rhs = My v + rhs; rhs = sigma Mz w + sigma rhs   -- GIP_DNS.h:343-345
template <bool TAB>
__global__ void __launch_bounds__(256) k_dns_rhs(SellView<double> Mx, SellView<double> My,
                                                 SellView<double> Mz, const double* __restrict__ u,
                                                 const double* __restrict__ v,
                                                 const double* __restrict__ w,
                                                 double* __restrict__ rhs, const DnsScalars* S) {
  const double sigma = S->sigma;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int ns = max(Mx.nslices, max(My.nslices, Mz.nslices));
  for (int s = gw; s < ns; s += nw) {
    const int i = s * 32 + lane;
    const SellView<double> M[3] = {Mx, My, Mz};
    const double* const X[3] = {u, v, w};
    double sm[3] = {0, 0, 0};
    bool an[3] = {false, false, false};
    // the row's previous value, loaded with the slots rather than after the gathers
    const double r_in = (i < Mx.nrows || i < My.nrows || i < Mz.nrows) ? rhs[i] : 0.0;
    sell_rows3_f64<TAB>(M, X, s, lane, sm, an);
    const double sx = sm[0], sy = sm[1], sz = sm[2];
    bool ax = an[0], ay = an[1], az = an[2];
    ax = ax && i < Mx.nrows;
    ay = ay && i < My.nrows;
    az = az && i < Mz.nrows;
    if (ax || ay || az) {
      double r = r_in;
      if (ax) r = sx;
      if (ay) r = axpby_row(1.0, sy, 1.0, r);
      if (az) r = axpby_row(sigma, sz, sigma, r);
      rhs[i] = r;
    }
  }
}

// p0 = p (inner); p = p0 (owned)   -- GIP_DNS.h:350-351
__global__ void k_dns_pcopy(int n_inner, int n_owned, double* __restrict__ p, double* __restrict__ p0) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_owned; i += gridDim.x * blockDim.x) {
    if (i < n_inner)
      p0[i] = p[i];
    else
      p[i] = p0[i];
  }
}

// ------------------------------------------------------------------ VelocityCorrection
// gp = G p (x,y,z); u -= gp/(rho sigma) over the inner cells   -- GIP_DNS.h:359-370
__global__ void __launch_bounds__(256) k_dns_gradcorr(SellView<double> Gx, SellView<double> Gy,
                                                      SellView<double> Gz, const double* __restrict__ p,
                                                      double* __restrict__ gpx, double* __restrict__ gpy,
                                                      double* __restrict__ gpz, double* __restrict__ u,
                                                      double* __restrict__ v, double* __restrict__ w,
                                                      int n_inner, double rho, const DnsScalars* S) {
  const double fact = ddiv(-1.0, dmul(rho, S->sigma));
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int ns = max(max(Gx.nslices, Gy.nslices), max(Gz.nslices, (n_inner + 31) / 32));
  for (int s = gw; s < ns; s += nw) {
    const int i = s * 32 + lane;
    const SellView<double> G[3] = {Gx, Gy, Gz};
    const double* const X[3] = {p, p, p};
    double sm[3] = {0, 0, 0};
    bool an[3] = {false, false, false};
    // the velocities to correct, loaded with the slots rather than after the gathers (one
    // dependent round trip less: the 256^3 correction 0.466 against 0.582 ms)
    double u_in = 0.0, v_in = 0.0, w_in = 0.0;
    if (i < n_inner) {
      u_in = u[i];
      v_in = v[i];
      w_in = w[i];
    }
    sell_rows3_f64(G, X, s, lane, sm, an);
    const double sx = sm[0], sy = sm[1], sz = sm[2];
    const bool ax = an[0], ay = an[1], az = an[2];
    if (ax && i < Gx.nrows) gpx[i] = sx;
    if (ay && i < Gy.nrows) gpy[i] = sy;
    if (az && i < Gz.nrows) gpz[i] = sz;
    if (i < n_inner) {
      const double gx = (ax && i < Gx.nrows) ? sx : gpx[i];
      const double gy = (ay && i < Gy.nrows) ? sy : gpy[i];
      const double gz = (az && i < Gz.nrows) ? sz : gpz[i];
      u[i] = dadd(u_in, dmul(fact, gx));
      v[i] = dadd(v_in, dmul(fact, gy));
      w[i] = dadd(w_in, dmul(fact, gz));
    }
  }
}

// ------------------------------------------------------------------ MassFluxes
// The same seven ordered updates with SFx, SFy, SFz merged per face (FaceOps3): slot j of
// a face belongs to SFx for j < cx, to SFy for j < cx + cy, else to SFz; every operator's
// sums run over its own entries in stored order, as in k_dns_massflux.
__global__ void __launch_bounds__(256) k_dns_massflux3(
    SellView<double> SO, SellView<double> SF, const unsigned short* __restrict__ cnt,
    const double* __restrict__ p, const double* __restrict__ gpx, const double* __restrict__ gpy,
    const double* __restrict__ gpz, const double* __restrict__ u, const double* __restrict__ v,
    const double* __restrict__ w, double* __restrict__ mf, double rho, const DnsScalars* S) {
  const double sigma = S->sigma;
  const double fact1 = ddiv(-1.0, sigma);
  const double fact2 = ddiv(1.0, sigma);
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int ns = max(SO.nslices, SF.nslices);
  for (int s = gw; s < ns; s += nw) {
    const int f = s * 32 + lane;
    double so = 0;
    bool a0 = false;
    double gx = 0, gy = 0, gz = 0, ux = 0, uy = 0, uz = 0;
    int cx = 0, cy = 0, cz = 0;
    // SO and the merged SF rows are walked together, so the slot loads of both and then
    // the gathers of both are in flight at once (three dependent round trips per face)
    long long ob = 0, fb = 0;
    int ol = 0, fl = 0;
    if (s < SO.nslices) slice_range(SO, s, ob, ol);
    if (s < SF.nslices) {
      slice_range(SF, s, fb, fl);
      const unsigned c = (f < SF.nrows) ? cnt[f] : 0u;
      cx = c & 15u;
      cy = (c >> 4) & 15u;
      cz = (c >> 8) & 15u;
    }
    const int len = max(ol, fl);
    for (int j0 = 0; j0 < len; j0 += 2) {
      int oc[2], fc[2];
      double ov[2], fv[2];
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int j = j0 + t;
        oc[t] = (j < ol) ? ld_stream(SO.col + ob + 32LL * j + lane) : -1;
        ov[t] = (j < ol) ? ld_stream(SO.val + ob + 32LL * j + lane) : 0.0;
        fc[t] = (j < fl) ? ld_stream(SF.col + fb + 32LL * j + lane) : -1;
        fv[t] = (j < fl) ? ld_stream(SF.val + fb + 32LL * j + lane) : 0.0;
      }
      double op[2], a[2], b[2];
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int j = j0 + t;
        const double* g = (j < cx) ? gpx : (j < cx + cy) ? gpy : gpz;
        const double* q = (j < cx) ? u : (j < cx + cy) ? v : w;
        op[t] = (oc[t] >= 0) ? __ldg(p + oc[t]) : 0.0;
        a[t] = (fc[t] >= 0) ? __ldg(g + fc[t]) : 0.0;
        b[t] = (fc[t] >= 0) ? __ldg(q + fc[t]) : 0.0;
      }
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        if (oc[t] >= 0) {  // SO's row, slot by slot as sell_row_f64 sums it
          so = dadd(so, dmul(op[t], ov[t]));
          a0 = true;
        }
        if (fc[t] < 0) continue;
        const int j = j0 + t;
        if (j < cx) {
          gx = dadd(gx, dmul(a[t], fv[t]));
          ux = dadd(ux, dmul(b[t], fv[t]));
        } else if (j < cx + cy) {
          gy = dadd(gy, dmul(a[t], fv[t]));
          uy = dadd(uy, dmul(b[t], fv[t]));
        } else {
          gz = dadd(gz, dmul(a[t], fv[t]));
          uz = dadd(uz, dmul(b[t], fv[t]));
        }
      }
    }
    a0 = a0 && f < SO.nrows;
    const bool ax = cx > 0, ay = cy > 0, az = cz > 0;
    if (a0 || ax || ay || az) {
      double m = mf[f];
      if (a0) m = axpby_row(fact1, so, 0.0, m);
      if (ax) m = axpby_row(fact2, gx, 1.0, m);
      if (ay) m = axpby_row(fact2, gy, 1.0, m);
      if (az) m = axpby_row(fact2, gz, 1.0, m);
      if (ax) m = axpby_row(rho, ux, 1.0, m);
      if (ay) m = axpby_row(rho, uy, 1.0, m);
      if (az) m = axpby_row(rho, uz, 1.0, m);
      mf[f] = m;
    }
  }
}

// k_dns_massflux3 for the common case in which every merged face row holds entries of one
// operator only (a structured grid's face is an x, y or z face): one gradient and one
// velocity sum per face, so the kernel fits the registers of six blocks per SM.  The
// updates keep their order: mf = fact1 SO p (a0), then fact2 SF_d gp_d, then rho SF_d u_d.
__global__ void __launch_bounds__(256, 5) k_dns_massflux1(
    SellView<double> SO, SellView<double> SF, const unsigned short* __restrict__ cnt,
    const double* __restrict__ p, const double* __restrict__ gpx, const double* __restrict__ gpy,
    const double* __restrict__ gpz, const double* __restrict__ u, const double* __restrict__ v,
    const double* __restrict__ w, double* __restrict__ mf, double rho, const DnsScalars* S) {
  const double sigma = S->sigma;
  const double fact1 = ddiv(-1.0, sigma);
  const double fact2 = ddiv(1.0, sigma);
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int ns = max(SO.nslices, SF.nslices);
  for (int s = gw; s < ns; s += nw) {
    const int f = s * 32 + lane;
    long long ob = 0, fb = 0;
    int ol = 0, fl = 0;
    const double* g = gpx;
    const double* q = u;
    bool any_f = false;
    if (s < SO.nslices) slice_range(SO, s, ob, ol);
    if (s < SF.nslices) {
      slice_range(SF, s, fb, fl);
      const unsigned c = (f < SF.nrows) ? cnt[f] : 0u;
      any_f = c != 0u;
      if ((c & 15u) == 0u) {
        g = ((c >> 4) & 15u) ? gpy : gpz;
        q = ((c >> 4) & 15u) ? v : w;
      }
    }
    double so = 0.0, gs = 0.0, us = 0.0;
    bool a0 = false;
    const int len = max(ol, fl);
    for (int j0 = 0; j0 < len; j0 += 2) {
      int oc[2], fc[2];
      double ov[2], fv[2];
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int j = j0 + t;
        oc[t] = (j < ol) ? ld_stream(SO.col + ob + 32LL * j + lane) : -1;
        ov[t] = (j < ol) ? ld_stream(SO.val + ob + 32LL * j + lane) : 0.0;
        fc[t] = (j < fl) ? ld_stream(SF.col + fb + 32LL * j + lane) : -1;
        fv[t] = (j < fl) ? ld_stream(SF.val + fb + 32LL * j + lane) : 0.0;
      }
      double op[2], a[2], b[2];
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        op[t] = (oc[t] >= 0) ? __ldg(p + oc[t]) : 0.0;
        a[t] = (fc[t] >= 0) ? __ldg(g + fc[t]) : 0.0;
        b[t] = (fc[t] >= 0) ? __ldg(q + fc[t]) : 0.0;
      }
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        if (oc[t] >= 0) {
          so = dadd(so, dmul(op[t], ov[t]));
          a0 = true;
        }
        if (fc[t] >= 0) {
          gs = dadd(gs, dmul(a[t], fv[t]));
          us = dadd(us, dmul(b[t], fv[t]));
        }
      }
    }
    a0 = a0 && f < SO.nrows;
    if (a0 || any_f) {
      double m = mf[f];
      if (a0) m = axpby_row(fact1, so, 0.0, m);
      if (any_f) {
        m = axpby_row(fact2, gs, 1.0, m);
        m = axpby_row(rho, us, 1.0, m);
      }
      mf[f] = m;
    }
  }
}

// mf = -dt SO p + dt SF gp + rho SF u, as seven ordered SpMV updates -- GIP_DNS.h:381-390
__global__ void __launch_bounds__(256) k_dns_massflux(
    SellView<double> SO, SellView<double> SFx, SellView<double> SFy, SellView<double> SFz,
    const double* __restrict__ p, const double* __restrict__ gpx, const double* __restrict__ gpy,
    const double* __restrict__ gpz, const double* __restrict__ u, const double* __restrict__ v,
    const double* __restrict__ w, double* __restrict__ mf, double rho, const DnsScalars* S) {
  const double sigma = S->sigma;
  const double fact1 = ddiv(-1.0, sigma);
  const double fact2 = ddiv(1.0, sigma);
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int ns = max(max(SO.nslices, SFx.nslices), max(SFy.nslices, SFz.nslices));
  for (int s = gw; s < ns; s += nw) {
    const int f = s * 32 + lane;
    double so = 0, gx = 0, gy = 0, gz = 0, ux = 0, uy = 0, uz = 0;
    bool a0 = false, ax = false, ay = false, az = false;
    if (s < SO.nslices) sell_row_f64(SO, p, s, lane, so, a0);
    // each SF row once, against the pressure gradient and the velocity together
    if (s < SFx.nslices) sell_row_f64_pair(SFx, gpx, u, s, lane, gx, ux, ax);
    if (s < SFy.nslices) sell_row_f64_pair(SFy, gpy, v, s, lane, gy, uy, ay);
    if (s < SFz.nslices) sell_row_f64_pair(SFz, gpz, w, s, lane, gz, uz, az);
    a0 = a0 && f < SO.nrows;
    ax = ax && f < SFx.nrows;
    ay = ay && f < SFy.nrows;
    az = az && f < SFz.nrows;
    if (a0 || ax || ay || az) {
      double m = mf[f];
      if (a0) m = axpby_row(fact1, so, 0.0, m);
      if (ax) m = axpby_row(fact2, gx, 1.0, m);
      if (ay) m = axpby_row(fact2, gy, 1.0, m);
      if (az) m = axpby_row(fact2, gz, 1.0, m);
      if (ax) m = axpby_row(rho, ux, 1.0, m);
      if (ay) m = axpby_row(rho, uy, 1.0, m);
      if (az) m = axpby_row(rho, uz, 1.0, m);
      mf[f] = m;
    }
  }
}

// ------------------------------------------------------------------ phase stamps
// Device time at phase boundary `mark` of the current step (the one-thread kernel runs
// after the previous phase's kernels and before the next phase's).  The boundary after the
// CFL kernel, which has already advanced the step counter, belongs to the step before.
__global__ void k_dns_stamp(const DnsScalars* __restrict__ S, DnsHistory H, int mark) {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  const int k = S->step - (mark == kPhaseMarks - 1 ? 1 : 0);
  if (k >= 0 && k < H.capacity) H.stamps[(size_t)k * kPhaseMarks + mark] = t;
}

// ------------------------------------------------------------------ CFLCondition
struct MassrFinish {
  const DnsScalars* S;
  DnsHistory H;
  __device__ void operator()(const double* t) const {
    const int k = S->step;
    if (k < H.capacity) H.massr[k] = t[0];
  }
};

// temp = Mres mf; massr = max |temp| over the inner cells   -- GIP_DNS.h:399-400
template <bool TAB>
__global__ void __launch_bounds__(256) k_dns_massr(SellView<double> Mres, const double* __restrict__ mf,
                                                   double* __restrict__ temp, int n_inner,
                                                   const DnsScalars* S, DnsHistory H,
                                                   ReduceScratch rs) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int ns = max(Mres.nslices, (n_inner + 31) / 32);
  double acc[1] = {0.0};
  for (int s = gw; s < ns; s += nw) {
    const int i = s * 32 + lane;
    double sum = 0;
    bool any = false;
    if (s < Mres.nslices) sell_row_f64<double, double, 8, TAB>(Mres, mf, s, lane, sum, any);
    any = any && i < Mres.nrows;
    if (any) temp[i] = sum;
    if (i < n_inner) {
      const double a = fabs(any ? sum : temp[i]);
      if (a > acc[0]) acc[0] = a;
    }
  }
  grid_reduce<MaxOp, 1>(acc, rs, MassrFinish{S, H});
}

__device__ __forceinline__ double cfl_candidate(double ut, double vt, double wt, double dx,
                                                double gamma, double rho, double dt) {
  const double convCoef = 0.25;
  double normit = (fabs(ut) > fabs(vt)) ? fabs(ut) : fabs(vt);
  if (normit < fabs(wt)) normit = fabs(wt);
  if (!(ddiv(dx, normit) < 1e-17)) {
    const double c = ddiv(dmul(convCoef, dx), normit);
    if (dt > c) dt = c;
  }
  if (!(ddiv(dmul(dmul(dx, dx), rho), gamma) < 1e-17)) {
    const double c = ddiv(dmul(dmul(dmul(0.2, dx), dx), rho), gamma);
    if (dt > c) dt = c;
  }
  return dt;
}

struct CflStepFinish {
  DnsScalars* S;
  DnsHistory H;
  const PcgScalars* P;
  int mode;  // 0: initial dt only (GIP_DNS.h:102-103); 1: end of a step (:402-408)
  int pcg_mixed;
  const double* dt_seq;  // prescribed steps (frozen-dt adjoint runs) or null
  int dt_seq_len;
  __device__ void operator()(const double* t) const {
    const double fin = t[0];
    double dtn = (dmul(0.8, fin) > 1e-1) ? 1e-1 : dmul(0.8, fin);
    if (dt_seq) {
      const int k = (mode == 1) ? S->step + 1 : S->step;
      dtn = dt_seq[k < dt_seq_len ? k : dt_seq_len - 1];
    }
    if (mode == 1) {
      const int k = S->step;
      const double tnew = dadd(S->time, S->dt);
      S->time = tnew;
      if (k < H.capacity) {
        H.time[k] = tnew;
        H.dt[k] = S->dt;
        H.iters[k] = pcg_mixed ? P->total_inner : P->iter;
        H.rr[k] = P->rr;
        H.outer[k] = pcg_mixed ? P->outer : 0;
        // the step's 10 kernels and the PCG's: init + 3 per iteration in the FP64 forms
        // (2 with AMG, whose V-cycle and direction kernels count themselves on the device),
        // all counted on the device in the mixed form
        H.kernels[k] = 10 + H.stamp_kernels +
                       (pcg_mixed ? P->kernels : 1 + (P->kernels ? 2 : 3) * P->iter + P->kernels);
      }
      S->step = k + 1;
    }
    S->dt = dtn;
    S->sigma = ddiv(1.0, dtn);
    S->started = 1;
  }
};

__global__ void __launch_bounds__(256) k_dns_cfl(int n, const double* __restrict__ u,
                                                 const double* __restrict__ v,
                                                 const double* __restrict__ w,
                                                 const double* __restrict__ dxs, double gamma,
                                                 double rho, DnsScalars* S, DnsHistory H,
                                                 const PcgScalars* P, int mode, int pcg_mixed,
                                                 const double* dt_seq, int dt_seq_len,
                                                 ReduceScratch rs) {
  double acc[1] = {1e20};
  // four cells per pass, their loads issued before any candidate is formed (the minimum
  // is exact in any order, so the result does not depend on the grouping)
  const int stride = gridDim.x * blockDim.x;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + 3 * stride < n; i += 4 * stride) {
    double cu[4], cv[4], cw[4], cd[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      cu[t] = u[i + t * stride];
      cv[t] = v[i + t * stride];
      cw[t] = w[i + t * stride];
      cd[t] = dxs[i + t * stride];
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) acc[0] = cfl_candidate(cu[t], cv[t], cw[t], cd[t], gamma, rho, acc[0]);
  }
  for (; i < n; i += stride) acc[0] = cfl_candidate(u[i], v[i], w[i], dxs[i], gamma, rho, acc[0]);
  grid_reduce<MinOp, 1>(acc, rs, CflStepFinish{S, H, P, mode, pcg_mixed, dt_seq, dt_seq_len});
}

// ------------------------------------------------------------------ engine
int Dns::grow_history(int need, cudaStream_t s) {
  if (need <= capacity) return GIPB200_OK;
  int cap = std::max(need, std::max(1024, capacity * 2));
  DevBuf<double> t, d, m, r;
  DevBuf<int> it, ou, kn;
  DevBuf<unsigned long long> st;
  GIPB_TRY(st.alloc((size_t)cap * kPhaseMarks));
  GIPB_CUDA(cudaMemsetAsync(st.p, 0, (size_t)cap * kPhaseMarks * 8, s));
  GIPB_TRY(ou.alloc(cap));
  GIPB_TRY(kn.alloc(cap));
  GIPB_TRY(t.alloc(cap));
  GIPB_TRY(d.alloc(cap));
  GIPB_TRY(m.alloc(cap));
  GIPB_TRY(r.alloc(cap));
  GIPB_TRY(it.alloc(cap));
  if (capacity > 0) {
    GIPB_CUDA(cudaMemcpyAsync(t.p, h_time.p, capacity * 8, cudaMemcpyDeviceToDevice, s));
    GIPB_CUDA(cudaMemcpyAsync(d.p, h_dt.p, capacity * 8, cudaMemcpyDeviceToDevice, s));
    GIPB_CUDA(cudaMemcpyAsync(m.p, h_massr.p, capacity * 8, cudaMemcpyDeviceToDevice, s));
    GIPB_CUDA(cudaMemcpyAsync(r.p, h_rr.p, capacity * 8, cudaMemcpyDeviceToDevice, s));
    GIPB_CUDA(cudaMemcpyAsync(it.p, h_iters.p, capacity * 4, cudaMemcpyDeviceToDevice, s));
    GIPB_CUDA(cudaMemcpyAsync(ou.p, h_outer.p, capacity * 4, cudaMemcpyDeviceToDevice, s));
    GIPB_CUDA(cudaMemcpyAsync(kn.p, h_kernels.p, capacity * 4, cudaMemcpyDeviceToDevice, s));
    GIPB_CUDA(cudaMemcpyAsync(st.p, h_stamps.p, (size_t)capacity * kPhaseMarks * 8,
                              cudaMemcpyDeviceToDevice, s));
  }
  GIPB_CUDA(cudaStreamSynchronize(s));
  std::swap(h_time.p, t.p);
  std::swap(h_dt.p, d.p);
  std::swap(h_massr.p, m.p);
  std::swap(h_rr.p, r.p);
  std::swap(h_iters.p, it.p);
  std::swap(h_outer.p, ou.p);
  std::swap(h_kernels.p, kn.p);
  std::swap(h_stamps.p, st.p);
  h_time.n = h_dt.n = h_massr.n = h_rr.n = h_iters.n = h_outer.n = h_kernels.n = cap;
  t.n = d.n = m.n = r.n = it.n = ou.n = kn.n = capacity;
  h_stamps.n = (size_t)cap * kPhaseMarks;
  st.n = (size_t)capacity * kPhaseMarks;
  capacity = cap;
  drop_graph();  // a captured graph refers to the old history arrays
  return GIPB200_OK;
}

int Dns::enqueue_initial_dt(cudaStream_t s) {
  k_dns_cfl<<<grid.cfl, 256, 0, s>>>(N, u.p, v.p, w.p, dxs.p, prm.gamma, prm.rho, sc.p,
                                        history(), pcg.sc.p, 0, 0,
                                        dt_seq_len > 0 ? dt_seq.p : nullptr, dt_seq_len, rs);
  GIPB_LAUNCH_CHECK();
  launches += 1;
  return GIPB200_OK;
}

int Dns::enqueue_step(cudaStream_t s, bool host_sync, int part) {
  const DnsHistory H = history();
  const long long pcg_before = pcg.launches;
  auto mark = [&](int k) {
    if (phase_events) cudaEventRecord(phase_events[k], s);
    if (stamps_on) k_dns_stamp<<<1, 1, 0, s>>>(sc.p, H, k);
  };
  if (part != 2) {
    mark(0);
    // PredictorVelocity: C's values from the face fluxes, then D/C products and AB2
    if (ec_slot && ec_ntab)
      GIPB_TRY(launch_csr_spmv_tab(ec_rows, ec_rp.p, ec_col.p, ec_vidx.p, ec_vtab.p, mf.p, cval.p,
                                   nullptr, 0.0, 0.0, 0, s));
    else if (ec_slot)
      GIPB_TRY(launch_csr_spmv(ec_rows, ec_rp.p, ec_col.p, ec_val.p, mf.p, cval.p, nullptr, 0.0,
                               0.0, 0, s));
    else
      GIPB_TRY(launch_csr_spmv(Ec.nrows, Ec.rowptr.p, Ec.csr_col.p, Ec.csr_val.p, mf.p, cval.p,
                               D.pos.p, 0.0, 0.0, 0, s));
    if (tab_d())
      k_dns_convdiff<true><<<grid.convdiff, 256, 0, s>>>(D.view(), cval.p, u.p, v.p, w.p, ax.p,
                                                         ay.p, az.p);
    else
      k_dns_convdiff<false><<<grid.convdiff, 256, 0, s>>>(D.view(), cval.p, u.p, v.p, w.p, ax.p,
                                                          ay.p, az.p);
    k_dns_ab2<<<grid.ab2, 256, 0, s>>>(N, u.p, v.p, w.p, ax.p, ay.p, az.p, ax0.p, ay0.p, az0.p,
                                       sc.p);
    mark(1);
    // PoissonEquation
    if (tab_m())
      k_dns_rhs<true><<<grid.rhs, 256, 0, s>>>(Mx.view(), My.view(), Mz.view(), u.p, v.p, w.p,
                                               rhs.p, sc.p);
    else
      k_dns_rhs<false><<<grid.rhs, 256, 0, s>>>(Mx.view(), My.view(), Mz.view(), u.p, v.p, w.p,
                                                rhs.p, sc.p);
    GIPB_LAUNCH_CHECK();
    mark(2);
  }
  if (part == 0) GIPB_TRY(pcg.enqueue(rhs.p, p.p, p0.p, s, host_sync));
  if (part != 1) {
    mark(3);
    k_dns_pcopy<<<blocks_owned, 256, 0, s>>>(N, NO, p.p, p0.p);
    GIPB_LAUNCH_CHECK();
    GIPB_TRY(launch_sell_spmv(Lb, Lb.val.p, p0.p, p.p, 1.0, 1.0, 1, s));
    mark(4);
    // VelocityCorrection
    k_dns_gradcorr<<<grid.gradcorr, 256, 0, s>>>(Gx.view(), Gy.view(), Gz.view(), p.p, gpx.p,
                                                 gpy.p, gpz.p, u.p, v.p, w.p, N, prm.rho, sc.p);
    mark(5);
    // MassFluxes
    if (SF3.on && SF3.single)
      k_dns_massflux1<<<grid.massflux, 256, 0, s>>>(SO.view(), SF3.S.view(), SF3.cnt.p, p.p,
                                                    gpx.p, gpy.p, gpz.p, u.p, v.p, w.p, mf.p,
                                                    prm.rho, sc.p);
    else if (SF3.on)
      k_dns_massflux3<<<grid.massflux, 256, 0, s>>>(SO.view(), SF3.S.view(), SF3.cnt.p, p.p,
                                                    gpx.p, gpy.p, gpz.p, u.p, v.p, w.p, mf.p,
                                                    prm.rho, sc.p);
    else
      k_dns_massflux<<<grid.massflux, 256, 0, s>>>(SO.view(), SFx.view(), SFy.view(), SFz.view(),
                                                   p.p, gpx.p, gpy.p, gpz.p, u.p, v.p, w.p, mf.p,
                                                   prm.rho, sc.p);
    mark(6);
    // CFLCondition
    if (Mres.ntab)
      k_dns_massr<true><<<grid.massr, 256, 0, s>>>(Mres.view(), mf.p, temp.p, N, sc.p, H, rs);
    else
      k_dns_massr<false><<<grid.massr, 256, 0, s>>>(Mres.view(), mf.p, temp.p, N, sc.p, H, rs);
    k_dns_cfl<<<grid.cfl, 256, 0, s>>>(N, u.p, v.p, w.p, dxs.p, prm.gamma, prm.rho, sc.p, H,
                                          pcg.sc.p, 1, prm.pcg.mode == GIPB200_PCG_MIXED,
                                          dt_seq_len > 0 ? dt_seq.p : nullptr, dt_seq_len, rs);
    GIPB_LAUNCH_CHECK();
    mark(7);
  }
  // the step's kernels: 4 before the solve, 6 after it, and the phase stamps
  const int own = part == 0 ? 10 : part == 1 ? 4 : 6;
  const int stamps = H.stamp_kernels == 0 ? 0 : part == 0 ? kPhaseMarks : part == 1 ? 3 : 5;
  launches += own + stamps + (pcg.launches - pcg_before);
  return GIPB200_OK;
}

// Compulsory traffic: every stored value and index once, slice offsets, each gathered
// vector once, each written vector once (a row without stored nonzeros writes nothing).
void Dns::phase_bytes(double out[7]) const {
  // a tabled operator streams a 4-byte column and a 1-byte value index per nonzero
  auto op = [](const Sell& M) {
    return (M.ntab ? 5.0 : 12.0) * M.nnz + 8.0 * (M.nslices + 1.0) + 8.0 * M.ntab;
  };
  const double n = N, no = NO, nf = NF;
  // predictor: C's values = Ec mf (CSR, rows scattered into C's slots), D/C products, AB2
  const double ec = ec_slot ? (ec_ntab ? 5.0 : 12.0) * Ec.nnz + 4.0 * (ec_rows + 1.0) + 8.0 * nf +
                                  8.0 * Ec.nrows
                            : 12.0 * Ec.nnz + 4.0 * (Ec.nrows + 1.0) + 4.0 * Ec.nrows + 8.0 * nf +
                                  8.0 * Ec.nrows;
  const double cd = op(D) + 8.0 * D.nnz + 24.0 * no + 24.0 * n;
  out[0] = ec + cd + 120.0 * n;
  out[1] = op(Mx) + op(My) + op(Mz) + 24.0 * no + 8.0 * n;          // rhs
  out[2] = 0.0;                                                      // PCG
  out[3] = 16.0 * no + op(Lb) + 24.0 * Lb.nnz;                       // p0/p copies, ghosts
  out[4] = op(Gx) + op(Gy) + op(Gz) + 8.0 * no + 24.0 * no + 48.0 * n;  // gp, u -= gp
  out[5] = op(SO) + (SF3.on ? op(SF3.S) + 2.0 * nf   // merged faces and their counts
                             : op(SFx) + op(SFy) + op(SFz)) +
           56.0 * no + 16.0 * nf;  // mf
  out[6] = op(Mres) + 8.0 * nf + 8.0 * n + 32.0 * n;                 // massr, CFL
}

double* Dns::field(const std::string& name, int* n) {
  struct E {
    const char* nm;
    DevBuf<double>* b;
    int sz;
  } tab[] = {{"u", &u, NO},     {"v", &v, NO},     {"w", &w, NO},     {"dxs", &dxs, NO},
             {"ax", &ax, NO},   {"ay", &ay, NO},   {"az", &az, NO},   {"ax0", &ax0, NO},
             {"ay0", &ay0, NO}, {"az0", &az0, NO}, {"rhs", &rhs, NO}, {"p", &p, NO},
             {"p0", &p0, NO},   {"gpx", &gpx, NO}, {"gpy", &gpy, NO}, {"gpz", &gpz, NO},
             {"temp", &temp, NO}, {"mf", &mf, NF}};
  for (auto& e : tab)
    if (name == e.nm) {
      *n = e.sz;
      return e.b->p;
    }
  return nullptr;
}

// ------------------------------------------------------------------ locality renumbering
// A std::allocator whose value-initialising construct() leaves the element uninitialised
// (renumbered operators are filled in parallel right after allocation).
template <typename T>
struct NoInitAlloc : std::allocator<T> {
  template <typename U>
  struct rebind {
    using other = NoInitAlloc<U>;
  };
  NoInitAlloc() = default;
  template <typename U>
  NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
  template <typename U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <typename U, typename... Args>
  void construct(U* p, Args&&... args) {
    ::new (static_cast<void*>(p)) U(std::forward<Args>(args)...);
  }
};

struct OwnedCsr {
  int nrows = 0, ncols = 0;
  std::vector<int, NoInitAlloc<int>> rp, col;
  std::vector<double, NoInitAlloc<double>> val;
  gipb200_host_csr view() const {
    gipb200_host_csr h;
    h.nrows = nrows;
    h.ncols = ncols;
    h.nnz = (int)col.size();
    h.rowptr = rp.data();
    h.col = col.data();
    h.val = val.data();
    return h;
  }
};

// Breadth-first order of the inner cells over L's graph, started from the last cell
// reached by a first sweep (a pseudo-peripheral cell), neighbours in stored order.
static void bfs_sweep(const gipb200_host_csr& L, int N, int start, std::vector<int>& order,
                      std::vector<char>& seen) {
  size_t head = order.size();
  order.push_back(start);
  seen[start] = 1;
  while (head < order.size()) {
    const int i = order[head++];
    if (i >= L.nrows) continue;
    for (int k = L.rowptr[i]; k < L.rowptr[i + 1]; ++k) {
      const int j = L.col[k];
      if (j >= 0 && j < N && !seen[j]) {
        seen[j] = 1;
        order.push_back(j);
      }
    }
  }
}

static std::vector<int> bfs_cells(const gipb200_host_csr& L, int N) {
  std::vector<int> order;
  order.reserve(N);
  std::vector<char> seen(N, 0);
  bfs_sweep(L, N, 0, order, seen);
  const int start = order.back();
  order.clear();
  std::fill(seen.begin(), seen.end(), 0);
  bfs_sweep(L, N, start, order, seen);
  for (int i = 0; i < N; ++i)
    if (!seen[i]) bfs_sweep(L, N, i, order, seen);
  return order;  // new -> old
}

// out row r = m row src[r] (src is a permutation of m's rows); columns through cmap
static void permute_rows(const gipb200_host_csr& m, const int* src, const int* cmap,
                         OwnedCsr* out) {
  out->nrows = m.nrows;
  out->ncols = m.ncols;
  out->rp.resize((size_t)m.nrows + 1);
  out->rp[0] = 0;
#pragma omp parallel for schedule(static)
  for (int r = 0; r < m.nrows; ++r) out->rp[r + 1] = m.rowptr[src[r] + 1] - m.rowptr[src[r]];
  for (int r = 0; r < m.nrows; ++r) out->rp[r + 1] += out->rp[r];
  out->col.resize((size_t)m.nnz);
  out->val.resize((size_t)m.nnz);
#pragma omp parallel for schedule(static)
  for (int r = 0; r < m.nrows; ++r) {
    int o = out->rp[r];
    for (int k = m.rowptr[src[r]]; k < m.rowptr[src[r] + 1]; ++k, ++o) {
      out->col[o] = cmap ? cmap[m.col[k]] : m.col[k];
      out->val[o] = m.val ? m.val[k] : 0.0;
    }
  }
}

__global__ void k_gather_field(int n, const int* __restrict__ perm, const double* __restrict__ in,
                               double* __restrict__ out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
    out[e] = in[perm[e]];
}
__global__ void k_scatter_field(int n, int offset, const int* __restrict__ perm,
                                const double* __restrict__ in, double* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    out[perm[offset + k]] = in[k];
}

static int check_op(const gipb200_host_csr& m, const char* name, int rows_max, int col_bound) {
  if (m.nrows > rows_max)
    return fail(GIPB200_ERR_ARG, "%s: %d rows exceed %d", name, m.nrows, rows_max);
  return validate_csr(m.nrows, m.ncols, m.nnz, m.rowptr, m.col, col_bound, name);
}

// The engine's sliced operators keep only what it reads: D its CSR columns and slot map
// (C's values, the adjoint), L everything (the solver's set-up), the others nothing.
// table: the phase kernel reads the values through a value table where the operator's
// values allow one (a uniform mesh's operators hold a handful of distinct values).  Used
// for D (C/D products), Mx/My/Mz (right-hand side) and Mres (massr), whose kernels gained
// 115, 16 and 53 us on the 256^3 cavity; the correction (G) gained nothing and the mass
// fluxes (SO, merged SF) lost 33 us to the dependent table read, so those read directly.
static int build_op(Sell* S, const gipb200_host_csr& m, unsigned keep = 0, bool table = false) {
  GIPB_TRY(sell_build(S, m.nrows, m.ncols, m.nnz, m.rowptr, m.col, m.val, 0, keep));
  if (table) GIPB_TRY(sell_add_value_table(S, m.val, m.nnz, 0));
  return GIPB200_OK;
}

// Sizes of an operator whose sliced layout is never read (phase byte counts only).
static void op_sizes(Sell* S, const gipb200_host_csr& m) {
  S->nrows = m.nrows;
  S->ncols = m.ncols;
  S->nnz = m.nnz;
  S->nslices = (m.nrows + 31) / 32;
}

// Ec in D's slot order (Dns::ec_slot): slot t of D's sliced layout holds the nonzero k of
// row i at position k - rowptr[i] of slice i / 32, lane i % 32.
static int build_ec_slot(Dns& E, const gipb200_host_csr& D, const gipb200_host_csr& Ec) {
  if (getenv("GIPB200_NO_EC_SLOT") || Ec.nrows != D.nnz) return GIPB200_OK;
  const int ns = (D.nrows + 31) / 32;
  std::vector<long long> sptr((size_t)ns + 1, 0);
  for (int sl = 0; sl < ns; ++sl) {
    int len = 0;
    for (int r = sl * 32; r < std::min(D.nrows, sl * 32 + 32); ++r)
      len = std::max(len, D.rowptr[r + 1] - D.rowptr[r]);
    sptr[sl + 1] = sptr[sl] + 32LL * len;
  }
  const long long nslots = sptr[ns];
  if (nslots > 0x7ffffffeLL) return GIPB200_OK;
  std::vector<int> src((size_t)nslots, -1);  // slot -> Ec row (the CSR nonzero of D)
#pragma omp parallel for schedule(static)
  for (int r = 0; r < D.nrows; ++r)
    for (int k = D.rowptr[r]; k < D.rowptr[r + 1]; ++k)
      src[(size_t)(sptr[r >> 5] + 32LL * (k - D.rowptr[r]) + (r & 31))] = k;
  // row lengths (in parallel), offsets, entries (in parallel)
  std::vector<int> rp((size_t)nslots + 1, 0);
#pragma omp parallel for schedule(static)
  for (long long t = 0; t < nslots; ++t) {
    const int k = src[(size_t)t];
    rp[(size_t)t + 1] = k >= 0 ? Ec.rowptr[k + 1] - Ec.rowptr[k] : 0;
  }
  for (long long t = 0; t < nslots; ++t) rp[(size_t)t + 1] += rp[(size_t)t];
  std::vector<int, NoInitAlloc<int>> col((size_t)rp[(size_t)nslots]);
  std::vector<double, NoInitAlloc<double>> val((size_t)rp[(size_t)nslots]);
#pragma omp parallel for schedule(static)
  for (long long t = 0; t < nslots; ++t) {
    const int k = src[(size_t)t];
    if (k < 0) continue;
    int o = rp[(size_t)t];
    for (int e = Ec.rowptr[k]; e < Ec.rowptr[k + 1]; ++e, ++o) {
      col[(size_t)o] = Ec.col[e];
      val[(size_t)o] = Ec.val[e];
    }
  }
  GIPB_TRY(E.ec_rp.upload(rp.data(), rp.size(), 0));
  GIPB_TRY(E.ec_col.upload(col.data(), std::max<size_t>(col.size(), 1), 0));
  // C's values through a value table of Ec's (few) distinct values where they allow one
  std::vector<double> tab;
  E.ec_ntab = 0;
  if (!getenv("GIPB200_NO_VALUE_TABLE") && !val.empty() &&
      value_table(val.data(), (long long)val.size(), 256, &tab)) {
    std::vector<unsigned long long> keys(tab.size());
    for (size_t t = 0; t < tab.size(); ++t) memcpy(&keys[t], &tab[t], 8);
    std::vector<unsigned char, NoInitAlloc<unsigned char>> idx(val.size());
#pragma omp parallel for schedule(static)
    for (long long e = 0; e < (long long)val.size(); ++e) {
      unsigned long long b;
      memcpy(&b, &val[(size_t)e], 8);
      idx[(size_t)e] =
          (unsigned char)(std::lower_bound(keys.begin(), keys.end(), b) - keys.begin());
    }
    GIPB_TRY(E.ec_vidx.upload(idx.data(), idx.size(), 0));
    GIPB_TRY(E.ec_vtab.upload(tab.data(), tab.size(), 0));
    E.ec_ntab = (int)tab.size();
  } else {
    GIPB_TRY(E.ec_val.upload(val.data(), std::max<size_t>(val.size(), 1), 0));
  }
  GIPB_CUDA(cudaStreamSynchronize(0));
  E.ec_rows = (int)nslots;
  E.ec_slot = true;
  return GIPB200_OK;
}

// FaceOps3 from the three face operators (host CSR, NF rows or none).  Left off when a
// face row of one operator has more than 15 entries.
static int build_face3(FaceOps3* F, const gipb200_host_csr* const op[3], int NF, int NO) {
  F->on = false;
  if (NF <= 0 || getenv("GIPB200_NO_FACE3")) return GIPB200_OK;
  // counts per face (in parallel), offsets, then the entries (in parallel)
  std::vector<int> rp((size_t)NF + 1, 0);
  std::vector<unsigned short> cnt((size_t)NF, 0);
  int too_long = 0, mixed = 0;
#pragma omp parallel for schedule(static) reduction(| : too_long, mixed)
  for (int f = 0; f < NF; ++f) {
    unsigned packed = 0, ops_here = 0;
    int total = 0;
    for (int o = 0; o < 3; ++o) {
      const gipb200_host_csr& m = *op[o];
      if (f >= m.nrows) continue;
      const int c = m.rowptr[f + 1] - m.rowptr[f];
      if (c > 15) too_long = 1;
      packed |= (unsigned)(c & 15) << (4 * o);
      ops_here += c > 0 ? 1u : 0u;
      total += c;
    }
    cnt[f] = (unsigned short)packed;
    rp[(size_t)f + 1] = total;
    if (ops_here > 1) mixed = 1;
  }
  if (too_long) return GIPB200_OK;
  const bool single = !mixed;
  for (int f = 0; f < NF; ++f) rp[(size_t)f + 1] += rp[f];
  std::vector<int, NoInitAlloc<int>> col((size_t)rp[NF]);
  std::vector<double, NoInitAlloc<double>> val((size_t)rp[NF]);
#pragma omp parallel for schedule(static)
  for (int f = 0; f < NF; ++f) {
    int o2 = rp[f];
    for (int o = 0; o < 3; ++o) {
      const gipb200_host_csr& m = *op[o];
      if (f >= m.nrows) continue;
      for (int k = m.rowptr[f]; k < m.rowptr[f + 1]; ++k, ++o2) {
        col[(size_t)o2] = m.col[k];
        val[(size_t)o2] = m.val[k];
      }
    }
  }
  GIPB_TRY(sell_build(&F->S, NF, NO, (int)col.size(), rp.data(), col.data(), val.data(), 0, 0u));
  GIPB_TRY(F->cnt.upload(cnt.data(), cnt.size(), 0));
  GIPB_CUDA(cudaStreamSynchronize(0));
  F->on = true;
  F->single = single && !getenv("GIPB200_NO_FACE1");
  return GIPB200_OK;
}

int check_dns_ops(const gipb200_dns_ops* ops) {
  const int N = ops->n_inner, NO = ops->n_owned, NF = ops->n_faces;
  if (N <= 0 || NO < N || NF < 0) return fail(GIPB200_ERR_ARG, "bad topology sizes");
  // row/column spaces of GIP_DNS's operators (GIP_DNS.h:143-238)
  GIPB_TRY(check_op(ops->D, "D", N, NO));
  GIPB_TRY(check_op(ops->L, "L", N, NO));
  GIPB_TRY(check_op(ops->Lb, "Lb", NO, NO));
  GIPB_TRY(check_op(ops->Mx, "Mx", N, NO));
  GIPB_TRY(check_op(ops->My, "My", N, NO));
  GIPB_TRY(check_op(ops->Mz, "Mz", N, NO));
  GIPB_TRY(check_op(ops->Mres, "Mres", N, NF));
  GIPB_TRY(check_op(ops->Gx, "Gx", NO, NO));
  GIPB_TRY(check_op(ops->Gy, "Gy", NO, NO));
  GIPB_TRY(check_op(ops->Gz, "Gz", NO, NO));
  GIPB_TRY(check_op(ops->SFx, "SFx", NF, NO));
  GIPB_TRY(check_op(ops->SFy, "SFy", NF, NO));
  GIPB_TRY(check_op(ops->SFz, "SFz", NF, NO));
  GIPB_TRY(check_op(ops->SO, "SO", NF, NO));
  GIPB_TRY(check_op(ops->Ec, "Ec", ops->D.nnz, NF));
  if (ops->Ec.nrows != ops->D.nnz)
    return fail(GIPB200_ERR_ARG, "Ec has %d rows, D has %d nonzeros", ops->Ec.nrows, ops->D.nnz);

  return GIPB200_OK;
}

int dns_init(Dns& E, const gipb200_dns_ops* ops, const double* h_u, const double* h_v,
             const double* h_w, const double* h_dxs, const gipb200_dns_params* prm) {
  const auto t_begin = std::chrono::steady_clock::now();
  auto since = [](std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
  };
  auto trace = [](const char* what) { setup_mark(what); };
  trace("start");
  GIPB_TRY(check_dns_ops(ops));
  trace("operator checks");
  if (prm->pcg.mode < 0 || prm->pcg.mode > 2) return fail(GIPB200_ERR_ARG, "bad PCG mode");
  const int N = ops->n_inner, NO = ops->n_owned, NF = ops->n_faces;
    E.N = N;
    E.NO = NO;
    E.NF = NF;
    E.prm = *prm;
    // Renumbering needs every operator's row space complete (cell rows: 0, N or NO rows;
    // face rows: 0 or NF rows), which GIP's operators satisfy at one rank.
    const gipb200_host_csr* all_ops[] = {&ops->D, &ops->L, &ops->Lb, &ops->Mx, &ops->My,
                                         &ops->Mz, &ops->Mres, &ops->Gx, &ops->Gy, &ops->Gz,
                                         &ops->SFx, &ops->SFy, &ops->SFz, &ops->SO};
    bool can_reorder = prm->reorder != 0 && ops->D.nrows == N;
    for (int k = 0; k < 10; ++k) {
      const int r = all_ops[k]->nrows;
      can_reorder = can_reorder && (r == 0 || r == N || r == NO);
    }
    for (int k = 10; k < 14; ++k) can_reorder = can_reorder && (all_ops[k]->nrows == 0 || all_ops[k]->nrows == NF);
    gipb200_dns_ops rops = *ops;
    OwnedCsr own[15];
    std::vector<double> fu, fv, fw, fdx;
    const double *pu = h_u, *pv = h_v, *pw = h_w, *pdx = h_dxs;
    if (can_reorder) {
      std::vector<int> inv_c = bfs_cells(ops->L, N);  // new -> old (inner)
      trace("breadth-first cells");
      inv_c.resize(NO);
      for (int g = N; g < NO; ++g) inv_c[g] = g;
      std::vector<int> perm_c(NO);
      for (int r = 0; r < NO; ++r) perm_c[inv_c[r]] = r;
      // faces ordered by the first (renumbered) inner cell that has them, then by face
      // index (faces of no inner cell last): a counting sort on that cell, filled in face
      // order
      std::vector<int> first_cell(NF, NO);
      for (int i = 0; i < ops->Mres.nrows; ++i)
        for (int k = ops->Mres.rowptr[i]; k < ops->Mres.rowptr[i + 1]; ++k) {
          const int f = ops->Mres.col[k];
          first_cell[f] = std::min(first_cell[f], perm_c[i]);
        }
      std::vector<int> bucket((size_t)NO + 2, 0);
      for (int f = 0; f < NF; ++f) bucket[(size_t)first_cell[f] + 1]++;
      for (int c = 0; c <= NO; ++c) bucket[(size_t)c + 1] += bucket[c];
      std::vector<int> inv_f(NF);
      for (int f = 0; f < NF; ++f) inv_f[bucket[first_cell[f]]++] = f;
      trace("face order");
      std::vector<int> perm_f(NF);
      for (int r = 0; r < NF; ++r) perm_f[inv_f[r]] = r;
      auto cell_op = [&](const gipb200_host_csr& m, OwnedCsr* o, bool face_cols) {
        permute_rows(m, inv_c.data(), face_cols ? perm_f.data() : perm_c.data(), o);
      };
      auto face_op = [&](const gipb200_host_csr& m, OwnedCsr* o) {
        permute_rows(m, inv_f.data(), perm_c.data(), o);
      };
      cell_op(ops->D, &own[0], false);
      cell_op(ops->L, &own[1], false);
      cell_op(ops->Lb, &own[2], false);
      cell_op(ops->Mx, &own[3], false);
      cell_op(ops->My, &own[4], false);
      cell_op(ops->Mz, &own[5], false);
      cell_op(ops->Mres, &own[6], true);
      cell_op(ops->Gx, &own[7], false);
      cell_op(ops->Gy, &own[8], false);
      cell_op(ops->Gz, &own[9], false);
      face_op(ops->SFx, &own[10]);
      face_op(ops->SFy, &own[11]);
      face_op(ops->SFz, &own[12]);
      face_op(ops->SO, &own[13]);
      // Ec rows follow the renumbered D's nonzeros, each kept in its stored order
      std::vector<int> ec_src;
      ec_src.reserve((size_t)ops->D.nnz);
      for (int r = 0; r < N; ++r)
        for (int k = ops->D.rowptr[inv_c[r]]; k < ops->D.rowptr[inv_c[r] + 1]; ++k) ec_src.push_back(k);
      permute_rows(ops->Ec, ec_src.data(), perm_f.data(), &own[14]);
      trace("operators renumbered");
      rops.D = own[0].view();
      rops.L = own[1].view();
      rops.Lb = own[2].view();
      rops.Mx = own[3].view();
      rops.My = own[4].view();
      rops.Mz = own[5].view();
      rops.Mres = own[6].view();
      rops.Gx = own[7].view();
      rops.Gy = own[8].view();
      rops.Gz = own[9].view();
      rops.SFx = own[10].view();
      rops.SFy = own[11].view();
      rops.SFz = own[12].view();
      rops.SO = own[13].view();
      rops.Ec = own[14].view();
      fu.resize(NO);
      fv.resize(NO);
      fw.resize(NO);
      fdx.resize(NO);
      for (int e = 0; e < NO; ++e) {
        fu[perm_c[e]] = h_u[e];
        fv[perm_c[e]] = h_v[e];
        fw[perm_c[e]] = h_w[e];
        fdx[perm_c[e]] = h_dxs[e];
      }
      pu = fu.data();
      pv = fv.data();
      pw = fw.data();
      pdx = fdx.data();
      GIPB_TRY(E.perm_c.upload(perm_c.data(), NO));
      GIPB_TRY(E.perm_f.upload(perm_f.data(), std::max(NF, 1)));
      GIPB_TRY(E.staging.alloc(std::max(NO, NF)));
      E.reordered = true;
    }
    E.setup_s[0] = since(t_begin);  // checks and renumbering
    const auto t_ops = std::chrono::steady_clock::now();
    const gipb200_dns_ops* bops = &rops;
    GIPB_TRY(build_op(&E.D, bops->D, kKeepDeviceCsr | kKeepPos, true));
    trace("sliced D");
    // Ec is only ever read row by row in CSR form (C's values, the adjoint's convective
    // term): no sliced copy
    GIPB_TRY(csr_build(&E.Ec, bops->Ec.nrows, bops->Ec.ncols, bops->Ec.nnz, bops->Ec.rowptr,
                       bops->Ec.col, bops->Ec.val, 0));
    GIPB_TRY(build_op(&E.L, bops->L, kKeepAll));
    trace("sliced L");
    GIPB_TRY(build_op(&E.Lb, bops->Lb));
    trace("sliced Lb");
    GIPB_TRY(build_op(&E.Mx, bops->Mx, 0, true));
    trace("sliced Mx");
    GIPB_TRY(build_op(&E.My, bops->My, 0, true));
    trace("sliced My");
    GIPB_TRY(build_op(&E.Mz, bops->Mz, 0, true));
    trace("sliced Mz");
    GIPB_TRY(build_op(&E.Mres, bops->Mres, 0, true));
    trace("sliced Mres");
    GIPB_TRY(build_op(&E.Gx, bops->Gx));
    trace("sliced Gx");
    GIPB_TRY(build_op(&E.Gy, bops->Gy));
    trace("sliced Gy");
    GIPB_TRY(build_op(&E.Gz, bops->Gz));
    trace("sliced Gz");
    {
      // SFx, SFy, SFz merged per face where they fit; their own layouts only otherwise
      const gipb200_host_csr* sf[3] = {&bops->SFx, &bops->SFy, &bops->SFz};
      GIPB_TRY(build_face3(&E.SF3, sf, NF, NO));
      if (E.SF3.on) {
        op_sizes(&E.SFx, bops->SFx);
        op_sizes(&E.SFy, bops->SFy);
        op_sizes(&E.SFz, bops->SFz);
      } else {
        GIPB_TRY(build_op(&E.SFx, bops->SFx));
        GIPB_TRY(build_op(&E.SFy, bops->SFy));
        GIPB_TRY(build_op(&E.SFz, bops->SFz));
      }
    }
    trace("face operators");
    GIPB_TRY(build_op(&E.SO, bops->SO));
    trace("sliced SO");
    GIPB_TRY(build_ec_slot(E, bops->D, bops->Ec));
    trace("Ec in C's slot order");
    // C starts with D's values (C.postConstruct reads the D file, GIP_DNS.h:151)
    GIPB_TRY(E.cval.alloc((size_t)std::max<long long>(E.D.nslots, 1)));
    GIPB_CUDA(cudaMemcpy(E.cval.p, E.D.val.p, E.cval.n * 8, cudaMemcpyDeviceToDevice));
    DevBuf<double>* cells[] = {&E.u, &E.v, &E.w, &E.dxs, &E.ax, &E.ay, &E.az, &E.ax0, &E.ay0,
                               &E.az0, &E.rhs, &E.p, &E.p0, &E.gpx, &E.gpy, &E.gpz, &E.temp};
    for (auto* b : cells) {
      GIPB_TRY(b->alloc(NO));
      GIPB_TRY(b->zero());
    }
    GIPB_TRY(E.mf.alloc(std::max(NF, 1)));
    GIPB_TRY(E.mf.zero());
    GIPB_CUDA(cudaMemcpy(E.u.p, pu, (size_t)NO * 8, cudaMemcpyHostToDevice));
    GIPB_CUDA(cudaMemcpy(E.v.p, pv, (size_t)NO * 8, cudaMemcpyHostToDevice));
    GIPB_CUDA(cudaMemcpy(E.w.p, pw, (size_t)NO * 8, cudaMemcpyHostToDevice));
    GIPB_CUDA(cudaMemcpy(E.dxs.p, pdx, (size_t)NO * 8, cudaMemcpyHostToDevice));
    trace("merged faces, fields");
    E.setup_s[1] = since(t_ops);  // device layouts of the operators, fields
    const auto t_pcg = std::chrono::steady_clock::now();
    GIPB_TRY(E.pcg.init(&E.L, NO, prm->pcg, 0));
    trace("pressure solver");
    E.setup_s[2] = since(t_pcg);  // the pressure solver (FP32 operator, packing, AMG)
    GIPB_TRY(E.sc.alloc(1));
    GIPB_TRY(E.sc.zero());
    GIPB_TRY(reduce_scratch_alloc(&E.partials, &E.ticket, &E.rs));
    GIPB_TRY(E.grow_history(1024, 0));
    GIPB_TRY(grid_blocks(256, std::max(N, NO), 1, kMaxReduceBlocks, &E.blocks_cells));
    GIPB_TRY(grid_blocks(256, std::max(NF, 1), 1, kMaxReduceBlocks, &E.blocks_faces));
    GIPB_TRY(grid_blocks(256, NO, 1, kMaxReduceBlocks, &E.blocks_owned));
    GIPB_TRY(grid_blocks(256, N, 4, kMaxReduceBlocks, &E.blocks_vec));
    GIPB_TRY(E.tab_d() ? one_wave(k_dns_convdiff<true>, E.blocks_cells, &E.grid.convdiff)
                       : one_wave(k_dns_convdiff<false>, E.blocks_cells, &E.grid.convdiff));
    GIPB_TRY(one_wave(k_dns_ab2, E.blocks_vec, &E.grid.ab2));
    GIPB_TRY(E.tab_m() ? one_wave(k_dns_rhs<true>, E.blocks_cells, &E.grid.rhs)
                       : one_wave(k_dns_rhs<false>, E.blocks_cells, &E.grid.rhs));
    GIPB_TRY(one_wave(k_dns_gradcorr, E.blocks_owned, &E.grid.gradcorr));
    if (E.SF3.on && E.SF3.single)
      GIPB_TRY(one_wave(k_dns_massflux1, E.blocks_faces, &E.grid.massflux));
    else if (E.SF3.on)
      GIPB_TRY(one_wave(k_dns_massflux3, E.blocks_faces, &E.grid.massflux));
    else
      GIPB_TRY(one_wave(k_dns_massflux, E.blocks_faces, &E.grid.massflux));
    GIPB_TRY(E.Mres.ntab ? one_wave(k_dns_massr<true>, E.blocks_cells, &E.grid.massr)
                         : one_wave(k_dns_massr<false>, E.blocks_cells, &E.grid.massr));
    GIPB_TRY(one_wave(k_dns_cfl, E.blocks_vec, &E.grid.cfl));
    GIPB_CUDA(cudaStreamCreateWithFlags(&E.cap_stream, cudaStreamNonBlocking));
    GIPB_CUDA(cudaDeviceSynchronize());
    E.setup_s[3] = since(t_begin);
    return GIPB200_OK;
}

int dns_advance(Dns& E, int nsteps, cudaStream_t s) {
  GIPB_TRY(E.grow_history(E.steps_enqueued + nsteps, s));
  if (!E.started) {
    GIPB_TRY(E.enqueue_initial_dt(s));
    E.started = true;
  }
  // Every mode is graphable: FIXED unrolls its iterations, TOL/MIXED loop in
  // conditional while-nodes that the device stops.
  const bool graphable = E.prm.use_graph != 0;
  for (int k = 0; k < nsteps; ++k) {
    if (graphable) {
      if (!E.exec) {
        cudaStream_t cs = E.cap_stream;
        GIPB_CUDA(cudaStreamSynchronize(s));
        GIPB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        const long long before = E.launches;
        int st = E.enqueue_step(cs, false);
        E.graph_kernels = E.launches - before;
        E.launches = before;
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(cs, &g);
        if (st != GIPB200_OK) {
          if (g) cudaGraphDestroy(g);
          return st;
        }
        if (ce != cudaSuccess)
          return fail(GIPB200_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
        E.graph = g;
        GIPB_CUDA(cudaGraphInstantiate(&E.exec, E.graph, 0));
      }
      GIPB_CUDA(cudaGraphLaunch(E.exec, s));
      E.launches += E.graph_kernels;
    } else {
      GIPB_TRY(E.enqueue_step(s, true));
    }
    E.steps_enqueued += 1;
  }
  return GIPB200_OK;
}

}  // namespace gipb200

using namespace gipb200;

extern "C" {

int gipb200_dns_create(const gipb200_dns_ops* ops, const double* h_u, const double* h_v,
                       const double* h_w, const double* h_dxs, const gipb200_dns_params* prm,
                       gipb200_dns* out) {
  if (!ops || !prm || !out || !h_u || !h_v || !h_w || !h_dxs)
    return fail(GIPB200_ERR_ARG, "null argument");
  *out = nullptr;
  gipb200_dns D = new (std::nothrow) gipb200_dns_s();
  if (!D) return fail(GIPB200_ERR_NOMEM, "host allocation failed");
  int st = dns_init(D->E, ops, h_u, h_v, h_w, h_dxs, prm);
  if (st != GIPB200_OK) {
    delete D;
    return st;
  }
  *out = D;
  return GIPB200_OK;
}

int gipb200_dns_destroy(gipb200_dns D) {
  delete D;
  return GIPB200_OK;
}

int gipb200_dns_advance(gipb200_dns Dh, int nsteps, void* stream) {
  if (!Dh || nsteps < 0) return fail(GIPB200_ERR_ARG, "bad arguments");
  return dns_advance(Dh->E, nsteps, as_stream(stream));
}

int gipb200_dns_step_phases(gipb200_dns Dh, void* stream, double* h_ms) {
  if (!Dh || !h_ms) return fail(GIPB200_ERR_ARG, "null argument");
  Dns& E = Dh->E;
  cudaStream_t s = as_stream(stream);
  GIPB_TRY(E.grow_history(E.steps_enqueued + 1, s));
  if (!E.started) {
    GIPB_TRY(E.enqueue_initial_dt(s));
    E.started = true;
  }
  cudaEvent_t ev[8];
  int made = 0;
  int st = GIPB200_OK;
  for (; made < 8; ++made)
    if (cudaEventCreate(&ev[made]) != cudaSuccess) {
      st = fail(GIPB200_ERR_CUDA, "cudaEventCreate failed");
      break;
    }
  if (st == GIPB200_OK) {
    E.phase_events = ev;
    st = E.enqueue_step(s, true);
    E.phase_events = nullptr;
    if (st == GIPB200_OK) {
      E.steps_enqueued += 1;
      if (cudaEventSynchronize(ev[7]) != cudaSuccess) st = fail(GIPB200_ERR_CUDA, "step failed");
      for (int k = 0; k < 7 && st == GIPB200_OK; ++k) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ev[k], ev[k + 1]) != cudaSuccess)
          st = fail(GIPB200_ERR_CUDA, "cudaEventElapsedTime failed");
        h_ms[k] = ms;
      }
    }
  }
  for (int k = 0; k < made; ++k) cudaEventDestroy(ev[k]);
  return st;
}

int gipb200_dns_phase_stamps(gipb200_dns Dh, int on) {
  if (!Dh) return fail(GIPB200_ERR_ARG, "null engine");
  Dns& E = Dh->E;
  if (E.stamps_on != (on != 0)) {
    GIPB_CUDA(cudaDeviceSynchronize());  // a launched graph may still run
    E.stamps_on = on != 0;
    E.drop_graph();  // the next advance captures the step with (or without) the stamps
  }
  return GIPB200_OK;
}

int gipb200_dns_phase_history(gipb200_dns Dh, int max_steps, double* h_ms, int* steps_out) {
  if (!Dh || max_steps < 0 || (max_steps > 0 && !h_ms)) return fail(GIPB200_ERR_ARG, "bad arguments");
  Dns& E = Dh->E;
  GIPB_CUDA(cudaDeviceSynchronize());
  DnsScalars S;
  GIPB_CUDA(cudaMemcpy(&S, E.sc.p, sizeof(S), cudaMemcpyDeviceToHost));
  const int n = std::min(std::min(S.step, E.capacity), max_steps);
  if (steps_out) *steps_out = n;
  if (n <= 0) return GIPB200_OK;
  std::vector<unsigned long long> st((size_t)n * kPhaseMarks);
  GIPB_CUDA(cudaMemcpy(st.data(), E.h_stamps.p, st.size() * 8, cudaMemcpyDeviceToHost));
  for (int k = 0; k < n; ++k)
    for (int ph = 0; ph < kPhaseMarks - 1; ++ph) {
      const unsigned long long a = st[(size_t)k * kPhaseMarks + ph];
      const unsigned long long b = st[(size_t)k * kPhaseMarks + ph + 1];
      h_ms[(size_t)k * (kPhaseMarks - 1) + ph] =
          (a && b && b >= a) ? (double)(b - a) * 1e-6 : std::nan("");
    }
  return GIPB200_OK;
}

int gipb200_dns_history(gipb200_dns Dh, int* steps, double* t, double* dt, double* massr,
                        int* iters, double* rr, int* outer, int* kernels) {
  if (!Dh) return fail(GIPB200_ERR_ARG, "null engine");
  Dns& E = Dh->E;
  GIPB_CUDA(cudaDeviceSynchronize());
  DnsScalars S;
  GIPB_CUDA(cudaMemcpy(&S, E.sc.p, sizeof(S), cudaMemcpyDeviceToHost));
  const int n = std::min(S.step, E.capacity);
  if (steps) *steps = S.step;
  if (t && n) GIPB_CUDA(cudaMemcpy(t, E.h_time.p, n * 8, cudaMemcpyDeviceToHost));
  if (dt && n) GIPB_CUDA(cudaMemcpy(dt, E.h_dt.p, n * 8, cudaMemcpyDeviceToHost));
  if (massr && n) GIPB_CUDA(cudaMemcpy(massr, E.h_massr.p, n * 8, cudaMemcpyDeviceToHost));
  if (iters && n) GIPB_CUDA(cudaMemcpy(iters, E.h_iters.p, n * 4, cudaMemcpyDeviceToHost));
  if (rr && n) GIPB_CUDA(cudaMemcpy(rr, E.h_rr.p, n * 8, cudaMemcpyDeviceToHost));
  if (outer && n) GIPB_CUDA(cudaMemcpy(outer, E.h_outer.p, n * 4, cudaMemcpyDeviceToHost));
  if (kernels && n) GIPB_CUDA(cudaMemcpy(kernels, E.h_kernels.p, n * 4, cudaMemcpyDeviceToHost));
  return GIPB200_OK;
}

int gipb200_dns_get_field(gipb200_dns Dh, const char* name, double* h_out, int n) {
  if (!Dh || !name || !h_out) return fail(GIPB200_ERR_ARG, "null argument");
  int sz = 0;
  double* p = Dh->E.field(name, &sz);
  if (!p) return fail(GIPB200_ERR_ARG, "unknown field '%s'", name);
  if (n < sz) return fail(GIPB200_ERR_ARG, "buffer of %d for field of %d", n, sz);
  Dns& E = Dh->E;
  GIPB_CUDA(cudaDeviceSynchronize());
  if (E.reordered && sz > 0) {
    const int* perm = (sz == E.NF && std::string(name) == "mf") ? E.perm_f.p : E.perm_c.p;
    int b;
    GIPB_TRY(grid_blocks(256, sz, 4, 0, &b));
    k_gather_field<<<b, 256>>>(sz, perm, p, E.staging.p);
    GIPB_LAUNCH_CHECK();
    GIPB_CUDA(cudaMemcpy(h_out, E.staging.p, (size_t)sz * 8, cudaMemcpyDeviceToHost));
    return GIPB200_OK;
  }
  GIPB_CUDA(cudaMemcpy(h_out, p, (size_t)sz * 8, cudaMemcpyDeviceToHost));
  return GIPB200_OK;
}

int gipb200_dns_copy_field(gipb200_dns Dh, const char* name, double* d_out, int n, void* stream) {
  if (!Dh || !name || !d_out) return fail(GIPB200_ERR_ARG, "null argument");
  int sz = 0;
  double* p = Dh->E.field(name, &sz);
  if (!p) return fail(GIPB200_ERR_ARG, "unknown field '%s'", name);
  if (n < sz) return fail(GIPB200_ERR_ARG, "buffer of %d for field of %d", n, sz);
  Dns& E = Dh->E;
  cudaStream_t s = as_stream(stream);
  if (sz == 0) return GIPB200_OK;
  if (E.reordered) {
    const int* perm = (std::string(name) == "mf") ? E.perm_f.p : E.perm_c.p;
    int b;
    GIPB_TRY(grid_blocks(256, sz, 4, 0, &b));
    k_gather_field<<<b, 256, 0, s>>>(sz, perm, p, d_out);
    GIPB_LAUNCH_CHECK();
  } else {
    GIPB_CUDA(cudaMemcpyAsync(d_out, p, (size_t)sz * 8, cudaMemcpyDeviceToDevice, s));
  }
  return GIPB200_OK;
}

int gipb200_dns_field_ptr(gipb200_dns Dh, const char* name, double** d_ptr, int* n) {
  if (!Dh || !name || !d_ptr) return fail(GIPB200_ERR_ARG, "null argument");
  int sz = 0;
  double* p = Dh->E.field(name, &sz);
  if (!p) return fail(GIPB200_ERR_ARG, "unknown field '%s'", name);
  *d_ptr = p;
  if (n) *n = sz;
  return GIPB200_OK;
}

int gipb200_dns_set_field(gipb200_dns Dh, const char* name, const double* h_in, int offset,
                          int n, void* stream) {
  if (!Dh || !name || (!h_in && n)) return fail(GIPB200_ERR_ARG, "null argument");
  int sz = 0;
  double* p = Dh->E.field(name, &sz);
  if (!p) return fail(GIPB200_ERR_ARG, "unknown field '%s'", name);
  if (offset < 0 || n < 0 || (long long)offset + n > sz)
    return fail(GIPB200_ERR_ARG, "range [%d,%d) outside field of %d", offset, offset + n, sz);
  if (!n) return GIPB200_OK;
  Dns& E = Dh->E;
  cudaStream_t s = as_stream(stream);
  if (E.reordered) {
    const int* perm = (std::string(name) == "mf") ? E.perm_f.p : E.perm_c.p;
    GIPB_CUDA(cudaMemcpyAsync(E.staging.p, h_in, (size_t)n * 8, cudaMemcpyHostToDevice, s));
    int b;
    GIPB_TRY(grid_blocks(256, n, 4, 0, &b));
    k_scatter_field<<<b, 256, 0, s>>>(n, offset, perm, E.staging.p, p);
    GIPB_LAUNCH_CHECK();
  } else {
    GIPB_CUDA(cudaMemcpyAsync(p + offset, h_in, (size_t)n * 8, cudaMemcpyHostToDevice, s));
  }
  return GIPB200_OK;
}

int gipb200_dns_set_launch(gipb200_dns Dh, int spmv_blocks, int vec_blocks) {
  if (!Dh) return fail(GIPB200_ERR_ARG, "null engine");
  Dns& E = Dh->E;
  GIPB_TRY(E.pcg.set_launch(spmv_blocks, vec_blocks));
  if (E.exec) {
    cudaGraphExecDestroy(E.exec);
    E.exec = nullptr;
  }
  if (E.graph) {
    cudaGraphDestroy(E.graph);
    E.graph = nullptr;
  }
  return GIPB200_OK;
}

int gipb200_dns_get_info(gipb200_dns Dh, gipb200_dns_info* info) {
  if (!Dh || !info) return fail(GIPB200_ERR_ARG, "null argument");
  const Dns& E = Dh->E;
  info->reordered = E.reordered;
  info->pin_row = E.pcg.pin_row;
  info->compressed = E.pcg.cop.enabled;
  info->value_table = E.pcg.cop.index_bits;
  info->compressed_fraction = E.pcg.cop.compressed_fraction;
  info->slots_L = E.L.nslots;
  info->nnz_L = E.L.nnz;
  const Amg* amg = E.pcg.amg.get();
  const Amg64* amg64 = E.pcg.amg64.get();
  info->amg_levels = amg ? (int)amg->lv.size() : amg64 ? (int)amg64->lv.size() : 0;
  info->amg_complexity = amg ? amg->op_complexity : amg64 ? amg64->op_complexity : 0.0;
  info->amg_setup_s = amg ? amg->setup_s : amg64 ? amg64->setup_s : 0.0;
  info->iteration_bytes = E.pcg.iteration_bytes();
  info->replacement_bytes = E.pcg.replacement_bytes();
  info->packed_residual = E.pcg.lpacked ? 1 : 0;
  info->value_tables = E.value_tables();
  return GIPB200_OK;
}

int gipb200_dns_snapshot(gipb200_dns Dh, int restore, void* stream) {
  if (!Dh) return fail(GIPB200_ERR_ARG, "null engine");
  Dns& E = Dh->E;
  cudaStream_t s = as_stream(stream);
  DevBuf<double>* state[] = {&E.u,   &E.v,   &E.w,   &E.ax,  &E.ay,  &E.az,  &E.ax0,
                             &E.ay0, &E.az0, &E.rhs, &E.p,   &E.p0,  &E.gpx, &E.gpy,
                             &E.gpz, &E.temp, &E.mf, &E.cval};
  const int ns = (int)(sizeof(state) / sizeof(state[0]));
  if (!restore) {
    if (E.snap.empty()) {
      for (int k = 0; k < ns; ++k) {
        DevBuf<double>* b = new DevBuf<double>();
        E.snap.push_back(b);
        GIPB_TRY(b->alloc(state[k]->n));
      }
      GIPB_TRY(E.snap_sc.alloc(1));
    }
    for (int k = 0; k < ns; ++k)
      GIPB_CUDA(cudaMemcpyAsync(E.snap[k]->p, state[k]->p, state[k]->n * 8, cudaMemcpyDeviceToDevice, s));
    GIPB_CUDA(cudaMemcpyAsync(E.snap_sc.p, E.sc.p, sizeof(DnsScalars), cudaMemcpyDeviceToDevice, s));
    E.snap_steps = E.steps_enqueued;
    return GIPB200_OK;
  }
  if (E.snap.empty() || E.snap_steps < 0) return fail(GIPB200_ERR_STATE, "no snapshot taken");
  for (int k = 0; k < ns; ++k)
    GIPB_CUDA(cudaMemcpyAsync(state[k]->p, E.snap[k]->p, state[k]->n * 8, cudaMemcpyDeviceToDevice, s));
  GIPB_CUDA(cudaMemcpyAsync(E.sc.p, E.snap_sc.p, sizeof(DnsScalars), cudaMemcpyDeviceToDevice, s));
  E.steps_enqueued = E.snap_steps;
  return GIPB200_OK;
}

int gipb200_dns_launch_count(gipb200_dns Dh, long long* count) {
  if (!Dh || !count) return fail(GIPB200_ERR_ARG, "null argument");
  *count = Dh->E.launches;
  return GIPB200_OK;
}

int gipb200_dns_kernel_time(gipb200_dns Dh, int kernel, int reps, void* stream, double* avg_ms,
                            double* bytes) {
  if (!Dh || !avg_ms || !bytes) return fail(GIPB200_ERR_ARG, "null argument");
  if (kernel == GIPB200_KERNEL_MIXED_UPDATE)
    return Dh->E.pcg.time_update(reps, as_stream(stream), avg_ms, bytes);
  if (kernel != GIPB200_KERNEL_PCG_SPMV_DOT && kernel != GIPB200_KERNEL_MIXED_SPMV_DOT)
    return fail(GIPB200_ERR_ARG, "unknown kernel id %d", kernel);
  return Dh->E.pcg.time_spmv(kernel == GIPB200_KERNEL_MIXED_SPMV_DOT, reps, as_stream(stream),
                             avg_ms, bytes);
}

int gipb200_dns_setup_profile(gipb200_dns Dh, double* h_seconds) {
  if (!Dh || !h_seconds) return fail(GIPB200_ERR_ARG, "null argument");
  for (int k = 0; k < 4; ++k) h_seconds[k] = Dh->E.setup_s[k];
  return GIPB200_OK;
}

int gipb200_dns_phase_bytes(gipb200_dns Dh, double* h_bytes) {
  if (!Dh || !h_bytes) return fail(GIPB200_ERR_ARG, "null argument");
  Dh->E.phase_bytes(h_bytes);
  return GIPB200_OK;
}

int gipb200_dns_vcycle_profile(gipb200_dns Dh, int reps, void* stream, int cap, int* n_kernels,
                               int* h_level, int* h_kind, double* h_ms, double* h_bytes) {
  if (!Dh) return fail(GIPB200_ERR_ARG, "null engine");
  return Dh->E.pcg.profile_vcycle(reps, as_stream(stream), cap, n_kernels, h_level, h_kind, h_ms,
                                  h_bytes);
}

int gipb200_dns_vcycle_forms(gipb200_dns Dh, int cap, int* n_kernels, int* h_form) {
  if (!Dh) return fail(GIPB200_ERR_ARG, "null engine");
  return Dh->E.pcg.vcycle_forms(cap, n_kernels, h_form);
}

int gipb200_dns_set_time(gipb200_dns Dh, double time, void* stream) {
  if (!Dh) return fail(GIPB200_ERR_ARG, "null engine");
  if (!std::isfinite(time)) return fail(GIPB200_ERR_ARG, "time must be finite");
  Dns& E = Dh->E;
  // ordered on `stream` after the work already queued there; the host value is read
  // before the call returns
  GIPB_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(E.sc.p) + offsetof(DnsScalars, time), &time,
                            sizeof(double), cudaMemcpyHostToDevice, as_stream(stream)));
  GIPB_CUDA(cudaStreamSynchronize(as_stream(stream)));
  return GIPB200_OK;
}

int gipb200_dns_scalars(gipb200_dns Dh, double* dt, double* sigma, double* time) {
  if (!Dh) return fail(GIPB200_ERR_ARG, "null engine");
  GIPB_CUDA(cudaDeviceSynchronize());
  DnsScalars S;
  GIPB_CUDA(cudaMemcpy(&S, Dh->E.sc.p, sizeof(S), cudaMemcpyDeviceToHost));
  if (dt) *dt = S.dt;
  if (sigma) *sigma = S.sigma;
  if (time) *time = S.time;
  return GIPB200_OK;
}

}  // extern "C"
