// Smoothed-aggregation AMG (setup on the host, FP32 V-cycle on the device).
//
// Setup per level (operator A, near-null vector z):
//   strength   |a_ij| > theta sqrt(|a_ii a_jj|), theta = 0 (with a positive threshold the
//              smoothed coarse operators lose their weak couplings to singleton aggregates
//              and fill in level after level)
//   aggregates greedy: (1) a node whose strong neighbours are all free starts an aggregate
//              with them; (2) a free node joins the aggregate of its strongest aggregated
//              neighbour; (3) what is left forms aggregates with its free neighbours
//   P0         tentative prolongator: P0[i, agg(i)] = z_i / |z restricted to agg(i)|
//   P          smoothed: (I - w D^-1 A) P0, w = 4 / (3 rho), rho = the Gershgorin bound of
//              D^-1 A; coarse near-null vector = the aggregate norms (so P z_c = z)
//   A_c        Galerkin: R A P with R = P^T, then sparsified: couplings below
//              kDrop sqrt(a_ii a_jj) lumped onto the diagonal along z (A_c z unchanged)
// The coarsest level (<= kCoarse unknowns) is inverted densely; for the pinned-Neumann
// inner system (A z = 0) the inverse is taken of A + sigma z z^T / |z|^2, which solves
// consistent right-hand sides exactly.
// V-cycle on level l (b -> x): x = D^-1 b (weighted Jacobi from zero), t = b - A x,
// b_{l+1} = R t, recurse, x += P x_{l+1}, result x + D^-1 (b - A x): the same smoother
// before and after, so the cycle is a symmetric operator.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <type_traits>

#include "amg.cuh"
#include "device.cuh"
#include "pcg.cuh"

namespace gipb200 {

namespace {

constexpr int kCoarse = 1024;    // largest level inverted densely
constexpr int kMaxLevels = 16;
constexpr double kTheta = 0.0;   // strength threshold: every nonzero coupling is strong
constexpr double kDrop = 0.02;   // coarse-operator drop threshold (sparsify); env GIPB200_AMG_DROP

struct HCsr {
  int nr = 0, nc = 0;
  std::vector<int> rp, ci;
  std::vector<double> v;
  long long nnz() const { return (long long)ci.size(); }
};

std::vector<double> diagonal(const HCsr& A) {
  std::vector<double> d((size_t)A.nr, 0.0);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < A.nr; ++i)
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] == i) d[i] += A.v[k];
  return d;
}

// Gershgorin bound of the spectral radius of D^-1 A.
double rho_bound(const HCsr& A, const std::vector<double>& d) {
  double rho = 0.0;
#pragma omp parallel for schedule(static) reduction(max : rho)
  for (int i = 0; i < A.nr; ++i) {
    double s = 0.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) s += std::fabs(A.v[k]);
    if (d[i] > 0.0) rho = std::max(rho, s / d[i]);
  }
  return rho > 0.0 ? rho : 1.0;
}

int aggregate(const HCsr& A, const std::vector<double>& d, std::vector<int>& agg) {
  const int n = A.nr;
  auto strong = [&](int i, int k) {
    const int j = A.ci[k];
    return j != i && A.v[k] != 0.0 && std::fabs(A.v[k]) > kTheta * std::sqrt(std::fabs(d[i] * d[j]));
  };
  agg.assign((size_t)n, -1);
  int na = 0;
  for (int i = 0; i < n; ++i) {  // phase 1
    if (agg[i] != -1) continue;
    bool free = true, any = false;
    for (int k = A.rp[i]; k < A.rp[i + 1] && free; ++k)
      if (strong(i, k)) {
        any = true;
        if (agg[A.ci[k]] != -1) free = false;
      }
    if (!free || !any) continue;
    agg[i] = na;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (strong(i, k)) agg[A.ci[k]] = na;
    ++na;
  }
  const std::vector<int> first = agg;
  for (int i = 0; i < n; ++i) {  // phase 2
    if (first[i] != -1) continue;
    int best = -1;
    double bw = 0.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (strong(i, k) && first[A.ci[k]] >= 0 && std::fabs(A.v[k]) > bw) {
        bw = std::fabs(A.v[k]);
        best = first[A.ci[k]];
      }
    if (best >= 0) agg[i] = best;
  }
  for (int i = 0; i < n; ++i) {  // phase 3
    if (agg[i] != -1) continue;
    agg[i] = na;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (strong(i, k) && agg[A.ci[k]] == -1) agg[A.ci[k]] = na;
    ++na;
  }
  return na;
}

// Row-wise product C = A B (Gustavson), rows in the order their columns first appear.
int spgemm(const HCsr& A, const HCsr& B, HCsr& C) {
  C.nr = A.nr;
  C.nc = B.nc;
  C.rp.assign((size_t)A.nr + 1, 0);
#pragma omp parallel
  {
    std::vector<int> mark((size_t)B.nc, -1);
#pragma omp for schedule(dynamic, 1024)
    for (int i = 0; i < A.nr; ++i) {
      int c = 0;
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        const int j = A.ci[k];
        for (int q = B.rp[j]; q < B.rp[j + 1]; ++q)
          if (mark[B.ci[q]] != i) {
            mark[B.ci[q]] = i;
            ++c;
          }
      }
      C.rp[i + 1] = c;
    }
  }
  long long total = 0;
  for (int i = 0; i < A.nr; ++i) total += C.rp[i + 1];
  if (total > 0x7fffffffLL)
    return fail(GIPB200_ERR_ARG, "AMG: a Galerkin product has %lld nonzeros (more than 2^31)", total);
  for (int i = 0; i < A.nr; ++i) C.rp[i + 1] += C.rp[i];
  C.ci.resize((size_t)C.rp[A.nr]);
  C.v.resize((size_t)C.rp[A.nr]);
#pragma omp parallel
  {
    std::vector<int> where((size_t)B.nc, -1);
#pragma omp for schedule(dynamic, 1024)
    for (int i = 0; i < A.nr; ++i) {
      int o = C.rp[i];
      const int o0 = o;
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
        const int j = A.ci[k];
        const double a = A.v[k];
        for (int q = B.rp[j]; q < B.rp[j + 1]; ++q) {
          const int c = B.ci[q];
          if (where[c] < o0) {
            where[c] = o;
            C.ci[o] = c;
            C.v[o] = a * B.v[q];
            ++o;
          } else {
            C.v[where[c]] += a * B.v[q];
          }
        }
      }
    }
  }
  return GIPB200_OK;
}

HCsr transpose(const HCsr& A) {
  HCsr T;
  T.nr = A.nc;
  T.nc = A.nr;
  T.rp.assign((size_t)A.nc + 1, 0);
  for (int c : A.ci) T.rp[c + 1]++;
  for (int i = 0; i < A.nc; ++i) T.rp[i + 1] += T.rp[i];
  T.ci.resize(A.ci.size());
  T.v.resize(A.v.size());
  std::vector<int> next(T.rp.begin(), T.rp.end() - 1);
  for (int i = 0; i < A.nr; ++i)
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      const int o = next[A.ci[k]]++;
      T.ci[o] = i;
      T.v[o] = A.v[k];
    }
  return T;
}

// Sparsified coarse operator (non-Galerkin): off-diagonal couplings with
// |a_ij| < theta sqrt(a_ii a_jj) are dropped and lumped onto the diagonal weighted by the
// near-null vector, a_ii += a_ij z_j / z_i, so that A z is unchanged.  The values are made
// exactly symmetric first ((A + A^T) / 2 on the common pattern), so the decision and the
// result are symmetric; a row or column whose z entry is 0 keeps its couplings, and so
// does a row whose diagonal would lose more than half.  Returns false, leaving A as it
// was, when A's pattern is not symmetric or a diagonal is missing or not positive.
bool sparsify(HCsr& A, const std::vector<double>& z, double theta) {
  const int n = A.nr;
  if (A.nc != n) return false;
  HCsr S = A;
#pragma omp parallel
  {
    std::vector<std::pair<int, double>> e;
#pragma omp for schedule(static)
    for (int i = 0; i < n; ++i) {  // columns in increasing order, as the transpose has them
      e.clear();
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) e.emplace_back(A.ci[k], A.v[k]);
      std::sort(e.begin(), e.end(),
                [](const std::pair<int, double>& a, const std::pair<int, double>& b) {
                  return a.first < b.first;
                });
      for (size_t q = 0; q < e.size(); ++q) {
        S.ci[A.rp[i] + q] = e[q].first;
        S.v[A.rp[i] + q] = e[q].second;
      }
    }
  }
  const HCsr T = transpose(S);
  if (T.rp != S.rp || T.ci != S.ci) return false;
  std::vector<double> d((size_t)n, 0.0);
  std::vector<int> dk((size_t)n, -1);
  for (int i = 0; i < n; ++i)
    for (int k = S.rp[i]; k < S.rp[i + 1]; ++k) {
      S.v[k] = 0.5 * (S.v[k] + T.v[k]);
      if (S.ci[k] == i) dk[i] = k;
    }
  for (int i = 0; i < n; ++i) {
    if (dk[i] < 0 || !(S.v[dk[i]] > 0.0)) return false;
    d[i] = S.v[dk[i]];
  }
  // A row whose diagonal would lose more than half to the lumping keeps its couplings,
  // and so do its partners' entries for it (a coupling goes only when both rows let it go)
  std::vector<char> keep_row((size_t)n, 0);
  auto droppable = [&](int i, int j, double a) {
    return j != i && z[i] != 0.0 && z[j] != 0.0 && !keep_row[i] && !keep_row[j] &&
           std::fabs(a) < theta * std::sqrt(d[i] * d[j]);
  };
  auto lumped = [&](int i) {
    double lump = 0.0;
    for (int k = S.rp[i]; k < S.rp[i + 1]; ++k)
      if (droppable(i, S.ci[k], S.v[k])) lump += S.v[k] * z[S.ci[k]] / z[i];
    return lump;
  };
  for (int i = 0; i < n; ++i)
    if (!(d[i] + lumped(i) > 0.5 * d[i])) keep_row[i] = 1;
  for (int i = 0; i < n; ++i)  // fewer drops can move a lump either way: check again
    if (!keep_row[i] && !(d[i] + lumped(i) > 0.5 * d[i])) return false;
  HCsr O;
  O.nr = O.nc = n;
  O.rp.assign((size_t)n + 1, 0);
  O.ci.reserve(S.ci.size());
  O.v.reserve(S.v.size());
  for (int i = 0; i < n; ++i) {
    double lump = 0.0;
    int diag_at = -1;
    for (int k = S.rp[i]; k < S.rp[i + 1]; ++k) {
      const int j = S.ci[k];
      const double a = S.v[k];
      if (droppable(i, j, a)) {
        lump += a * z[j] / z[i];
        continue;
      }
      if (j == i) diag_at = (int)O.ci.size();
      O.ci.push_back(j);
      O.v.push_back(a);
    }
    O.v[diag_at] += lump;
    O.rp[i + 1] = (int)O.ci.size();
  }
  A = std::move(O);
  return true;
}

// Smoothed prolongator (I - w D^-1 A) P0 with P0[i, agg(i)] = p0[i].
HCsr smoothed_prolongator(const HCsr& A, const std::vector<double>& d, const std::vector<int>& agg,
                          const std::vector<double>& p0, int na, double w) {
  HCsr P;
  P.nr = A.nr;
  P.nc = na;
  P.rp.assign((size_t)A.nr + 1, 0);
  auto row = [&](int i, std::vector<std::pair<int, double>>& e) {
    e.clear();
    e.emplace_back(agg[i], p0[i]);
    const double s = d[i] > 0.0 ? w / d[i] : 0.0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      const int j = A.ci[k];
      const double val = -s * A.v[k] * p0[j];
      bool found = false;
      for (auto& q : e)
        if (q.first == agg[j]) {
          q.second += val;
          found = true;
          break;
        }
      if (!found) e.emplace_back(agg[j], val);
    }
  };
#pragma omp parallel
  {
    std::vector<std::pair<int, double>> e;
#pragma omp for schedule(static)
    for (int i = 0; i < A.nr; ++i) {
      row(i, e);
      P.rp[i + 1] = (int)e.size();
    }
  }
  for (int i = 0; i < A.nr; ++i) P.rp[i + 1] += P.rp[i];
  P.ci.resize((size_t)P.rp[A.nr]);
  P.v.resize((size_t)P.rp[A.nr]);
#pragma omp parallel
  {
    std::vector<std::pair<int, double>> e;
#pragma omp for schedule(static)
    for (int i = 0; i < A.nr; ++i) {
      row(i, e);
      int o = P.rp[i];
      for (auto& q : e) {
        P.ci[o] = q.first;
        P.v[o] = q.second;
        ++o;
      }
    }
  }
  return P;
}

// Dense inverse of the SPD matrix M (m x m, row-major) by Cholesky; false if not SPD.
bool dense_inverse(int m, std::vector<double>& M, std::vector<double>& inv) {
  std::vector<double> Lc((size_t)m * m, 0.0);
  for (int j = 0; j < m; ++j) {
    double s = M[(size_t)j * m + j];
    for (int k = 0; k < j; ++k) s -= Lc[(size_t)j * m + k] * Lc[(size_t)j * m + k];
    if (!(s > 0.0)) return false;
    const double ljj = std::sqrt(s);
    Lc[(size_t)j * m + j] = ljj;
    for (int i = j + 1; i < m; ++i) {
      double t = M[(size_t)i * m + j];
      for (int k = 0; k < j; ++k) t -= Lc[(size_t)i * m + k] * Lc[(size_t)j * m + k];
      Lc[(size_t)i * m + j] = t / ljj;
    }
  }
  inv.assign((size_t)m * m, 0.0);
  std::vector<double> y((size_t)m);
  for (int c = 0; c < m; ++c) {  // column c of the inverse: L L^T x = e_c
    for (int i = 0; i < m; ++i) {
      double t = (i == c) ? 1.0 : 0.0;
      for (int k = 0; k < i; ++k) t -= Lc[(size_t)i * m + k] * y[k];
      y[i] = t / Lc[(size_t)i * m + i];
    }
    for (int i = m - 1; i >= 0; --i) {
      double t = y[i];
      for (int k = i + 1; k < m; ++k) t -= Lc[(size_t)k * m + i] * inv[(size_t)k * m + c];
      inv[(size_t)i * m + c] = t / Lc[(size_t)i * m + i];
    }
  }
  return true;
}

// compact: a long-row (CSR) operator whose rows each span at most 65536 columns is stored
// with 16-bit offsets from each row's smallest column (the FP32 cycle); half: FP16 values.
template <typename T>
int upload(const HCsr& A, SellT<T>* S, cudaStream_t s, bool half = false, bool compact = false,
           bool transfer = false) {
  S->half = half;
  GIPB_TRY(validate_csr(A.nr, A.nc, (int)A.nnz(), A.rp.data(), A.ci.data(), A.nc, "AMG operator"));
  S->nrows = A.nr;
  S->ncols = A.nc;
  S->nnz = A.nnz();
  S->nslices = (A.nr + 31) / 32;
  const double avg = (double)A.nnz() / std::max(A.nr, 1);
  // Rows of at least 32 entries on average are CSR, shorter ones sliced (a lane per row,
  // eight slots in flight): on the 256^3 cavity the level-1 operator (21 per row) and the
  // level-0 restriction (29) ran 72 and 124 us sliced against 91 and 128 us in CSR.
  // GIPB200_AMG_CSR_ROWS overrides the threshold.
  const char* csr_env = getenv("GIPB200_AMG_CSR_ROWS");
  const double csr_rows = csr_env ? atof(csr_env) : 32.0;
  if (avg >= csr_rows) {  // long rows: CSR, 4 to 32 threads per row
    // FP32 cycle's transfer operators (FP16 values): as few threads per row as cover its
    // entries in one pass (4 threads x 8 entries, 8 x 4, ...), so that a warp works on more
    // rows per dependent round trip (restriction of the 256^3 cavity: 128 against 153 us);
    // coarse operators (FP32 values, where the narrow form measured 107 against 90 us),
    // the FP64 cycle and GIPB200_AMG_WIDE_ROWS=1: 8 to 32 threads per row
    const bool narrow = std::is_same<T, float>::value && transfer &&
                        !getenv("GIPB200_AMG_WIDE_ROWS");
    S->lanes = narrow ? (avg < 32.0 ? 4 : avg < 64.0 ? 8 : avg < 128.0 ? 16 : 32)
                      : (avg >= 48.0 ? 32 : avg >= 24.0 ? 16 : 8);
    GIPB_TRY(S->rp.upload(A.rp.data(), A.rp.size(), s));
    bool fits = compact && std::is_same<T, float>::value;
    std::vector<int> cb((size_t)std::max(A.nr, 1), 0);
    for (int r = 0; r < A.nr && fits; ++r) {
      int lo = A.nc, hi = -1;
      for (int k = A.rp[r]; k < A.rp[r + 1]; ++k) lo = std::min(lo, A.ci[k]), hi = std::max(hi, A.ci[k]);
      cb[r] = hi >= 0 ? lo : 0;
      fits = hi < 0 || hi - lo <= 65535;
    }
    if (fits) {
      S->short_cols = true;
      std::vector<unsigned short> dc(std::max<size_t>(A.ci.size(), 1), 0);
      for (int r = 0; r < A.nr; ++r)
        for (int k = A.rp[r]; k < A.rp[r + 1]; ++k) dc[k] = (unsigned short)(A.ci[k] - cb[r]);
      GIPB_TRY(S->dcol.upload(dc.data(), dc.size(), s));
      GIPB_TRY(S->cbase.upload(cb.data(), cb.size(), s));
    } else {
      GIPB_TRY(S->col.upload(A.ci.data(), std::max<size_t>(A.ci.size(), 1), s));
    }
    if (half) {
      std::vector<__half> hv(std::max<size_t>(A.v.size(), 1), __float2half_rn(0.0f));
      for (size_t k = 0; k < A.v.size(); ++k) hv[k] = __float2half_rn((float)A.v[k]);
      GIPB_TRY(S->hval.upload(hv.data(), hv.size(), s));
    } else {
      std::vector<T> val(std::max<size_t>(A.v.size(), 1), T(0));
      for (size_t k = 0; k < A.v.size(); ++k) val[k] = (T)A.v[k];
      GIPB_TRY(S->val.upload(val.data(), val.size(), s));
    }
    GIPB_CUDA(cudaStreamSynchronize(s));
    return GIPB200_OK;
  }
  // The FP32 cycle's sliced transfer operators with rows of two or more 8-slot batches on
  // average run software-pipelined (k_amg_spmv_pf at 4 CTAs per SM): the 256^3 cavity's
  // level-0 restriction (29 entries per row) 116.5 against 123.1 us.  Rows of one batch
  // lose more to the halved occupancy than the overlap gains (its level-0 prolongation:
  // 209.5 against 143.2 us), and the level-1 operator (21 per row) gained nothing (73.2
  // against 71.9 us).  GIPB200_AMG_PIPE=0: never; =1: every sliced FP32 operator (read per
  // call).
  {
    const char* pe = getenv("GIPB200_AMG_PIPE");
    const bool f32 = std::is_same<T, float>::value;
    S->pipe = f32 && (pe ? atoi(pe) == 1 : transfer && avg >= 16.0) ? 1 : 0;
  }
  std::vector<long long> sptr((size_t)S->nslices + 1, 0);
  for (int sl = 0; sl < S->nslices; ++sl) {
    int len = 0;
    for (int r = sl * 32; r < std::min(A.nr, sl * 32 + 32); ++r) len = std::max(len, A.rp[r + 1] - A.rp[r]);
    sptr[sl + 1] = sptr[sl] + 32LL * len;
  }
  S->nslots = sptr[S->nslices];
  if (S->nslots > 0x7fffffffLL) return fail(GIPB200_ERR_ARG, "AMG operator too large");
  // compact: 16-bit slot columns from a per-row base (0xffff marks padding) when every
  // row spans at most 65535 columns
  bool fits16 = compact && std::is_same<T, float>::value;
  std::vector<int> cb(fits16 ? (size_t)std::max(A.nr, 1) : 0, 0);
  for (int r = 0; r < A.nr && fits16; ++r) {
    int lo = A.nc, hi = -1;
    for (int k = A.rp[r]; k < A.rp[r + 1]; ++k) lo = std::min(lo, A.ci[k]), hi = std::max(hi, A.ci[k]);
    cb[r] = hi >= 0 ? lo : 0;
    fits16 = hi < 0 || hi - lo < 65535;
  }
  std::vector<int> col(fits16 ? 0 : (size_t)std::max<long long>(S->nslots, 1), -1);
  std::vector<unsigned short> col16(fits16 ? (size_t)std::max<long long>(S->nslots, 1) : 0,
                                    (unsigned short)0xffff);
  std::vector<T> val((size_t)std::max<long long>(S->nslots, 1), T(0));
#pragma omp parallel for schedule(static)
  for (int r = 0; r < A.nr; ++r) {
    const int sl = r >> 5, lane = r & 31;
    for (int k = A.rp[r]; k < A.rp[r + 1]; ++k) {
      const long long slot = sptr[sl] + 32LL * (k - A.rp[r]) + lane;
      if (fits16)
        col16[slot] = (unsigned short)(A.ci[k] - cb[r]);
      else
        col[slot] = A.ci[k];
      val[slot] = (T)A.v[k];
    }
  }
  GIPB_TRY(S->sptr.upload(sptr.data(), sptr.size(), s));
  if (fits16) {
    S->short_cols = true;
    GIPB_TRY(S->dcol.upload(col16.data(), col16.size(), s));
    GIPB_TRY(S->cbase.upload(cb.data(), cb.size(), s));
  } else {
    GIPB_TRY(S->col.upload(col.data(), col.size(), s));
  }
  if (half) {
    std::vector<__half> hv(val.size());
    for (size_t k = 0; k < val.size(); ++k) hv[k] = __float2half_rn((float)val[k]);
    GIPB_TRY(S->hval.upload(hv.data(), hv.size(), s));
  } else {
    GIPB_TRY(S->val.upload(val.data(), val.size(), s));
  }
  GIPB_CUDA(cudaStreamSynchronize(s));  // host staging goes out of scope
  return GIPB200_OK;
}

// ------------------------------------------------------------------ V-cycle kernels
// All of them count their launch and return at once when the solve has finished.
__device__ __forceinline__ bool amg_enter(PcgScalars* S) {
  dep_begin();
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&S->kernels, 1);
  return S->done != 0;
}

__device__ __forceinline__ float fmat(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmat(double a, double b, double c) { return fma(a, b, c); }
// a * b rounded on its own (the Jacobi start x = D^-1 b, formed where it is gathered)
__device__ __forceinline__ float mulr(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mulr(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float addr(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double addr(double a, double b) { return __dadd_rn(a, b); }

// Stored operator values to the arithmetic type (FP16-stored transfer operators).
__device__ __forceinline__ float to_arith(__half v) { return __half2float(v); }
__device__ __forceinline__ float to_arith(float v) { return v; }
__device__ __forceinline__ double to_arith(double v) { return v; }

// One row of a sliced operator whose slice starts at slot `base` and has `len` slots,
// summed slot by slot (padding: column -1, skipped).
// XS: the gathered vector is xs * x elementwise, each product rounded on its own (the
// same value a separate x = xs * x pass would store).  A compile-time choice: a run-time
// test in the gather loop measured 8-21% slower on the kernels that never scale.
template <typename T, int CH, typename V = T, bool XS = false>
__device__ __forceinline__ T amg_row_at(const SellView<V>& A, const T* __restrict__ x,
                                        long long base, int len, int lane,
                                        const T* __restrict__ xs = nullptr) {
  const int* cp = A.col + base + lane;
  const V* vp = A.val + base + lane;
  T sum = T(0);
  for (int j0 = 0; j0 < len; j0 += CH) {
    int c[CH];
    T v[CH];
#pragma unroll
    for (int t = 0; t < CH; ++t) {
      c[t] = (j0 + t < len) ? ld_stream(cp + (size_t)(j0 + t) * 32) : -1;
      v[t] = (j0 + t < len) ? (T)to_arith(ld_stream(vp + (size_t)(j0 + t) * 32)) : T(0);
    }
    T xv[CH];
#pragma unroll
    for (int t = 0; t < CH; ++t)
      xv[t] = (c[t] >= 0) ? (XS ? mulr(__ldg(xs + c[t]), __ldg(x + c[t])) : __ldg(x + c[t])) : T(0);
#pragma unroll
    for (int t = 0; t < CH; ++t) sum = fmat(xv[t], v[t], sum);
  }
  return sum;
}

// The same row with 16-bit slot columns: column = cb + d (cb the row's base column), the
// offset 0xffff marking padding.
template <typename T, int CH, typename V, bool XS>
__device__ __forceinline__ T amg_row_at16(const unsigned short* __restrict__ dcol,
                                          const V* __restrict__ val, const T* __restrict__ x,
                                          long long base, int len, int lane, int cb,
                                          const T* __restrict__ xs) {
  const unsigned short* cp = dcol + base + lane;
  const V* vp = val + base + lane;
  T sum = T(0);
  for (int j0 = 0; j0 < len; j0 += CH) {
    int c[CH];
    T v[CH];
#pragma unroll
    for (int t = 0; t < CH; ++t) {
      const unsigned d = (j0 + t < len) ? (unsigned)ld_stream(cp + (size_t)(j0 + t) * 32) : 0xffffu;
      c[t] = (d == 0xffffu) ? -1 : cb + (int)d;
      v[t] = (j0 + t < len) ? (T)to_arith(ld_stream(vp + (size_t)(j0 + t) * 32)) : T(0);
    }
    T xv[CH];
#pragma unroll
    for (int t = 0; t < CH; ++t)
      xv[t] = (c[t] >= 0) ? (XS ? mulr(__ldg(xs + c[t]), __ldg(x + c[t])) : __ldg(x + c[t])) : T(0);
#pragma unroll
    for (int t = 0; t < CH; ++t) sum = fmat(xv[t], v[t], sum);
  }
  return sum;
}

template <typename T, int CH, typename V = T>
__device__ __forceinline__ T amg_row(const SellView<V>& A, const T* __restrict__ x, int s, int lane) {
  const long long base = A.sptr[s];
  return amg_row_at<T, CH, V>(A, x, base, (int)((A.sptr[s + 1] - base) >> 5), lane);
}

// x = dinv b
template <typename T>
__global__ void __launch_bounds__(256) k_amg_jacobi0(int n, const T* __restrict__ dinv,
                                                     const T* __restrict__ b, T* __restrict__ x,
                                                     PcgScalars* S) {
  if (amg_enter(S)) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = dinv[i] * b[i];
}

enum { kResid = 0, kPlain = 1, kAdd = 2, kSmooth = 3, kScaleAdd = 4, kDiagAdd = 5 };
// kDiagAdd: y = D^-1 b + A x (a coarse level's prolongation onto its Jacobi start, which
// the cycle no longer forms: rounded as the two separate steps round it)
// kResid: y = b - A x;  kPlain: y = A x;  kAdd: y += A x;  kSmooth: y = x + dinv (b - A x);
// kScaleAdd: y = w b + A x (the level-0 prolongation onto x0 = w r, never formed)
// C16: 16-bit slot columns (dcol, offsets from the row's base column cbase[row]).
// The rows of slices gw, gw + nw, ... (warp gw of nw).
template <typename T, int MODE, typename V = T, bool C16 = false, bool XS = false>
__device__ __forceinline__ void sell_rows(const SellView<V>& A, const T* __restrict__ x,
                                          const T* __restrict__ b, const T* __restrict__ dinv,
                                          T* __restrict__ y, T w, const int* __restrict__ yperm,
                                          const T* __restrict__ xs,
                                          const unsigned short* __restrict__ dcol,
                                          const int* __restrict__ cbase, int gw, int nw) {
  // slots a lane loads before gathering: 8 in FP32 (a prolongation row's slots in one
  // round trip), 4 in FP64
  constexpr int kCh = sizeof(T) == 4 ? 8 : 4;
  const int lane = threadIdx.x & 31;
  for (int s = gw; s < A.nslices; s += nw) {
    const long long b0 = A.sptr[s];
    const int len = (int)((A.sptr[s + 1] - b0) >> 5);
    const int i = s * 32 + lane;
    T sum;
    if (C16) {
      const int cb = (i < A.nrows) ? __ldg(cbase + i) : 0;
      sum = amg_row_at16<T, kCh, V, XS>(dcol, A.val, x, b0, len, lane, cb, xs);
    } else {
      sum = amg_row_at<T, kCh, V, XS>(A, x, b0, len, lane, xs);
    }
    if (i < A.nrows) {
      // kResid: level 0 may write its residual in aggregate order (yperm)
      if (MODE == kResid) y[yperm ? yperm[i] : i] = (w == T(1)) ? b[i] - sum : fmat(-w, sum, b[i]);
      else if (MODE == kPlain) y[i] = sum;
      else if (MODE == kAdd) y[i] += sum;
      else if (MODE == kScaleAdd) y[i] = fmat(w, b[i], sum);
      else if (MODE == kDiagAdd) y[i] = addr(mulr(dinv[i], b[i]), sum);
      else y[i] = fmat(dinv[i], b[i] - sum, x[i]);
    }
  }
}

template <typename T, int MODE, typename V = T, bool C16 = false, bool XS = false>
__global__ void __launch_bounds__(256, sizeof(T) == 8 ? 6 : 8) k_amg_spmv(SellView<V> A, const T* __restrict__ x,
                                                     const T* __restrict__ b,
                                                     const T* __restrict__ dinv,
                                                     T* __restrict__ y, PcgScalars* S, T w,
                                                     const int* __restrict__ yperm,
                                                     const T* __restrict__ xs,
                                                     const unsigned short* __restrict__ dcol,
                                                     const int* __restrict__ cbase) {
  if (amg_enter(S)) return;
  sell_rows<T, MODE, V, C16, XS>(A, x, b, dinv, y, w, yperm, xs, dcol, cbase,
                                 (blockIdx.x * blockDim.x + threadIdx.x) >> 5,
                                 (gridDim.x * blockDim.x) >> 5);
}

// The sliced products software-pipelined over each warp's sequence of 8-slot batches: the
// loads of the next batch (in this slice, or in the warp's next slice, whose slot range is
// read one slice ahead) are issued before the gathers of the current one, and a slice's
// row operands (b, dinv, x, y, yperm) before its first gathers, so a warp always has
// operator words in flight.  The same fused multiply-adds in the same order as sell_rows
// (batches of 8 slots from slot 0), so the results are identical.  OCC: resident CTAs per
// SM it is compiled for (the second batch in registers lowers the CTAs that fit: 64
// registers a thread at 4, no spills).
template <typename V>
__device__ __forceinline__ void sell_batch(const SellView<V>& A, long long base, int len, int j0,
                                           int lane, int (&c)[8], V (&v)[8]) {
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    const bool in = j0 + t < len;
    c[t] = in ? ld_stream(A.col + base + 32LL * (j0 + t) + lane) : -1;
    v[t] = in ? ld_stream(A.val + base + 32LL * (j0 + t) + lane) : V(0.0f);
  }
}

template <typename T, int MODE, typename V, bool XS, int OCC>
__global__ void __launch_bounds__(256, OCC) k_amg_spmv_pf(SellView<V> A, const T* __restrict__ x,
                                                          const T* __restrict__ b,
                                                          const T* __restrict__ dinv,
                                                          T* __restrict__ y, PcgScalars* S, T w,
                                                          const int* __restrict__ yperm,
                                                          const T* __restrict__ xs) {
  if (amg_enter(S)) return;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (s >= A.nslices) return;
  long long base, nbase = 0;
  int len, nlen = 0;
  slice_range(A, s, base, len);
  int sn = s + nw;
  if (sn < A.nslices) slice_range(A, sn, nbase, nlen);
  // row operands of slice s (the writes below need them; loaded ahead of the gathers)
  T rb = T(0), rd = T(0), rx = T(0);
  int ri = 0;
  auto row_ops = [&](int sl) {
    const int i = sl * 32 + lane;
    if (i < A.nrows) {
      if (MODE != kPlain && MODE != kAdd) rb = b[i];
      if (MODE == kAdd) rb = y[i];
      if (MODE == kDiagAdd || MODE == kSmooth) rd = dinv[i];
      if (MODE == kSmooth) rx = x[i];
      if (MODE == kResid) ri = yperm ? yperm[i] : i;
    }
  };
  row_ops(s);
  int c[8];
  V v[8];
  sell_batch(A, base, len, 0, lane, c, v);
  int j0 = 0;
  T sum = T(0);
  while (true) {
    const bool last = j0 + 8 >= len;
    const bool more = !last || sn < A.nslices;
    int cn[8];
    V vn[8];
    if (more) {
      sell_batch(A, last ? nbase : base, last ? nlen : len, last ? 0 : j0 + 8, lane, cn, vn);
    } else {
#pragma unroll
      for (int t = 0; t < 8; ++t) cn[t] = -1, vn[t] = V(0.0f);
    }
    T xv[8];
#pragma unroll
    for (int t = 0; t < 8; ++t)
      xv[t] = (c[t] >= 0) ? (XS ? mulr(__ldg(xs + c[t]), __ldg(x + c[t])) : __ldg(x + c[t])) : T(0);
#pragma unroll
    for (int t = 0; t < 8; ++t) sum = fmat(xv[t], (T)to_arith(v[t]), sum);
    if (last) {
      const int i = s * 32 + lane;
      if (i < A.nrows) {
        if (MODE == kResid) y[ri] = (w == T(1)) ? rb - sum : fmat(-w, sum, rb);
        else if (MODE == kPlain) y[i] = sum;
        else if (MODE == kAdd) y[i] = rb + sum;
        else if (MODE == kScaleAdd) y[i] = fmat(w, rb, sum);
        else if (MODE == kDiagAdd) y[i] = addr(mulr(rd, rb), sum);
        else y[i] = fmat(rd, rb - sum, rx);
      }
      if (!more) break;
      s = sn;
      base = nbase;
      len = nlen;
      sn = s + nw;
      if (sn < A.nslices) slice_range(A, sn, nbase, nlen);
      row_ops(s);
      sum = T(0);
      j0 = 0;
    } else {
      j0 += 8;
    }
#pragma unroll
    for (int t = 0; t < 8; ++t) c[t] = cn[t], v[t] = vn[t];
  }
}

// The same products from the CSR form: LANES threads per row, each summing a strided part
// of the row, combined by a fixed shuffle tree (deterministic).  The row loop is uniform
// across the warp (32 / LANES rows per warp per pass), so every lane takes part in the
// shuffles.  Software-pipelined: the next pass's row bounds are loaded while this pass's
// gathers are in flight, and each lane loads up to U of its entries (8 with 4 threads per
// row, else 4) before gathering them, so a pass costs two dependent memory round trips
// instead of two per entry plus one for the bounds.  Each lane still adds its entries in
// increasing order.
template <typename T, int MODE, int LANES, typename V = T, typename CI = int, bool XS = false>
__device__ __forceinline__ void csr_rows(int nrows, const int* __restrict__ rp,
                                         const CI* __restrict__ col, const V* __restrict__ val,
                                         const T* __restrict__ x, const T* __restrict__ b,
                                         const T* __restrict__ dinv, T* __restrict__ y, T w,
                                         const T* __restrict__ xs, const int* __restrict__ cbase,
                                         int gw, int nw) {
  constexpr int RPW = 32 / LANES;        // rows per warp per pass
  constexpr int U = LANES <= 4 ? 8 : 4;  // entries a lane loads before their gathers
  const int lane = threadIdx.x & 31, sub = lane % LANES;
  constexpr bool kShort = sizeof(CI) == 2;  // 16-bit offsets from each row's base column
  int r0 = gw * RPW;
  int kb = 0, ke = 0, cb = 0;
  {
    const int i = r0 + lane / LANES;
    if (i < nrows) {
      kb = __ldg(rp + i), ke = __ldg(rp + i + 1);
      if (kShort) cb = __ldg(cbase + i);
    }
  }
  for (; r0 < nrows; r0 += nw * RPW) {
    const int i = r0 + lane / LANES;
    int kbn = 0, ken = 0, cbn = 0;  // the next pass's row, loaded ahead
    const int in = i + nw * RPW;
    if (in < nrows) {
      kbn = __ldg(rp + in), ken = __ldg(rp + in + 1);
      if (kShort) cbn = __ldg(cbase + in);
    }
    T sum = T(0);
    for (int k0 = kb + sub; k0 < ke; k0 += U * LANES) {
      int c[U];
      V v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = k0 + u * LANES;
        c[u] = (k < ke) ? (kShort ? cb + (int)ld_stream(col + k) : (int)ld_stream(col + k)) : -1;
        v[u] = (k < ke) ? ld_stream(val + k) : V(0);
      }
      T xv[U];
#pragma unroll
      for (int u = 0; u < U; ++u)
        xv[u] = (c[u] >= 0) ? (XS ? mulr(__ldg(xs + c[u]), __ldg(x + c[u])) : __ldg(x + c[u]))
                            : T(0);
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (c[u] >= 0) sum = fmat((T)to_arith(v[u]), xv[u], sum);
    }
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o, LANES);
    if (i < nrows && sub == 0) {
      if (MODE == kResid) y[i] = (w == T(1)) ? b[i] - sum : fmat(-w, sum, b[i]);
      else if (MODE == kPlain) y[i] = sum;
      else if (MODE == kAdd) y[i] += sum;
      else if (MODE == kScaleAdd) y[i] = fmat(w, b[i], sum);
      else if (MODE == kDiagAdd) y[i] = addr(mulr(dinv[i], b[i]), sum);
      else y[i] = fmat(dinv[i], b[i] - sum, x[i]);
    }
    kb = kbn;
    ke = ken;
    cb = cbn;
  }
}

template <typename T, int MODE, int LANES, typename V = T, typename CI = int, bool XS = false>
__global__ void __launch_bounds__(256) k_amg_csr(int nrows, const int* __restrict__ rp,
                                                 const CI* __restrict__ col,
                                                 const V* __restrict__ val, const T* __restrict__ x,
                                                 const T* __restrict__ b,
                                                 const T* __restrict__ dinv, T* __restrict__ y,
                                                 PcgScalars* S, T w, const T* __restrict__ xs,
                                                 const int* __restrict__ cbase) {
  if (amg_enter(S)) return;
  csr_rows<T, MODE, LANES, V, CI, XS>(nrows, rp, col, val, x, b, dinv, y, w, xs, cbase,
                                      (blockIdx.x * blockDim.x + threadIdx.x) >> 5,
                                      (gridDim.x * blockDim.x) >> 5);
}

int vec_blocks(int n);

// y (mode) A x for an AMG operator in either form; XS: the gathered x scaled by xs.
template <typename T, int MODE, typename V, bool XS>
void amg_mv_vx(const SellT<T>& M, SellView<V> view, const V* v, const T* x, const T* b,
               const T* dinv, T* y, PcgScalars* S, cudaStream_t s, T w, const T* xs) {
  if (M.lanes == 0) {
    if constexpr (std::is_same<T, float>::value) {
      if (M.pipe > 0 && !M.short_cols) {
        constexpr int kOcc = 4;
        DeviceInfo di;
        const int nsm = device_info(&di) == GIPB200_OK ? di.nsm : 1;
        const int nb = std::min(vec_blocks(M.nslices * 32), nsm * kOcc);
        launch_dep(k_amg_spmv_pf<T, MODE, V, XS, kOcc>, nb, 256, s, view, x, b, dinv, y, S, w,
                   (const int*)nullptr, xs);
        return;
      }
    }
    if (M.short_cols)
      launch_dep(k_amg_spmv<T, MODE, V, true, XS>, vec_blocks(M.nslices * 32), 256, s, view, x,
                 b, dinv, y, S, w, (const int*)nullptr, xs, (const unsigned short*)M.dcol.p,
                 (const int*)M.cbase.p);
    else
      launch_dep(k_amg_spmv<T, MODE, V, false, XS>, vec_blocks(M.nslices * 32), 256, s, view, x,
                 b, dinv, y, S, w, (const int*)nullptr, xs, (const unsigned short*)nullptr,
                 (const int*)nullptr);
    return;
  }
  const int nb = vec_blocks((int)std::min<long long>((long long)M.nrows * M.lanes, 1LL << 30));
  const int* rp = M.rp.p;
#define GIPB_CSR(L, CI, COLS)                                                                \
  launch_dep(k_amg_csr<T, MODE, L, V, CI, XS>, nb, 256, s, M.nrows, rp, (const CI*)COLS, v, x, \
             b, dinv, y, S, w, xs, (const int*)M.cbase.p)
  if (M.short_cols) {
    if (M.lanes == 32) GIPB_CSR(32, unsigned short, M.dcol.p);
    else if (M.lanes == 16) GIPB_CSR(16, unsigned short, M.dcol.p);
    else if (M.lanes == 8) GIPB_CSR(8, unsigned short, M.dcol.p);
    else GIPB_CSR(4, unsigned short, M.dcol.p);
  } else {
    if (M.lanes == 32) GIPB_CSR(32, int, M.col.p);
    else if (M.lanes == 16) GIPB_CSR(16, int, M.col.p);
    else if (M.lanes == 8) GIPB_CSR(8, int, M.col.p);
    else GIPB_CSR(4, int, M.col.p);
  }
#undef GIPB_CSR
}

template <typename T, int MODE, typename V>
void amg_mv_v(const SellT<T>& M, SellView<V> view, const V* v, const T* x, const T* b,
              const T* dinv, T* y, PcgScalars* S, cudaStream_t s, T w, const T* xs) {
  if constexpr (MODE == kResid) {  // only the folded residual scales its gathers
    if (xs) {
      amg_mv_vx<T, MODE, V, true>(M, view, v, x, b, dinv, y, S, s, w, xs);
      return;
    }
  }
  amg_mv_vx<T, MODE, V, false>(M, view, v, x, b, dinv, y, S, s, w, nullptr);
}

// y (mode) A x; xs (optional) scales the gathered x elementwise.
template <typename T, int MODE>
void amg_mv(const SellT<T>& M, const T* x, const T* b, const T* dinv, T* y, PcgScalars* S,
            cudaStream_t s, T w = T(1), const T* xs = nullptr) {
  if constexpr (std::is_same<T, float>::value) {
    if (M.half) {
      amg_mv_v<T, MODE, __half>(M, M.hview(), M.hval.p, x, b, dinv, y, S, s, w, xs);
      return;
    }
  }
  amg_mv_v<T, MODE, T>(M, M.view(), M.val.p, x, b, dinv, y, S, s, w, xs);
}

struct CycleFinish {
  PcgScalars* S;
  int first;
  __device__ void operator()(const double* t) const {
    const double rz = t[0];
    if (!(rz > 0.0) || !isfinite(rz)) {  // preconditioner lost definiteness: restart CG
      S->beta = 0.0;
      S->rz = 0.0;
      return;
    }
    S->beta = (!first && S->rz > 0.0) ? rz / S->rz : 0.0;
    S->rz = rz;
  }
};

// Level 0 post-smoothing with the dot: z = x + d (r - A x), r.z, beta; d = dinv[i], or the
// constant w when dinv is null (unit-diagonal level 0).
template <typename T>
__global__ void __launch_bounds__(256, 8) k_amg_smooth_dot(SellView<T> A, const T* __restrict__ x,
                                                           const T* __restrict__ r,
                                                           const T* __restrict__ dinv,
                                                           T* __restrict__ z, PcgScalars* S,
                                                           ReduceScratch rs, int first, T w) {
  if (amg_enter(S)) return;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  double acc[1] = {0.0};
  for (int s = gw; s < A.nslices; s += nw) {
    const T sum = amg_row<T, 4>(A, x, s, lane);
    const int i = s * 32 + lane;
    if (i < A.nrows) {
      const T ri = r[i];
      const T zi = fmat(dinv ? dinv[i] : w, ri - sum, x[i]);
      z[i] = zi;
      acc[0] += (double)ri * (double)zi;
    }
  }
  grid_reduce<SumOp, 1>(acc, rs, CycleFinish{S, first});
}

// Level-0 products from the packed FP32 operator (same FMA order as the plain layout, so
// the same results): kResid y = b - w A x; kSmooth z = x + d (r - A x) with r.z and beta,
// d = dinv[i], or the constant w when dinv is null (unit-diagonal level 0).
template <int NIB, int K, int MODE>
__global__ void __launch_bounds__(256, 8) k_amgp_spmv(SellView<float> A, PackedView pk,
                                                      const float* __restrict__ x,
                                                      const float* __restrict__ b,
                                                      const float* __restrict__ dinv,
                                                      float* __restrict__ y, PcgScalars* S,
                                                      ReduceScratch rs, int first, float w,
                                                      const int* __restrict__ yperm) {
  if (amg_enter(S)) return;
  constexpr int NT = 1 << NIB;
  __shared__ float tab[NT];
  for (int t = threadIdx.x; t < NT; t += blockDim.x) tab[t] = pk.table[t];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  double acc[1] = {0.0};
  PackedWords cur;
  for (int s = gw; s < A.nslices; s += nw) {
    packed_words<NIB>(pk.delta, pk.idx, pk.plain, s, lane, cur);
    int c[8];
    packed_cols(pk.base, s, cur.d, c);
    const int i = s * 32 + lane;
    // the row's own right-hand side, loaded with its words rather than after its gathers
    // (the 256^3 smoothing 112.5 against 118.8 us)
    const float rb = (i < A.nrows) ? b[i] : 0.f;
    float sum;
    if (cur.plain) {
      sum = amg_row<float, 2>(A, x, s, lane);
    } else {
      float xv[K];
#pragma unroll
      for (int j = 0; j < K; ++j) xv[j] = __ldg(x + c[j]);
      sum = 0.f;
#pragma unroll
      for (int j = 0; j < K; ++j) sum = fmaf(xv[j], tab[packed_index<NIB>(cur, j)], sum);
    }
    if (i < A.nrows) {
      if (MODE == kResid) {  // in aggregate order when yperm is given
        y[yperm ? yperm[i] : i] = (w == 1.0f) ? rb - sum : fmaf(-w, sum, rb);
      } else {
        const float ri = rb;
        const float zi = fmaf(dinv ? dinv[i] : w, ri - sum, x[i]);
        y[i] = zi;
        acc[0] += (double)ri * (double)zi;
      }
    }
  }
  if (MODE == kSmooth) grid_reduce<SumOp, 1>(acc, rs, CycleFinish{S, first});
}

template <int MODE>
void launch_amgp(const PackedView& pk, SellView<float> A, int nb, const float* x, const float* b,
                 const float* dinv, float* y, PcgScalars* S, ReduceScratch rs, int first,
                 cudaStream_t s, float w, const int* yperm) {
  if (pk.nib == 4 && pk.slots == 7)
    launch_dep(k_amgp_spmv<4, 7, MODE>, nb, 256, s, A, pk, x, b, dinv, y, S, rs, first, w, yperm);
  else if (pk.nib == 4)
    launch_dep(k_amgp_spmv<4, 8, MODE>, nb, 256, s, A, pk, x, b, dinv, y, S, rs, first, w, yperm);
  else if (pk.slots == 7)
    launch_dep(k_amgp_spmv<8, 7, MODE>, nb, 256, s, A, pk, x, b, dinv, y, S, rs, first, w, yperm);
  else
    launch_dep(k_amgp_spmv<8, 8, MODE>, nb, 256, s, A, pk, x, b, dinv, y, S, rs, first, w, yperm);
}

// Coarsest level: x = C b, one warp per row of the dense inverse.
template <typename T>
__device__ __forceinline__ void dense_rows(int m, const T* __restrict__ C, const T* __restrict__ b,
                                           T* __restrict__ x, int gw, int nw) {
  const int lane = threadIdx.x & 31;
  for (int i = gw; i < m; i += nw) {
    T acc = T(0);
    for (int j = lane; j < m; j += 32) acc = fmat(C[(size_t)i * m + j], b[j], acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) x[i] = acc;
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_amg_dense(int m, const T* __restrict__ C,
                                                   const T* __restrict__ b, T* __restrict__ x,
                                                   PcgScalars* S) {
  if (amg_enter(S)) return;
  dense_rows<T>(m, C, b, x, (blockIdx.x * blockDim.x + threadIdx.x) >> 5,
                (gridDim.x * blockDim.x) >> 5);
}

// ------------------------------------------------------------------ coarse tail
// The FP32 cycle's small levels in one cooperative launch: the products of those levels
// (the same row functions, so the same results as one kernel each) run one after the other
// over the whole grid, separated by a grid barrier instead of a kernel boundary; a dozen
// latency-bound launches of a few microseconds each become one.
namespace tail {

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// All CTAs of the grid have arrived and their earlier writes are visible; false in every
// thread when the wait gave up (about 2 s of SM clock).
__device__ bool grid_sync(unsigned* bar, unsigned target, int* s_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(bar, 1u);
    const long long t0 = clock64();
    int ok = 1;
    while (ld_acquire(bar) < target)
      if (clock64() - t0 > 4000000000LL) {
        ok = 0;
        break;
      }
    __threadfence();
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

template <int MODE, int LANES, typename V, bool XS>
__device__ __forceinline__ void csr_op(const TailOp& o, int gw, int nw) {
  csr_rows<float, MODE, LANES, V, int, XS>(o.nrows, o.rp, o.col, (const V*)o.val, o.x, o.b,
                                           o.dinv, o.y, 1.0f, o.xs, nullptr, gw, nw);
}

template <int MODE, typename V, bool XS>
__device__ __forceinline__ void sell_op(const TailOp& o, int gw, int nw) {
  const SellView<V> A{o.nrows, o.nslices, o.sptr, o.col, (const V*)o.val, 0};
  sell_rows<float, MODE, V, false, XS>(A, o.x, o.b, o.dinv, o.y, 1.0f, nullptr, o.xs, nullptr,
                                       nullptr, gw, nw);
}

// The forms a small level's operators take (TailOp::form): coarse operators with FP32
// values (residual with the folded Jacobi start, smoothing), transfers with FP16 values
// (restriction, prolongation onto the folded start).
__device__ void exec(const TailOp& o, int gw, int nw) {
  switch (o.form) {
    case kTailDense: dense_rows<float>(o.nrows, (const float*)o.val, o.b, o.y, gw, nw); break;
    case kTailSellResid: sell_op<kResid, float, true>(o, gw, nw); break;
    case kTailSellSmooth: sell_op<kSmooth, float, false>(o, gw, nw); break;
    case kTailSellRestrict: sell_op<kPlain, __half, false>(o, gw, nw); break;
    case kTailSellProlong: sell_op<kDiagAdd, __half, false>(o, gw, nw); break;
    case kTailCsrResid:
      if (o.lanes == 32) csr_op<kResid, 32, float, true>(o, gw, nw);
      else if (o.lanes == 16) csr_op<kResid, 16, float, true>(o, gw, nw);
      else csr_op<kResid, 8, float, true>(o, gw, nw);
      break;
    case kTailCsrSmooth:
      if (o.lanes == 32) csr_op<kSmooth, 32, float, false>(o, gw, nw);
      else if (o.lanes == 16) csr_op<kSmooth, 16, float, false>(o, gw, nw);
      else csr_op<kSmooth, 8, float, false>(o, gw, nw);
      break;
    case kTailCsrRestrict:
      if (o.lanes == 32) csr_op<kPlain, 32, __half, false>(o, gw, nw);
      else if (o.lanes == 16) csr_op<kPlain, 16, __half, false>(o, gw, nw);
      else if (o.lanes == 8) csr_op<kPlain, 8, __half, false>(o, gw, nw);
      else csr_op<kPlain, 4, __half, false>(o, gw, nw);
      break;
    case kTailCsrProlong:
      if (o.lanes == 32) csr_op<kDiagAdd, 32, __half, false>(o, gw, nw);
      else if (o.lanes == 16) csr_op<kDiagAdd, 16, __half, false>(o, gw, nw);
      else if (o.lanes == 8) csr_op<kDiagAdd, 8, __half, false>(o, gw, nw);
      else csr_op<kDiagAdd, 4, __half, false>(o, gw, nw);
      break;
    default: break;
  }
}

}  // namespace tail

// bar[0]: barrier arrivals, bar[1]: CTAs done; both zero between launches (the last CTA
// to leave resets them).  A barrier that gives up stops the solve with
// GIPB200_ERR_TIMEOUT.
__global__ void __launch_bounds__(256) k_amg_tail(const TailOp* __restrict__ ops, int nops,
                                                  unsigned* bar, PcgScalars* S) {
  if (amg_enter(S)) return;
  __shared__ int s_ok;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  bool ok = true;
  for (int k = 0; k < nops; ++k) {
    if (k > 0 && !tail::grid_sync(bar, (unsigned)k * gridDim.x, &s_ok)) {
      ok = false;
      break;
    }
    tail::exec(ops[k], gw, nw);
  }
  if (!ok) {
    if (threadIdx.x == 0) {
      S->status = GIPB200_ERR_TIMEOUT;
      S->done = 1;
    }
    return;  // the counters stay set; the solve's start clears them
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(bar + 1, 1u) == gridDim.x - 1) {
      bar[0] = 0u;
      bar[1] = 0u;
      __threadfence();
    }
  }
}

int vec_blocks(int n) {
  int b = 1;
  grid_blocks(256, std::max(n, 1), 1, kMaxReduceBlocks, &b);
  return b;
}

}  // namespace

// The packed level-0 products exist for FP32 only.
template <int MODE, typename T>
void launch_packed0(const PackedView& pk, SellView<T> A, int nb, const T* x, const T* b,
                    const T* dinv, T* y, PcgScalars* S, ReduceScratch rs, int first,
                    cudaStream_t s, T w = T(1), const int* yperm = nullptr) {
  if constexpr (std::is_same<T, float>::value)
    launch_amgp<MODE>(pk, A, nb, x, b, dinv, y, S, rs, first, s, w, yperm);
}

namespace {

// One level of the host hierarchy, handed to the consumer as soon as it is built.
struct HostLevel {
  int l = 0;
  const HCsr* A = nullptr;                 // the level's operator
  const std::vector<double>* d = nullptr;  // its diagonal
  const std::vector<double>* z = nullptr;  // its near-null vector
  double w = 0.0;                          // Jacobi weight 4 / (3 rho)
  const HCsr* P = nullptr;                 // prolongation / restriction (not on the coarsest)
  const HCsr* R = nullptr;
  const std::vector<int>* agg = nullptr;   // aggregate of every row (not on the coarsest)
  const std::vector<double>* cinv = nullptr;  // coarsest only: dense (pseudo-)inverse
};

// The smoothed-aggregation hierarchy of the n x n operator (host CSR, FP64), built on the
// host level by level; emit(const HostLevel&) consumes each level (returns a status).
template <typename F>
int host_hierarchy(int n, const int* rp, const int* ci, const double* v, const double* z0,
                   bool singular, double drop, F&& emit) {
  HCsr A;
  A.nr = A.nc = n;
  A.rp.assign(rp, rp + n + 1);
  A.ci.assign(ci, ci + rp[n]);
  A.v.assign(v, v + rp[n]);
  std::vector<double> z(z0, z0 + n);
  for (int l = 0; l < kMaxLevels; ++l) {
    HostLevel H;
    H.l = l;
    H.A = &A;
    H.z = &z;
    const std::vector<double> d = diagonal(A);
    H.d = &d;
    for (int i = 0; i < A.nr; ++i)
      if (!(d[i] > 0.0)) return fail(GIPB200_ERR_ARG, "AMG: level %d row %d has no positive diagonal", l, i);
    H.w = 4.0 / (3.0 * rho_bound(A, d));
    if (A.nr <= kCoarse && l > 0) {  // coarsest: dense inverse
      const int m = A.nr;
      std::vector<double> M((size_t)m * m, 0.0);
      for (int i = 0; i < m; ++i)
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) M[(size_t)i * m + A.ci[k]] += A.v[k];
      if (singular) {
        double zz = 0.0, dm = 0.0;
        for (int i = 0; i < m; ++i) zz += z[i] * z[i], dm += d[i];
        const double sigma = dm / m;
        for (int i = 0; i < m; ++i)
          for (int j = 0; j < m; ++j) M[(size_t)i * m + j] += sigma * z[i] * z[j] / zz;
      }
      std::vector<double> inv;
      if (!dense_inverse(m, M, inv))
        return fail(GIPB200_ERR_ARG, "AMG: coarsest operator (%d) is not positive definite", m);
      H.cinv = &inv;
      return emit(H);
    }
    setup_mark("AMG level: diagonal, bound");
    std::vector<int> agg;
    const int na = aggregate(A, d, agg);
    setup_mark("AMG level: aggregation");
    if (na == 0 || na > 0.8 * A.nr)
      return fail(GIPB200_ERR_ARG, "AMG: level %d (%d unknowns) coarsens only to %d", l, A.nr, na);
    // GIPB200_AMG_RELABEL=1: aggregates numbered by their first row instead of in the
    // order the greedy passes create them (measured on the 256^3 cavity: 4% more FP32
    // iterations and slower level-1 products, so off by default)
    if (getenv("GIPB200_AMG_RELABEL")) {
      std::vector<int> first((size_t)na, A.nr);
      for (int i = 0; i < A.nr; ++i) first[agg[i]] = std::min(first[agg[i]], i);
      std::vector<int> ord((size_t)na);
      for (int a = 0; a < na; ++a) ord[a] = a;
      std::sort(ord.begin(), ord.end(), [&](int a, int b) { return first[a] < first[b]; });
      std::vector<int> relabel((size_t)na);
      for (int k = 0; k < na; ++k) relabel[ord[k]] = k;
      for (int i = 0; i < A.nr; ++i) agg[i] = relabel[agg[i]];
    }
    std::vector<double> nrm((size_t)na, 0.0);
    for (int i = 0; i < A.nr; ++i) nrm[agg[i]] += z[i] * z[i];
    for (auto& q : nrm) q = std::sqrt(q);
    std::vector<double> p0((size_t)A.nr);
    for (int i = 0; i < A.nr; ++i) p0[i] = nrm[agg[i]] > 0.0 ? z[i] / nrm[agg[i]] : 0.0;
    HCsr P = smoothed_prolongator(A, d, agg, p0, na, H.w);
    HCsr R = transpose(P);
    setup_mark("AMG level: prolongator");
    HCsr AP, Ac;
    GIPB_TRY(spgemm(A, P, AP));
    GIPB_TRY(spgemm(R, AP, Ac));
    setup_mark("AMG level: Galerkin product");
    if (drop > 0.0) sparsify(Ac, nrm, drop);
    setup_mark("AMG level: sparsification");
    H.P = &P;
    H.R = &R;
    H.agg = &agg;
    GIPB_TRY(emit(H));
    setup_mark("AMG level: device upload");
    A = std::move(Ac);
    z = std::move(nrm);
  }
  return fail(GIPB200_ERR_ARG, "AMG: more than %d levels", kMaxLevels);
}

double amg_drop() {
  const char* e = getenv("GIPB200_AMG_DROP");
  return e ? atof(e) : kDrop;
}

}  // namespace

template <typename T>
int AmgT<T>::build(int n, const int* rp, const int* ci, const double* v, const double* z0,
                   bool singular, int x0_len, cudaStream_t s) {
  const auto t0 = std::chrono::steady_clock::now();
  lv.clear();
  nc = 0;
  const double nnz0 = (double)rp[n];
  double nnz_all = 0.0;
  GIPB_TRY(host_hierarchy(n, rp, ci, v, z0, singular, amg_drop(), [&](const HostLevel& H) -> int {
    std::unique_ptr<AmgLevel<T>> Lp(new AmgLevel<T>());
    AmgLevel<T>& L = *Lp;
    const HCsr& A = *H.A;
    L.n = A.nr;
    std::vector<T> dinv((size_t)A.nr);
    for (int i = 0; i < A.nr; ++i) dinv[i] = (T)(H.w / (*H.d)[i]);
    if (H.l == 0) {
      // the residual then gathers r (length n) where it gathered x0 (length x0_len): only
      // when level 0's operator gathers no column past n
      bool unit = A.nr > 0 && x0_len <= A.nr && !getenv("GIPB200_AMG_ROWDIAG");
      for (int i = 0; i < A.nr && unit; ++i) unit = std::fabs((*H.d)[i] - 1.0) <= 0.1;
      unit0 = unit;
      omega0 = H.w;
    }
    GIPB_TRY(L.dinv.upload(dinv.data(), dinv.size(), s));
    GIPB_TRY(L.x.alloc((size_t)(H.l == 0 ? std::max(A.nr, x0_len) : A.nr)));
    GIPB_TRY(L.x.zero(s));  // level 0: entries past n are gathered (as zero) by A0
    GIPB_TRY(L.t.alloc((size_t)A.nr));
    if (H.l > 0) {  // level 0 runs on the solver's own operator
      GIPB_TRY(L.b.alloc((size_t)A.nr));
      // GIPB200_AMG_COMPACT=1: 16-bit columns where they fit; GIPB200_AMG_COARSE_HALF=1:
      // FP16 values (both off: measured no faster)
      GIPB_TRY(upload(A, &L.A, s, std::is_same<T, float>::value && getenv("GIPB200_AMG_COARSE_HALF"),
                      getenv("GIPB200_AMG_COMPACT") != nullptr));
    }
    nnz_all += (double)A.nnz();
    if (H.cinv) {
      std::vector<T> cf(H.cinv->begin(), H.cinv->end());
      GIPB_TRY(cinv.upload(cf.data(), cf.size(), s));
      nc = A.nr;
    } else {
      // the FP32 cycle keeps its transfer operators in FP16 (R = P^T still holds exactly:
      // both round the same values), halving their value stream
      const bool half = std::is_same<T, float>::value;
      // (GIPB200_AMG_COMPACT=1: 16-bit columns where they fit; measured no faster for the
      // CSR operators and slower for the sliced prolongation, 191 against 163 us)
      const bool compact = getenv("GIPB200_AMG_COMPACT") != nullptr;
      GIPB_TRY(upload(*H.P, &L.P, s, half, compact, true));
      if (H.l == 0 && getenv("GIPB200_AMG_AGG_ORDER")) {
        // GIPB200_AMG_AGG_ORDER=1: level 0's residual is written in aggregate order (the
        // rows of aggregate 0, then of aggregate 1, ..., each in row order), and the
        // restriction reads it there, so a coarse row's columns lie close together.
        // Measured on the 256^3 cavity: the scattered residual writes cost 27 us and the
        // restriction gained nothing, so off by default.
        const std::vector<int>& agg = *H.agg;
        std::vector<int> start((size_t)H.R->nr + 1, 0);
        for (int a : agg) start[(size_t)a + 1]++;
        for (int j = 0; j < H.R->nr; ++j) start[j + 1] += start[j];
        std::vector<int> perm((size_t)A.nr);
        for (int i = 0; i < A.nr; ++i) perm[i] = start[agg[i]]++;
        HCsr Rp = *H.R;  // columns renumbered, each row's entries sorted by the new column
        for (int j = 0; j < Rp.nr; ++j) {
          std::vector<std::pair<int, double>> e;
          for (int k = Rp.rp[j]; k < Rp.rp[j + 1]; ++k) e.push_back({perm[Rp.ci[k]], Rp.v[k]});
          std::sort(e.begin(), e.end());
          for (int k = Rp.rp[j]; k < Rp.rp[j + 1]; ++k) {
            Rp.ci[k] = e[k - Rp.rp[j]].first;
            Rp.v[k] = e[k - Rp.rp[j]].second;
          }
        }
        GIPB_TRY(upload(Rp, &L.R, s, half, compact, true));
        GIPB_TRY(perm0.upload(perm.data(), perm.size(), s));
      } else {
        GIPB_TRY(upload(*H.R, &L.R, s, half, compact, true));
      }
    }
    lv.push_back(std::move(Lp));
    return GIPB200_OK;
  }));
  op_complexity = nnz_all / std::max(nnz0, 1.0);
  GIPB_TRY(build_tail(s));
  GIPB_CUDA(cudaStreamSynchronize(s));
  setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return GIPB200_OK;
}

// The coarse tail's product list: levels tail_from..L-2 down (folded residual,
// restriction), the dense coarsest solve, then the same levels up (prolongation onto the
// folded start, smoothing) -- the order and the data of the separate kernels.  Left off
// (tail_from = -1) for the FP64 cycle, without folding, or when an operator has a form
// the tail does not run (16-bit columns, FP16 coarse values, 4 threads per coarse row).
template <typename T>
int AmgT<T>::build_tail(cudaStream_t s) {
  tail_from = -1;
  tail_nops = 0;
  if constexpr (!std::is_same<T, float>::value) {
    return GIPB200_OK;
  } else {
    const int L = (int)lv.size();
    // GIPB200_AMG_TAIL=<CTAs per SM>: on (measured no faster than the separate kernels in
    // the step's graph: its grid barriers cost what the launches did)
    const char* tail_env = getenv("GIPB200_AMG_TAIL");
    const int tail_per_sm = tail_env ? atoi(tail_env) : 0;
    if (tail_per_sm <= 0 || !fold_coarse || L < 3 || nc <= 0) return GIPB200_OK;
    int tf = L - 1;
    while (tf - 1 >= 1 && lv[tf - 1]->n <= kTailRows) --tf;
    if (tf > L - 2) return GIPB200_OK;  // no level above the coarsest is small
    for (int l = tf; l < L - 1; ++l)
      if (!folds(l)) return GIPB200_OK;
    std::vector<TailOp> ops;
    const double w = sizeof(T);
    // the operator's form for one product; false when the tail does not run it
    auto add = [&](const SellT<T>& M, bool transfer, int sell_form, int csr_form,
                   const float* x, const float* b, const float* dinv, const float* xs, float* y,
                   int level, int kind, double bytes) -> bool {
      if (M.short_cols || M.half != transfer) return false;
      TailOp o{};
      o.nrows = M.nrows;
      o.nslices = M.nslices;
      o.sptr = M.sptr.p;
      o.rp = M.rp.p;
      o.col = M.col.p;
      o.val = transfer ? (const void*)M.hval.p : (const void*)M.val.p;
      o.lanes = M.lanes;
      if (M.lanes == 0) {
        o.form = sell_form;
      } else {
        if (!transfer && M.lanes < 8) return false;
        o.form = csr_form;
      }
      o.x = x;
      o.b = b;
      o.dinv = dinv;
      o.xs = xs;
      o.y = y;
      o.level = level;
      o.kind = kind;
      o.bytes = bytes;
      ops.push_back(o);
      return true;
    };
    for (int l = tf; l < L - 1; ++l) {
      const AmgLevel<T>& V = *lv[l];
      const double n = V.n, nn = lv[l + 1]->n;
      if (!add(V.A, false, kTailSellResid, kTailCsrResid, V.b.p, V.b.p, nullptr, V.dinv.p, V.t.p,
               l, GIPB200_CYCLE_RESIDUAL, stream_bytes(V.A) + 3.0 * n * w) ||
          !add(V.R, true, kTailSellRestrict, kTailCsrRestrict, V.t.p, nullptr, nullptr, nullptr,
               lv[l + 1]->b.p, l, GIPB200_CYCLE_RESTRICT, stream_bytes(V.R) + (n + nn) * w))
        return GIPB200_OK;
    }
    {
      TailOp o{};
      o.form = kTailDense;
      o.nrows = nc;
      o.val = cinv.p;
      o.b = lv[L - 1]->b.p;
      o.y = lv[L - 1]->x.p;
      o.level = L - 1;
      o.kind = GIPB200_CYCLE_DENSE;
      o.bytes = ((double)nc * nc + 2.0 * nc) * w;
      ops.push_back(o);
    }
    for (int l = L - 2; l >= tf; --l) {
      const AmgLevel<T>& V = *lv[l];
      const double n = V.n, nn = lv[l + 1]->n;
      const float* xc = (l + 1 == L - 1) ? lv[l + 1]->x.p : lv[l + 1]->t.p;
      if (!add(V.P, true, kTailSellProlong, kTailCsrProlong, xc, V.b.p, V.dinv.p, nullptr,
               V.x.p, l, GIPB200_CYCLE_PROLONG, stream_bytes(V.P) + (nn + 3.0 * n) * w) ||
          !add(V.A, false, kTailSellSmooth, kTailCsrSmooth, V.x.p, V.b.p, V.dinv.p, nullptr,
               V.t.p, l, GIPB200_CYCLE_SMOOTH, stream_bytes(V.A) + 4.0 * n * w))
        return GIPB200_OK;
    }
    DeviceInfo di;
    GIPB_TRY(device_info(&di));
    int per_sm = 0;
    GIPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_amg_tail, 256, 0));
    if (per_sm < 1) return GIPB200_OK;
    tail_grid = std::min(per_sm, tail_per_sm) * di.nsm;
    GIPB_TRY(tail_ops.upload(ops.data(), ops.size(), s));
    GIPB_TRY(tail_bar.alloc(2));
    GIPB_TRY(tail_bar.zero(s));
    tail_bytes = 0.0;
    for (const TailOp& o : ops) tail_bytes += o.bytes;
    tail_nops = (int)ops.size();
    tail_from = tf;
    return GIPB200_OK;
  }
}

template <typename T>
int AmgT<T>::reset_tail(cudaStream_t s) const {
  if (tail_from >= 0) GIPB_CUDA(cudaMemsetAsync(tail_bar.p, 0, 2 * sizeof(unsigned), s));
  return GIPB200_OK;
}

int CycleTrace::mark(cudaStream_t s, int lvl, int knd, double by, int frm) {
  GIPB_TRY(close(s));
  level.push_back(lvl);
  kind.push_back(knd);
  form.push_back(frm);
  bytes.push_back(by);
  return GIPB200_OK;
}

int CycleTrace::close(cudaStream_t s) {
  cudaEvent_t e;
  GIPB_CUDA(cudaEventCreate(&e));
  ev.push_back(e);
  GIPB_CUDA(cudaEventRecordWithFlags(e, s, captured ? cudaEventRecordExternal : 0));
  return GIPB200_OK;
}

CycleTrace::~CycleTrace() {
  for (cudaEvent_t e : ev) cudaEventDestroy(e);
}

template <typename T>
int AmgT<T>::enqueue(SellView<T> A0, const T* r, T* z0, PcgScalars* S, ReduceScratch rs, int first,
                     cudaStream_t s, const PackedView* pk, CycleTrace* tr,
                     double a0_stream_bytes) const {
  const bool packed = pk && pk->on && std::is_same<T, float>::value;
  const int L = (int)lv.size();
  const double w = sizeof(T);
  // bytes of each kernel as cycle_bytes counts them (profiling marks only)
  auto mark = [&](int l, int kind, double by, int form) -> int {
    return tr ? tr->mark(s, l, kind, by, form) : GIPB200_OK;
  };
  auto a_bytes = [&](int l) { return l == 0 ? a0_stream_bytes : stream_bytes(lv[l]->A); };
  // downward: pre-smooth from zero, residual, restriction (levels below the coarse tail)
  const bool u0 = unit0;  // level 0 never forms x0 = omega0 r
  const int tf = tail_from;
  for (int l = 0; l < L - 1 && (tf < 0 || l < tf); ++l) {
    const AmgLevel<T>& V = *lv[l];
    const T* b = l == 0 ? r : V.b.p;
    const double n = V.n, nn = lv[l + 1]->n;
    const bool skip = l == 0 && u0;
    // small levels >= 1 gather D^-1 b where they would gather the Jacobi start x = D^-1 b
    const bool fold = folds(l);
    if (!skip && !fold) {
      GIPB_TRY(mark(l, GIPB200_CYCLE_JACOBI0, 3.0 * n * w, GIPB200_FORM_VECTOR));
      launch_dep(k_amg_jacobi0<T>, vec_blocks(V.n), 256, s, V.n, (const T*)V.dinv.p, b, V.x.p, S);
    }
    GIPB_TRY(mark(l, GIPB200_CYCLE_RESIDUAL,
                  a_bytes(l) + (skip ? 2.0 : 3.0) * n * w + (l == 0 && perm0.p ? 4.0 * n : 0.0),
                  l == 0 ? (packed ? GIPB200_FORM_PACKED : GIPB200_FORM_SLICED)
                         : product_form(V.A)));
    if (l == 0) {
      const int bs = vec_blocks(A0.nslices * 32);
      if (packed)
        launch_packed0<kResid>(*pk, A0, bs, skip ? r : V.x.p, b, (const T*)nullptr, V.t.p, S, rs,
                               first, s, skip ? (T)omega0 : T(1), perm0.p);
      else
        launch_dep(k_amg_spmv<T, kResid, T, false>, bs, 256, s, A0, skip ? r : (const T*)V.x.p,
                   b, (const T*)nullptr, V.t.p, S, skip ? (T)omega0 : T(1), (const int*)perm0.p,
                   (const T*)nullptr, (const unsigned short*)nullptr, (const int*)nullptr);
    } else if (fold) {  // t = b - A (D^-1 b)
      amg_mv<T, kResid>(V.A, b, b, (const T*)nullptr, V.t.p, S, s, T(1), V.dinv.p);
    } else {  // t = b - A x
      amg_mv<T, kResid>(V.A, V.x.p, b, (const T*)nullptr, V.t.p, S, s);
    }
    GIPB_TRY(mark(l, GIPB200_CYCLE_RESTRICT, stream_bytes(V.R) + (n + nn) * w,
                  product_form(V.R)));
    amg_mv<T, kPlain>(V.R, V.t.p, (const T*)nullptr, (const T*)nullptr, lv[l + 1]->b.p, S, s);
  }
  const AmgLevel<T>& C = *lv[L - 1];
  if (tf >= 0) {  // the small levels and the coarsest in one cooperative launch
    GIPB_TRY(mark(tf, GIPB200_CYCLE_TAIL, tail_bytes, GIPB200_FORM_TAIL));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)tail_grid);
    cfg.blockDim = dim3(256);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    GIPB_CUDA(cudaLaunchKernelEx(&cfg, k_amg_tail, (const TailOp*)tail_ops.p, tail_nops,
                                 tail_bar.p, S));
  } else {
    GIPB_TRY(mark(L - 1, GIPB200_CYCLE_DENSE, ((double)nc * nc + 2.0 * nc) * w,
                  GIPB200_FORM_DENSE));
    launch_dep(k_amg_dense<T>, std::min(kMaxReduceBlocks, (nc + 7) / 8), 256, s, nc,
               (const T*)cinv.p, (const T*)C.b.p, C.x.p, S);
  }
  // upward: prolongation, post-smoothing (level 0 also reduces r.z)
  for (int l = std::min(L - 2, tf >= 0 ? tf - 1 : L - 2); l >= 0; --l) {
    const AmgLevel<T>& V = *lv[l];
    const T* xc = (l + 1 == L - 1) ? lv[l + 1]->x.p : lv[l + 1]->t.p;
    const double n = V.n, nn = lv[l + 1]->n;
    const bool skip = l == 0 && u0;
    const bool fold = folds(l);
    GIPB_TRY(mark(l, GIPB200_CYCLE_PROLONG, stream_bytes(V.P) + (nn + (fold ? 3.0 : 2.0) * n) * w,
                  product_form(V.P)));
    if (skip)  // x0 = omega0 r + P x1
      amg_mv<T, kScaleAdd>(V.P, xc, r, (const T*)nullptr, V.x.p, S, s, (T)omega0);
    else if (fold)  // x = D^-1 b + P x_coarse
      amg_mv<T, kDiagAdd>(V.P, xc, V.b.p, V.dinv.p, V.x.p, S, s);
    else
      amg_mv<T, kAdd>(V.P, xc, (const T*)nullptr, (const T*)nullptr, V.x.p, S, s);
    GIPB_TRY(mark(l, GIPB200_CYCLE_SMOOTH, a_bytes(l) + (skip ? 3.0 : 4.0) * n * w,
                  l == 0 ? (packed ? GIPB200_FORM_PACKED : GIPB200_FORM_SMOOTH_DOT)
                         : product_form(V.A)));
    if (l == 0) {
      const int bs = vec_blocks(A0.nslices * 32);
      if (packed)
        launch_packed0<kSmooth>(*pk, A0, bs, V.x.p, r, skip ? (const T*)nullptr : V.dinv.p, z0,
                                S, rs, first, s, (T)omega0);
      else
        launch_dep(k_amg_smooth_dot<T>, bs, 256, s, A0, (const T*)V.x.p, r,
                   skip ? (const T*)nullptr : (const T*)V.dinv.p, z0, S, rs, first, (T)omega0);
    } else {
      amg_mv<T, kSmooth>(V.A, V.x.p, V.b.p, V.dinv.p, V.t.p, S, s);
    }
  }
  if (tr) GIPB_TRY(tr->close(s));
  GIPB_LAUNCH_CHECK();
  return GIPB200_OK;
}

template <typename T>
double AmgT<T>::cycle_bytes(double a0_stream_bytes) const {
  const double w = sizeof(T);
  const int L = (int)lv.size();
  double b = 0.0;
  for (int l = 0; l < L - 1; ++l) {
    const AmgLevel<T>& V = *lv[l];
    const double n = V.n, nn = lv[l + 1]->n;
    const double a = l == 0 ? a0_stream_bytes : stream_bytes(V.A);
    const bool skip = l == 0 && unit0;                   // x0 = omega0 r not formed
    const bool fold = folds(l);                          // x = D^-1 b formed where gathered
    if (!skip && !fold) b += 3.0 * n * w;                // x = dinv b
    b += a + (skip ? 2.0 : 3.0) * n * w;                 // t = b - A x
    if (l == 0 && perm0.p) b += 4.0 * n;                 // its aggregate-order positions
    b += stream_bytes(V.R) + (n + nn) * w;               // b_next = R t
    b += stream_bytes(V.P) + (nn + (fold ? 3.0 : 2.0) * n) * w;  // x (+)= P x_next
    b += a + (skip ? 3.0 : 4.0) * n * w;                 // smoothed x
  }
  b += ((double)nc * nc + 2.0 * nc) * w;                 // dense coarsest
  return b;
}

template struct AmgT<float>;
template struct AmgT<double>;

namespace {

// max |a_ij - a_ji| / max |a| over the stored pattern (1 when the pattern is not symmetric).
double asymmetry(const HCsr& A) {
  HCsr S = A;
  for (int i = 0; i < S.nr; ++i) {
    std::vector<std::pair<int, double>> e;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) e.emplace_back(A.ci[k], A.v[k]);
    std::sort(e.begin(), e.end(),
              [](const std::pair<int, double>& a, const std::pair<int, double>& b) {
                return a.first < b.first;
              });
    for (size_t q = 0; q < e.size(); ++q) {
      S.ci[A.rp[i] + q] = e[q].first;
      S.v[A.rp[i] + q] = e[q].second;
    }
  }
  const HCsr T = transpose(S);
  if (T.rp != S.rp || T.ci != S.ci) return 1.0;
  double big = 0.0, diff = 0.0;
  for (size_t k = 0; k < S.v.size(); ++k) {
    big = std::max(big, std::fabs(S.v[k]));
    diff = std::max(diff, std::fabs(S.v[k] - T.v[k]));
  }
  return big > 0.0 ? diff / big : 0.0;
}

}  // namespace

}  // namespace gipb200

using namespace gipb200;

extern "C" int gipb200_amg_host_levels(int n, const int* rowptr, const int* col, const double* val,
                                       const double* z, int singular, double drop, int max_levels,
                                       int* levels, int* rows, long long* nnz, double* checks) {
  if (n <= 0 || !rowptr || !col || !val || !z || max_levels < 1 || !levels || !rows || !nnz ||
      !checks)
    return fail(GIPB200_ERR_ARG, "bad arguments");
  GIPB_TRY(validate_csr(n, n, rowptr[n], rowptr, col, n, "AMG operator"));
  int count = 0;
  const int st = host_hierarchy(n, rowptr, col, val, z, singular != 0, drop, [&](const HostLevel& H) -> int {
    if (count >= max_levels) return GIPB200_OK;
    const HCsr& A = *H.A;
    const std::vector<double>& zl = *H.z;
    double amax = 0.0, zmax = 0.0, res = 0.0, dmin = HUGE_VAL;
    for (double a : A.v) amax = std::max(amax, std::fabs(a));
    for (double q : zl) zmax = std::max(zmax, std::fabs(q));
    for (int i = 0; i < A.nr; ++i) {
      double t = 0.0;
      for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) t += A.v[k] * zl[A.ci[k]];
      res = std::max(res, std::fabs(t));
      dmin = std::min(dmin, (*H.d)[i]);
    }
    rows[count] = A.nr;
    nnz[count] = A.nnz();
    checks[3 * count + 0] = asymmetry(A);
    checks[3 * count + 1] = (amax > 0.0 && zmax > 0.0) ? res / (amax * zmax) : 0.0;
    checks[3 * count + 2] = dmin;
    ++count;
    return GIPB200_OK;
  });
  *levels = count;
  return st;
}
