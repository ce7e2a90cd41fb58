// Context and C ABI of libggbtddft (include/ggbtddft.h).
//
// Owns every device buffer (src/main.cu:228-423 allocates the reference's), builds the angular
// chain matrices of each grid group, computes the initial potentials (h_timePropagation.cuh:47-57)
// and advances all runs by replaying a captured CUDA graph of a chunk of steps
// (h_timePropagation.cuh:59-112 runs ~30 + 4 N_kso N_l launches and syncs per step instead).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ggbtddft.h"
#include "ggb_internal.cuh"
#include "ggb_mixed.cuh"

using namespace ggb;

namespace {

struct GroupHost {
  ggb_group_desc d{};
  int n_cols = 0, n_tiles = 0, obs_seg = TR, ldS = 0;
  std::vector<int> runs;         // ctx run indices
  bool grid_set = false, w_set = false;
  std::vector<double> r, drdx, P;
  // angular eigen-systems as given: [coupling][m] -> V (n_l*n_l), D (n_l)
  std::vector<std::vector<std::vector<double>>> V, D;
  std::vector<std::vector<bool>> ang_set;
  // device
  double *r_d = nullptr, *drdx_d = nullptr, *P_d = nullptr;
  double2* W_d = nullptr;        // FP64 form
  double *mats_d = nullptr, *dph_d = nullptr, *coef_d = nullptr;
  double2 *x_d = nullptr, *y_d = nullptr;     // FP64 orbitals
  int *col_run_d = nullptr, *col_m_d = nullptr, *col_occ_d = nullptr, *runs_d = nullptr;
  double* dens_d = nullptr;
  double4* obs_d = nullptr;
  int* step_d = nullptr;
  unsigned* done_d = nullptr;
  unsigned* fin_cnt_d = nullptr;
  double* fin_scr_d = nullptr;
  bool needs_init = true;
  GroupArgs args{};
  ThetaArgs theta_args{};        // theta form with n_har > 4 (ggb_theta.cu)
  MixedGroup mixed;              // split-precision form (ggb_mixed.cu)
  // flags shared by the runs of the group
  int n_har = 0, use_hartree = 0, target_id = 0, theta = 0;
  double dt = 0.0;
};

struct RunHost {
  ggb_run_desc d{};
  int col0 = 0;
  bool orb_set = false, field_set = false;
  double *E_d = nullptr, *v_d = nullptr, *v0_d = nullptr, *vexc_d = nullptr, *vexc0_d = nullptr;
  double *rho_frozen_d = nullptr, *norm_d = nullptr, *norm0_d = nullptr;
  double2 *dip_d = nullptr, *acc_d = nullptr, *dip_tot_d = nullptr, *acc_tot_d = nullptr;
  double* htab_d = nullptr;      // theta form with n_har > 4
  std::vector<int> l, m, occ;
};

}  // namespace

struct ggb_ctx {
  ggb_dims dims{};
  std::vector<GroupHost> groups;
  std::vector<RunHost> runs;
  RunDev* runs_dev = nullptr;
  unsigned* status_d = nullptr;
  bool prepared = false;
  std::string err;
  int device = 0;
  // graphs of `graph_steps` steps and of one step: a call of n steps replays the first n / 32 times
  // and the second n % 32 times, so every step runs from a graph
  int graph_steps = 32;
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraphExec_t graph1_exec = nullptr;
  cudaStream_t cap_stream = nullptr;
  // one stream per grid group (groups share no buffers, so their steps run concurrently), with the
  // events that fork them from and join them to the caller's stream
  std::vector<cudaStream_t> group_streams;
  std::vector<cudaEvent_t> group_done;
  cudaEvent_t fork_ev = nullptr;
  std::vector<void*> allocs;
};

static int fail(ggb_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(ctx, GGB_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                                   \
  } while (0)

template <class T>
static int dalloc(ggb_ctx* ctx, T** p, size_t count) {
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess)
    return fail(ctx, GGB_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
  ctx->allocs.push_back(*p);
  e = cudaMemset(*p, 0, count * sizeof(T));
  if (e != cudaSuccess) return fail(ctx, GGB_ERR_CUDA, "cudaMemset failed: %s", cudaGetErrorString(e));
  return GGB_OK;
}

// ----------------------------------------------------------------------------------------------
// angular coefficients (angularCoefficients.cuh:1-174), host copies for the coefficient tables
// ----------------------------------------------------------------------------------------------
static double h_cu(int ll, int mm) {
  if (ll >= 0 && ll >= mm) {
    double l = ll, m = mm;
    return std::sqrt((std::pow(l + 1.0, 2.0) - std::pow(m, 2.0)) / ((2.0 * l + 1.0) * (2.0 * l + 3.0)));
  }
  return 0.0;
}
static double h_cd(int ll, int mm) {
  if (ll >= 1 && ll - 1 >= mm) {
    double l = ll, m = mm;
    return std::sqrt((std::pow(l, 2.0) - std::pow(m, 2.0)) / ((2.0 * l + 1.0) * (2.0 * l - 1.0)));
  }
  return 0.0;
}
static double h_p(int ll, int mm) {
  if (mm <= ll && ll >= 1) {
    double l = ll, m = mm;
    return (l * (l + 1.0) - 3.0 * std::pow(m, 2.0)) / ((2.0 * l - 1.0) * (2.0 * l + 3.0));
  }
  return 0.0;
}
static double h_qu(int ll, int mm) {
  if (mm <= ll && ll >= 0) {
    double l = ll, m = mm;
    return 1.50 / (2.0 * l + 3.0) *
           std::sqrt((std::pow(l + 1.0, 2.0) - std::pow(m, 2.0)) * (std::pow(l + 2.0, 2.0) - std::pow(m, 2.0)) /
                     ((2.0 * l + 1.0) * (2.0 * l + 5.0)));
  }
  return 0.0;
}
static double h_qd(int ll, int mm) {
  if (mm <= ll - 2 && ll >= 2) {
    double l = ll, m = mm;
    return 1.50 / (2.0 * l - 1.0) *
           std::sqrt((std::pow(l, 2.0) - std::pow(m, 2.0)) * (std::pow(l - 1.0, 2.0) - std::pow(m, 2.0)) /
                     ((2.0 * l + 1.0) * (2.0 * l - 3.0)));
  }
  return 0.0;
}
static double h_p3(int ll, int mm) {
  if (ll >= mm) {
    double l = ll, m = mm;
    return 1.50 * (l * (l + 2.0) - 5.0 * std::pow(m, 2.0)) / (2.0 * l - 1.0) / (2.0 * l + 5.0) *
           std::sqrt((std::pow(l + 1.0, 2.0) - std::pow(m, 2.0)) / (2.0 * l + 1.0) / (2.0 * l + 3.0));
  }
  return 0.0;
}
static double h_f3(int ll, int mm) {
  if (ll >= mm) {
    double l = ll, m = mm;
    return 2.50 / (2.0 * l + 3.0) / (2.0 * l + 5.0) *
           std::sqrt((std::pow(l + 1.0, 2.0) - std::pow(m, 2.0)) * (std::pow(l + 2.0, 2.0) - std::pow(m, 2.0)) *
                     (std::pow(l + 3.0, 2.0) - std::pow(m, 2.0)) / (2.0 * l + 1.0) / (2.0 * l + 7.0));
  }
  return 0.0;
}

// ----------------------------------------------------------------------------------------------
// chain construction
// ----------------------------------------------------------------------------------------------
namespace {
struct Act {
  int coupling;
  int phase;
};
}  // namespace

// Active couplings of the first half in the reference's order FF, FP, D, P
// (h_timePropagation.cuh:62-72).  A coupling whose phase is identically zero is skipped: its
// rotations are an orthogonal V V^T = I (e.g. FP without Hartree, h_timePropagation.cuh:65).
static std::vector<Act> active_couplings(const GroupHost& g) {
  const bool h = g.use_hartree == 1 && g.target_id > 0;
  std::vector<Act> a;
  if (g.theta) {
    // the theta form: the P coupling's eigenbasis only, with the whole angular potential in its phase
    a.push_back({GGB_COUPLING_P, PH_THETA});
    return a;
  }
  if (h && g.n_har >= 4) a.push_back({GGB_COUPLING_FF, PH_FF});   // couplingF.cuh:103
  if (h && g.n_har >= 3) a.push_back({GGB_COUPLING_FP, PH_FP});   // couplingP.cuh:148
  if (h && g.n_har >= 3) a.push_back({GGB_COUPLING_D, PH_D});     // couplingD.cuh:103 (v_2 = 0 without Hartree)
  a.push_back({GGB_COUPLING_P, PH_P});
  return a;
}

// S[l][j] of a product step y = A x:  first A = V_a^T  ->  S = V_a;
// pair A = V_b^T V_a  ->  S = V_a^T V_b;  last A = V_a  ->  S = V_a^T.
static void build_chain(GroupHost& g, const std::vector<Act>& seq, int half, int mat_base, Chain& ch,
                        std::vector<double>& mats) {
  const int n_l = g.d.n_l, n_m = g.d.n_m, ldS = g.ldS;
  const size_t per_m = (size_t)n_l * ldS, per_mat = per_m * n_m;
  const int k = (int)seq.size();
  ch.n_ops = k + 1;
  // couplingS.cuh:18,49; the theta form carries the S terms in its one phase
  const bool s_on = !g.theta && g.n_har >= 3 && g.use_hartree == 1 && g.target_id > 0;
  ch.pre_s = (half == 1) && s_on;
  ch.post_s = (half == 0) && s_on;
  for (int o = 0; o <= k; ++o) {
    const int mat = mat_base + o;
    ch.ops[o].mat = mat;
    ch.ops[o].phase = o < k ? seq[o].phase : PH_NONE;
    ch.ops[o].coupling = o < k ? seq[o].coupling : 0;
    for (int m = 0; m < n_m; ++m) {
      double* S = mats.data() + (size_t)mat * per_mat + (size_t)m * per_m;
      if (o == 0) {
        const auto& Va = g.V[seq[0].coupling][m];
        for (int l = 0; l < n_l; ++l)
          for (int j = 0; j < n_l; ++j) S[(size_t)l * ldS + j] = Va[(size_t)l * n_l + j];
      } else if (o == k) {
        const auto& Va = g.V[seq[k - 1].coupling][m];
        for (int l = 0; l < n_l; ++l)
          for (int j = 0; j < n_l; ++j) S[(size_t)l * ldS + j] = Va[(size_t)j * n_l + l];
      } else {
        const auto& Va = g.V[seq[o - 1].coupling][m];
        const auto& Vb = g.V[seq[o].coupling][m];
        for (int l = 0; l < n_l; ++l)
          for (int j = 0; j < n_l; ++j) {
            long double s = 0.0L;
            for (int q = 0; q < n_l; ++q) s += (long double)Va[(size_t)q * n_l + l] * Vb[(size_t)q * n_l + j];
            S[(size_t)l * ldS + j] = (double)s;
          }
      }
    }
  }
}

// Gauss-Legendre nodes and weights of order n (x_k > 0 for k < n/2, x_(n-1-k) = -x_k), Newton on
// P_n from the Chebyshev guesses, in long double.
static void gauss_legendre(int n, std::vector<long double>& x, std::vector<long double>& w) {
  x.assign(n, 0.0L);
  w.assign(n, 0.0L);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int i = 0; i < (n + 1) / 2; ++i) {
    long double z = std::cos(pi * (i + 0.75L) / (n + 0.5L)), dp = 0.0L;
    for (int it = 0; it < 100; ++it) {
      long double p0 = 1.0L, p1 = z;
      for (int k = 2; k <= n; ++k) {
        const long double p2 = ((2.0L * k - 1.0L) * z * p1 - (k - 1.0L) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0L);
      const long double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-19L) break;
    }
    x[i] = z;
    x[n - 1 - i] = -z;
    w[i] = w[n - 1 - i] = 2.0L / ((1.0L - z * z) * dp * dp);
  }
}

// Tables and buffers of the exact multipoles of the theta form with n_har > 4 (ggb_theta.cu).
static int prepare_theta_tables(ggb_ctx* ctx, GroupHost& g, int n_mp) {
  const int n_l = g.d.n_l, n_m = g.d.n_m, n_r = g.d.n_r, nq = n_l, ldS = g.ldS;
  std::vector<long double> xq, wq;
  gauss_legendre(2 * n_l, xq, wq);   // xq[0 .. n_l-1] > 0
  std::vector<double> T((size_t)n_m * nq * n_l, 0.0), wP((size_t)n_mp * nq), PLj((size_t)n_m * n_mp * ldS, 0.0);
  for (int m = 0; m < n_m; ++m)
    for (int q = 0; q < nq; ++q) {
      // normalised associated Legendre functions of order m by the dipole coupling's recurrence
      // x Theta_l = c_u(l) Theta_(l+1) + c_d(l) Theta_(l-1); Theta_m = C (1 - x^2)^(m/2),
      // C^2 = (2m+1)! / (2^(2m+1) (m!)^2)
      const long double z = xq[q];
      long double c2 = 0.5L;
      for (int k = 1; k <= m; ++k) c2 *= (2.0L * k + 1.0L) * (2.0L * k) / (4.0L * k * k);
      long double tm1 = 0.0L, t0 = std::sqrt(c2) * std::pow(1.0L - z * z, 0.5L * m);
      double* row = T.data() + ((size_t)m * nq + q) * n_l;
      for (int l = m; l < n_l; ++l) {
        row[l] = (double)t0;
        if (l + 1 < n_l) {
          const long double t1 = (z * t0 - (l > m ? (long double)h_cd(l, m) * tm1 : 0.0L)) / (long double)h_cu(l, m);
          tm1 = t0;
          t0 = t1;
        }
      }
    }
  for (int q = 0; q < nq; ++q) {
    long double p0 = 1.0L, p1 = xq[q];
    for (int L = 0; L < n_mp; ++L) {
      const long double pl = L == 0 ? 1.0L : p1;
      wP[(size_t)L * nq + q] = (double)(wq[q] * pl);
      if (L >= 1) {
        const long double p2 = ((2.0L * L + 1.0L) * xq[q] * p1 - L * p0) / (L + 1.0L);
        p0 = p1;
        p1 = p2;
      }
    }
  }
  for (int m = 0; m < n_m; ++m)
    for (int j = m; j < n_l; ++j) {
      const long double z = g.D[GGB_COUPLING_P][m][j];
      long double p0 = 1.0L, p1 = z;
      for (int L = 0; L < n_mp; ++L) {
        PLj[((size_t)m * n_mp + L) * ldS + j] = (double)(L == 0 ? 1.0L : p1);
        if (L >= 1) {
          const long double p2 = ((2.0L * L + 1.0L) * z * p1 - L * p0) / (L + 1.0L);
          p0 = p1;
          p1 = p2;
        }
      }
    }
  // ratio powers of the Hartree recurrences, fixed by the grid: (r_(a-1)/r_a)^L for L = 0 .. n_mp
  std::vector<double> rq((size_t)(n_mp + 1) * n_r, 0.0);
  for (int a = 1; a < n_r; ++a) {
    const long double lq = std::log((long double)g.r[a - 1] / (long double)g.r[a]);
    for (int L = 0; L <= n_mp; ++L) rq[(size_t)L * n_r + a] = (double)std::exp((long double)L * lq);
  }
  ThetaArgs& t = g.theta_args;
  t.n_mp = n_mp;
  t.nq = nq;
  double *Td, *wPd, *PLd, *rqd, *fine, *rho, *vmp;
  int rc;
  const size_t nrun = g.runs.size();
  if ((rc = dalloc(ctx, &Td, T.size())) || (rc = dalloc(ctx, &wPd, wP.size())) || (rc = dalloc(ctx, &PLd, PLj.size())) ||
      (rc = dalloc(ctx, &rqd, rq.size())) || (rc = dalloc(ctx, &fine, nrun * 2 * nq * n_r)) ||
      (rc = dalloc(ctx, &rho, nrun * n_mp * n_r)) || (rc = dalloc(ctx, &vmp, nrun * n_mp * n_r)))
    return rc;
  CK(cudaMemcpy(Td, T.data(), T.size() * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(wPd, wP.data(), wP.size() * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(PLd, PLj.data(), PLj.size() * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(rqd, rq.data(), rq.size() * sizeof(double), cudaMemcpyHostToDevice));
  t.T = Td; t.wP = wPd; t.PLj = PLd; t.rq = rqd; t.fine = fine; t.rho = rho; t.vmp = vmp;
  for (int ri : g.runs) {
    RunHost& r = ctx->runs[ri];
    if ((rc = dalloc(ctx, &r.htab_d, (size_t)n_m * n_l * n_r))) return rc;
  }
  return GGB_OK;
}

static int prepare(ggb_ctx* ctx) {
  if (ctx->prepared) return GGB_OK;
  int n_l_max = 0, n_r_max = 0;
  for (const GroupHost& g : ctx->groups) {
    n_l_max = std::max(n_l_max, g.d.n_l);
    n_r_max = std::max(n_r_max, g.d.n_r);
  }
  CK(configure_kernels_fp64(n_l_max, n_r_max));
  for (size_t gi = 0; gi < ctx->groups.size(); ++gi) {
    GroupHost& g = ctx->groups[gi];
    if (!g.grid_set) return fail(ctx, GGB_ERR_STATE, "group %zu: grid not set", gi);
    if (!g.w_set) return fail(ctx, GGB_ERR_STATE, "group %zu: radial propagators not set", gi);
    std::vector<Act> seq = active_couplings(g);
    for (const Act& a : seq)
      for (int m = 0; m < g.d.n_m; ++m)
        if (!g.ang_set[a.coupling][m])
          return fail(ctx, GGB_ERR_STATE, "group %zu: angular coupling %d for m=%d not set", gi, a.coupling, m);
    const int n_l = g.d.n_l, n_m = g.d.n_m, ldS = g.ldS;
    const int k = (int)seq.size();
    const int n_mats = 2 * (k + 1);
    std::vector<double> mats((size_t)n_mats * n_m * n_l * ldS, 0.0);
    std::vector<Act> rev(seq.rbegin(), seq.rend());
    Chain c0{}, c1{}, c2{};
    build_chain(g, seq, 0, 0, c0, mats);
    build_chain(g, rev, 1, k + 1, c1, mats);
    c2.n_ops = 0;
    int rc;
    if ((rc = dalloc(ctx, &g.mats_d, mats.size()))) return rc;
    CK(cudaMemcpy(g.mats_d, mats.data(), mats.size() * sizeof(double), cudaMemcpyHostToDevice));
    std::vector<double> dph((size_t)4 * n_m * ldS, 0.0);
    for (int c = 0; c < 4; ++c)
      for (int m = 0; m < n_m; ++m)
        if (g.ang_set[c][m])
          for (int j = 0; j < n_l; ++j) dph[((size_t)c * n_m + m) * ldS + j] = g.D[c][m][j];
    if ((rc = dalloc(ctx, &g.dph_d, dph.size()))) return rc;
    CK(cudaMemcpy(g.dph_d, dph.data(), dph.size() * sizeof(double), cudaMemcpyHostToDevice));
    std::vector<double> coef((size_t)COEF_N * n_m * n_l);
    for (int m = 0; m < n_m; ++m)
      for (int l = 0; l < n_l; ++l) {
        coef[((size_t)CF_CU * n_m + m) * n_l + l] = h_cu(l, m);
        coef[((size_t)CF_CD * n_m + m) * n_l + l] = h_cd(l, m);
        coef[((size_t)CF_P * n_m + m) * n_l + l] = h_p(l, m);
        coef[((size_t)CF_QU * n_m + m) * n_l + l] = h_qu(l, m);
        coef[((size_t)CF_QD * n_m + m) * n_l + l] = h_qd(l, m);
        coef[((size_t)CF_P3 * n_m + m) * n_l + l] = h_p3(l, m);
        coef[((size_t)CF_F3 * n_m + m) * n_l + l] = h_f3(l, m);
      }
    if ((rc = dalloc(ctx, &g.coef_d, coef.size()))) return rc;
    CK(cudaMemcpy(g.coef_d, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice));

    GroupArgs& a = g.args;
    a.n_r = g.d.n_r; a.n_l = n_l; a.n_m = n_m; a.n_cols = g.n_cols; a.n_tiles = g.n_tiles; a.obs_seg = g.obs_seg; a.ldS = ldS;
    a.n_runs = (int)g.runs.size();
    a.hartree_on = (g.use_hartree == 1 && g.target_id > 0);
    a.p_hartree = (g.use_hartree == 1 && g.n_har > 1 && g.target_id > 0);
    a.theta = g.theta;
    // the theta form with n_har > 4 takes its multipoles L >= 1 from the exact quadratures of
    // ggb_theta.cu; the angular kernels' l-space partials then only carry L = 0 (monopole, norm)
    a.theta_tab = (g.theta && a.hartree_on && g.n_har > N_DEN) ? 1 : 0;
    a.n_den = a.hartree_on ? (a.theta_tab ? 1 : std::min(g.n_har, N_DEN)) : 0;
    if (a.theta_tab)
      if ((rc = prepare_theta_tables(ctx, g, g.n_har))) return rc;
    a.per_l = ctx->dims.per_l;
    a.dt = g.dt;
    // the FP64 form never raises a norm (its propagators are contractions, rounding is ~1e-15); the
    // split forms carry a representation error of their operators that may drift it by a few 1e-5
    // over a long pulse
    a.norm_tol = ctx->dims.precision == GGB_FP64 ? 1e-6 : 1e-3;
    const int n_g = g.d.n_r + 1;
    a.n_g_fac = (double)(n_g * (n_g + 1)) / 2.0;
    a.r = g.r_d; a.drdx = g.drdx_d; a.P = g.P_d;
    a.mats = g.mats_d; a.dph = g.dph_d; a.coef = g.coef_d;
    a.col_run = g.col_run_d; a.col_m = g.col_m_d; a.col_occ = g.col_occ_d; a.runs_of_group = g.runs_d;
    a.runs = ctx->runs_dev;
    a.dens = g.dens_d; a.obs = g.obs_d; a.step = g.step_d; a.status = ctx->status_d; a.done = g.done_d;
    a.fin_cnt = g.fin_cnt_d; a.fin_scr = g.fin_scr_d;
    a.chain[0] = c0; a.chain[1] = c1;
    a.chain[2] = c2;
    if (ctx->dims.precision != GGB_FP64) {
      if ((rc = mixed_prepare(g.mixed, a, g.W_d, g.x_d, g.y_d, ctx->dims.precision, ctx->err))) return rc;
    }
  }
  // device-side run table
  std::vector<RunDev> rd(ctx->runs.size());
  for (size_t i = 0; i < ctx->runs.size(); ++i) {
    RunHost& r = ctx->runs[i];
    if (!r.orb_set) return fail(ctx, GGB_ERR_STATE, "run %zu: orbitals not set", i);
    if (!r.field_set) return fail(ctx, GGB_ERR_STATE, "run %zu: field not set", i);
    rd[i] = RunDev{r.E_d, r.v_d, r.v0_d, r.vexc_d, r.vexc0_d, r.rho_frozen_d, r.dip_d, r.acc_d,
                   r.dip_tot_d, r.acc_tot_d, r.norm_d, r.norm0_d, r.htab_d, r.col0, r.d.n_orb, ctx->dims.n_t,
                   r.d.flags};
  }
  CK(cudaMemcpy(ctx->runs_dev, rd.data(), rd.size() * sizeof(RunDev), cudaMemcpyHostToDevice));
  ctx->prepared = true;
  return GGB_OK;
}

// one step of one group: angular half 1, radial, angular half 2 (+ partials), finalize
static void launch_group_step(ggb_ctx* ctx, GroupHost& g, cudaStream_t s) {
  const GroupArgs& a = g.args;
  if (ctx->dims.precision == GGB_FP64) {
    launch_angular_fp64(a, 0, g.x_d, g.y_d, 0, s);
    launch_radial_fp64(a, g.W_d, g.y_d, g.x_d, s);
    launch_angular_fp64(a, 1, g.x_d, g.x_d, 1, s);
  } else {
    mixed_step(g.mixed, a, s);
  }
  if (a.theta_tab) launch_theta_potentials(a, g.theta_args, g.x_d, s);
  launch_finalize(a, 1, s);
}

// n steps of every group.  With several groups, each group's steps go to its own stream, forked
// from and joined back to s by events (inside a graph capture this becomes parallel branches).
static int launch_steps(ggb_ctx* ctx, cudaStream_t s, int n) {
  if (n <= 0) return GGB_OK;
  if (ctx->groups.size() == 1) {
    for (int i = 0; i < n; ++i) launch_group_step(ctx, ctx->groups[0], s);
    return GGB_OK;
  }
  if (ctx->group_streams.empty()) {
    ctx->group_streams.assign(ctx->groups.size(), nullptr);
    ctx->group_done.assign(ctx->groups.size(), nullptr);
    for (size_t i = 0; i < ctx->groups.size(); ++i) {
      CK(cudaStreamCreateWithFlags(&ctx->group_streams[i], cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&ctx->group_done[i], cudaEventDisableTiming));
    }
    CK(cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming));
  }
  CK(cudaEventRecord(ctx->fork_ev, s));
  for (size_t gi = 0; gi < ctx->groups.size(); ++gi) {
    cudaStream_t gs = ctx->group_streams[gi];
    CK(cudaStreamWaitEvent(gs, ctx->fork_ev, 0));
    for (int i = 0; i < n; ++i) launch_group_step(ctx, ctx->groups[gi], gs);
    CK(cudaEventRecord(ctx->group_done[gi], gs));
    CK(cudaStreamWaitEvent(s, ctx->group_done[gi], 0));
  }
  return GGB_OK;
}

static int launch_init(ggb_ctx* ctx, GroupHost& g, cudaStream_t s) {
  const GroupArgs& a = g.args;
  if (ctx->dims.precision == GGB_FP64) {
    launch_angular_fp64(a, 2, g.x_d, g.x_d, 1, s);   // empty chain: partials of the initial orbitals
  } else {
    mixed_init(g.mixed, a, g.x_d, s);
  }
  launch_finalize(a, 0, s);
  if (a.theta_tab) launch_theta_potentials(a, g.theta_args, g.x_d, s);
  CK(cudaGetLastError());
  g.needs_init = false;
  return GGB_OK;
}

// ----------------------------------------------------------------------------------------------
// C ABI
// ----------------------------------------------------------------------------------------------
extern "C" {

const char* ggb_version(void) { return "ggbtddft-b200 0.2 (sm_100a)"; }

int ggb_create(const ggb_dims* dims, const ggb_group_desc* groups, const ggb_run_desc* runs, ggb_ctx** out) {
  if (!out) return GGB_ERR_ARG;
  *out = nullptr;
  if (!dims || !groups || !runs) return GGB_ERR_ARG;
  if (dims->n_groups <= 0 || dims->n_runs <= 0 || dims->n_t <= 0) return GGB_ERR_ARG;
  if (dims->precision < GGB_FP64 || dims->precision > GGB_SPLIT_INT8) return GGB_ERR_ARG;
  ggb_ctx* ctx = new ggb_ctx();
  ctx->dims = *dims;
  cudaGetDevice(&ctx->device);
  ctx->groups.resize(dims->n_groups);
  ctx->runs.resize(dims->n_runs);
  auto bad = [&](int code, const char* what) {
    ggb_destroy(ctx);
    (void)what;
    return code;
  };
  for (int i = 0; i < dims->n_groups; ++i) {
    GroupHost& g = ctx->groups[i];
    g.d = groups[i];
    if (g.d.n_r < 2 || g.d.n_r > MAX_NR || g.d.n_l < 2 || g.d.n_l > MAX_NL || g.d.n_m < 1 || g.d.n_m > g.d.n_l)
      return bad(GGB_ERR_ARG, "group dims");
    g.V.assign(4, std::vector<std::vector<double>>(g.d.n_m));
    g.D.assign(4, std::vector<std::vector<double>>(g.d.n_m));
    g.ang_set.assign(4, std::vector<bool>(g.d.n_m, false));
    // observables partials: one per CTA tile of radii.  The angular kernels take 32 radii per CTA
    // (each CTA streams the chain matrices once per product: fewer radii per CTA cost more of that
    // traffic than the extra CTAs gain, measured for the FP64 form), the int8 form 16 when N_l > 128
    // (two M tiles of channels)
    // radii per observables partial = the angular tile: 16 for the FP64 form and for the int8 form
    // with two channel tiles (N_l > 128), 32 otherwise
    g.obs_seg = (dims->precision == GGB_FP64 || (dims->precision == GGB_SPLIT_INT8 && g.d.n_l > 128)) ? 16 : TR;
    g.n_tiles = (g.d.n_r + g.obs_seg - 1) / g.obs_seg;
    g.ldS = ((g.d.n_l + 7) / 8) * 8;
  }
  for (int i = 0; i < dims->n_runs; ++i) {
    RunHost& r = ctx->runs[i];
    r.d = runs[i];
    if (r.d.group < 0 || r.d.group >= dims->n_groups || r.d.n_orb <= 0 || r.d.n_har < 0 || !(r.d.dt > 0.0))
      return bad(GGB_ERR_ARG, "run dims");
    GroupHost& g = ctx->groups[r.d.group];
    const int theta = (r.d.flags & GGB_RUN_THETA) ? 1 : 0;
    if (theta && dims->precision == GGB_SPLIT_BF16) return bad(GGB_ERR_ARG, "theta form with split_bf16");
    if (theta && r.d.n_har > 2 * groups[r.d.group].n_l - 1) return bad(GGB_ERR_ARG, "theta form: n_har > 2 l_max + 1");
    if (!g.runs.empty()) {
      if (g.n_har != r.d.n_har || g.use_hartree != r.d.use_hartree || (g.target_id > 0) != (r.d.target_id > 0) ||
          g.dt != r.d.dt || g.theta != theta)
        return bad(GGB_ERR_ARG, "runs of a group must share n_har, use_hartree, targetID>0, dt and the theta flag");
    } else {
      g.n_har = r.d.n_har; g.use_hartree = r.d.use_hartree; g.target_id = r.d.target_id; g.dt = r.d.dt;
      g.theta = theta;
    }
    r.col0 = g.n_cols;
    g.n_cols += r.d.n_orb;
    g.runs.push_back(i);
  }
  int rc;
  for (GroupHost& g : ctx->groups) {
    if (g.runs.empty()) return bad(GGB_ERR_ARG, "empty group");
    const size_t nr = g.d.n_r, nl = g.d.n_l, nc = g.n_cols;
    if ((rc = dalloc(ctx, &g.r_d, nr)) || (rc = dalloc(ctx, &g.drdx_d, nr)) || (rc = dalloc(ctx, &g.P_d, nr)) ||
        (rc = dalloc(ctx, &g.dens_d, nc * N_DEN * nr)) || (rc = dalloc(ctx, &g.obs_d, 2 * nc * nl * g.n_tiles)) ||
        (rc = dalloc(ctx, &g.step_d, 1)) || (rc = dalloc(ctx, &g.done_d, 1)) ||
        (rc = dalloc(ctx, &g.fin_cnt_d, g.runs.size())) || (rc = dalloc(ctx, &g.fin_scr_d, nc * FIN_OB * 8)) ||
        (rc = dalloc(ctx, &g.col_run_d, nc)) || (rc = dalloc(ctx, &g.col_m_d, nc)) ||
        (rc = dalloc(ctx, &g.col_occ_d, nc)) || (rc = dalloc(ctx, &g.runs_d, g.runs.size())))
      return bad(rc, "alloc");
    if (dims->precision == GGB_FP64 || dims->precision == GGB_SPLIT_INT8) {
      if ((rc = dalloc(ctx, &g.W_d, nl * nr * nr)) || (rc = dalloc(ctx, &g.x_d, nl * nc * nr)) ||
          (rc = dalloc(ctx, &g.y_d, nl * nc * nr)))
        return bad(rc, "alloc");
    } else {
      // the split forms convert W and the orbitals at set-up; FP64 staging copies are kept
      if ((rc = dalloc(ctx, &g.W_d, nl * nr * nr)) || (rc = dalloc(ctx, &g.x_d, nl * nc * nr)))
        return bad(rc, "alloc");
    }
    cudaMemcpy(g.runs_d, g.runs.data(), g.runs.size() * sizeof(int), cudaMemcpyHostToDevice);
  }
  for (RunHost& r : ctx->runs) {
    const GroupHost& g = ctx->groups[r.d.group];
    const size_t nr = g.d.n_r, nl = g.d.n_l, no = r.d.n_orb, nt = dims->n_t;
    if ((rc = dalloc(ctx, &r.E_d, nt)) || (rc = dalloc(ctx, &r.v_d, 4 * nr)) || (rc = dalloc(ctx, &r.v0_d, nr)) ||
        (rc = dalloc(ctx, &r.vexc_d, nr)) || (rc = dalloc(ctx, &r.vexc0_d, nr)) ||
        (rc = dalloc(ctx, &r.rho_frozen_d, nr)) || (rc = dalloc(ctx, &r.norm_d, no * nt)) ||
        (rc = dalloc(ctx, &r.norm0_d, no)) || (rc = dalloc(ctx, &r.dip_tot_d, no * nt)) ||
        (rc = dalloc(ctx, &r.acc_tot_d, no * nt)))
      return bad(rc, "alloc");
    if (dims->per_l)
      if ((rc = dalloc(ctx, &r.dip_d, nl * no * nt)) || (rc = dalloc(ctx, &r.acc_d, nl * no * nt)))
        return bad(rc, "alloc");
  }
  if ((rc = dalloc(ctx, &ctx->runs_dev, ctx->runs.size())) || (rc = dalloc(ctx, &ctx->status_d, 1)))
    return bad(rc, "alloc");
  *out = ctx;
  return GGB_OK;
}

int ggb_set_grid(ggb_ctx* ctx, int group, const double* r, const double* drdx, const double* P, int n_r) {
  if (!ctx) return GGB_ERR_ARG;
  if (group < 0 || group >= (int)ctx->groups.size()) return fail(ctx, GGB_ERR_ARG, "bad group %d", group);
  GroupHost& g = ctx->groups[group];
  if (n_r != g.d.n_r || !r || !drdx || !P) return fail(ctx, GGB_ERR_ARG, "grid size %d != %d", n_r, g.d.n_r);
  g.r.assign(n_r, 0.0);
  CK(cudaMemcpy(g.r.data(), r, n_r * sizeof(double), cudaMemcpyDefault));
  for (int i = 0; i < n_r; ++i)
    if (!(g.r[i] > 0.0)) return fail(ctx, GGB_ERR_ARG, "r[%d] = %g must be > 0", i, g.r[i]);
  for (int i = 1; i < n_r; ++i)
    if (!(g.r[i] > g.r[i - 1])) return fail(ctx, GGB_ERR_ARG, "r must increase (r[%d] <= r[%d])", i, i - 1);
  CK(cudaMemcpy(g.r_d, r, n_r * sizeof(double), cudaMemcpyDefault));
  CK(cudaMemcpy(g.drdx_d, drdx, n_r * sizeof(double), cudaMemcpyDefault));
  CK(cudaMemcpy(g.P_d, P, n_r * sizeof(double), cudaMemcpyDefault));
  g.grid_set = true;
  return GGB_OK;
}

int ggb_set_radial_propagators(ggb_ctx* ctx, int group, const double* W) {
  if (!ctx) return GGB_ERR_ARG;
  if (group < 0 || group >= (int)ctx->groups.size() || !W) return fail(ctx, GGB_ERR_ARG, "bad group/pointer");
  GroupHost& g = ctx->groups[group];
  const size_t n = (size_t)g.d.n_l * g.d.n_r * g.d.n_r;
  CK(cudaMemcpy(g.W_d, W, n * sizeof(double2), cudaMemcpyDefault));
  g.w_set = true;
  ctx->prepared = ctx->prepared && ctx->dims.precision == GGB_FP64;
  return GGB_OK;
}

int ggb_set_angular(ggb_ctx* ctx, int group, int coupling, int m, const double* V, const double* D) {
  if (!ctx) return GGB_ERR_ARG;
  if (group < 0 || group >= (int)ctx->groups.size()) return fail(ctx, GGB_ERR_ARG, "bad group %d", group);
  GroupHost& g = ctx->groups[group];
  if (coupling < 0 || coupling > 3 || m < 0 || m >= g.d.n_m || !V || !D)
    return fail(ctx, GGB_ERR_ARG, "bad coupling %d / m %d", coupling, m);
  if (ctx->prepared) return fail(ctx, GGB_ERR_STATE, "angular data must be set before the first step");
  const int n_l = g.d.n_l;
  g.V[coupling][m].resize((size_t)n_l * n_l);
  g.D[coupling][m].resize(n_l);
  CK(cudaMemcpy(g.V[coupling][m].data(), V, (size_t)n_l * n_l * sizeof(double), cudaMemcpyDefault));
  CK(cudaMemcpy(g.D[coupling][m].data(), D, (size_t)n_l * sizeof(double), cudaMemcpyDefault));
  g.ang_set[coupling][m] = true;
  return GGB_OK;
}

int ggb_set_orbitals(ggb_ctx* ctx, int run, const double* x, const int* l, const int* m, const int* occ,
                     const double* rho_frozen) {
  if (!ctx) return GGB_ERR_ARG;
  if (run < 0 || run >= (int)ctx->runs.size() || !x || !l || !m || !occ || !rho_frozen)
    return fail(ctx, GGB_ERR_ARG, "bad run/pointer");
  RunHost& r = ctx->runs[run];
  GroupHost& g = ctx->groups[r.d.group];
  const int no = r.d.n_orb, nr = g.d.n_r, nl = g.d.n_l;
  r.l.assign(no, 0); r.m.assign(no, 0); r.occ.assign(no, 0);
  CK(cudaMemcpy(r.l.data(), l, no * sizeof(int), cudaMemcpyDefault));
  CK(cudaMemcpy(r.m.data(), m, no * sizeof(int), cudaMemcpyDefault));
  CK(cudaMemcpy(r.occ.data(), occ, no * sizeof(int), cudaMemcpyDefault));
  for (int k = 0; k < no; ++k)
    if (r.m[k] < 0 || r.m[k] >= g.d.n_m || r.l[k] < r.m[k] || r.l[k] >= nl)
      return fail(ctx, GGB_ERR_ARG, "orbital %d: l=%d m=%d outside 0<=m<N_m, m<=l<N_l", k, r.l[k], r.m[k]);
  CK(cudaMemcpy(g.col_m_d + r.col0, r.m.data(), no * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(g.col_occ_d + r.col0, r.occ.data(), no * sizeof(int), cudaMemcpyHostToDevice));
  std::vector<int> cr(no, run);
  CK(cudaMemcpy(g.col_run_d + r.col0, cr.data(), no * sizeof(int), cudaMemcpyHostToDevice));
  // x[l][kso][r] -> group x[l][col0 + kso][r]
  CK(cudaMemcpy2D(g.x_d + (size_t)r.col0 * nr, (size_t)g.n_cols * nr * sizeof(double2), x,
                  (size_t)no * nr * sizeof(double2), (size_t)no * nr * sizeof(double2), nl, cudaMemcpyDefault));
  CK(cudaMemcpy(r.rho_frozen_d, rho_frozen, nr * sizeof(double), cudaMemcpyDefault));
  CK(cudaMemset(r.v_d, 0, 4 * (size_t)nr * sizeof(double)));
  CK(cudaMemset(r.v0_d, 0, nr * sizeof(double)));
  CK(cudaMemset(r.vexc_d, 0, nr * sizeof(double)));
  CK(cudaMemset(r.vexc0_d, 0, nr * sizeof(double)));
  CK(cudaMemset(g.step_d, 0, sizeof(int)));
  CK(cudaMemset(g.done_d, 0, sizeof(unsigned)));
  CK(cudaMemset(g.fin_cnt_d, 0, g.runs.size() * sizeof(unsigned)));
  r.orb_set = true;
  g.needs_init = true;
  if (ctx->dims.precision != GGB_FP64 && ctx->prepared) {
    int rc = mixed_load_orbitals(g.mixed, g.args, g.x_d);
    if (rc) return fail(ctx, rc, "orbital conversion failed");
  }
  return GGB_OK;
}

int ggb_set_field(ggb_ctx* ctx, int run, const double* E, int n_t) {
  if (!ctx) return GGB_ERR_ARG;
  if (run < 0 || run >= (int)ctx->runs.size() || !E) return fail(ctx, GGB_ERR_ARG, "bad run/pointer");
  if (n_t <= 0 || n_t > ctx->dims.n_t) return fail(ctx, GGB_ERR_ARG, "n_t %d outside 1..%d", n_t, ctx->dims.n_t);
  RunHost& r = ctx->runs[run];
  CK(cudaMemcpy(r.E_d, E, n_t * sizeof(double), cudaMemcpyDefault));
  r.field_set = true;
  return GGB_OK;
}

int ggb_step(ggb_ctx* ctx, int n_steps, void* stream) {
  if (!ctx) return GGB_ERR_ARG;
  if (n_steps < 0) return fail(ctx, GGB_ERR_ARG, "n_steps < 0");
  cudaStream_t s = (cudaStream_t)stream;
  const bool was_prepared = ctx->prepared;
  int rc = prepare(ctx);
  if (rc) return rc;
  if (!was_prepared && ctx->dims.precision != GGB_FP64)
    for (GroupHost& g : ctx->groups)
      if ((rc = mixed_load_orbitals(g.mixed, g.args, g.x_d))) return fail(ctx, rc, "orbital conversion failed");
  for (GroupHost& g : ctx->groups)
    if (g.needs_init)
      if ((rc = launch_init(ctx, g, s))) return rc;
  const int G = ctx->graph_steps;
  if (!ctx->graph_exec) {
    // capture once, on the first call, so that later calls only replay
    if (!ctx->cap_stream) CK(cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking));
    for (int k = 0; k < 2; ++k) {
      cudaGraph_t graph;
      CK(cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal));
      const int rc_cap = launch_steps(ctx, ctx->cap_stream, k == 0 ? G : 1);
      CK(cudaStreamEndCapture(ctx->cap_stream, &graph));
      if (rc_cap) {
        cudaGraphDestroy(graph);
        return rc_cap;
      }
      CK(cudaGraphInstantiate(k == 0 ? &ctx->graph_exec : &ctx->graph1_exec, graph, 0));
      cudaGraphDestroy(graph);
    }
  }
  if (n_steps == 0) return GGB_OK;
  for (int i = 0; i + G <= n_steps; i += G) CK(cudaGraphLaunch(ctx->graph_exec, s));
  for (int i = 0; i < n_steps % G; ++i) CK(cudaGraphLaunch(ctx->graph1_exec, s));
  CK(cudaGetLastError());
  return GGB_OK;
}

int ggb_set_tuning(ggb_ctx* ctx, int group, int radial_bn, int radial_stages) {
  if (!ctx) return GGB_ERR_ARG;
  if (group < 0 || group >= (int)ctx->groups.size()) return fail(ctx, GGB_ERR_ARG, "group %d out of range", group);
  if (ctx->dims.precision != GGB_SPLIT_INT8)
    return fail(ctx, GGB_ERR_STATE, "ggb_set_tuning applies to the split_int8 form only");
  if (ctx->prepared) return fail(ctx, GGB_ERR_STATE, "ggb_set_tuning after the first ggb_step");
  if (radial_bn != 0 && radial_bn != 16 && radial_bn != 32 && radial_bn != 64)
    return fail(ctx, GGB_ERR_ARG, "radial_bn %d is not 0, 16, 32 or 64", radial_bn);
  if (radial_stages != 0 && (radial_stages < 2 || radial_stages > 8))
    return fail(ctx, GGB_ERR_ARG, "radial_stages %d outside 2..8", radial_stages);
  ctx->groups[group].mixed.i8.tune_bn = radial_bn;
  ctx->groups[group].mixed.i8.tune_stages = radial_stages;
  return GGB_OK;
}

int ggb_set_angular_fp64(ggb_ctx* ctx, int group, int on) {
  if (!ctx) return GGB_ERR_ARG;
  if (group < 0 || group >= (int)ctx->groups.size()) return fail(ctx, GGB_ERR_ARG, "group %d out of range", group);
  if (ctx->dims.precision != GGB_SPLIT_INT8)
    return fail(ctx, GGB_ERR_STATE, "ggb_set_angular_fp64 applies to the split_int8 form only");
  if (ctx->prepared) return fail(ctx, GGB_ERR_STATE, "ggb_set_angular_fp64 after the first ggb_step");
  ctx->groups[group].mixed.angular_fp64 = on != 0;
  return GGB_OK;
}

int ggb_set_theta_reuse(ggb_ctx* ctx, int group, int on) {
  if (!ctx) return GGB_ERR_ARG;
  if (group < 0 || group >= (int)ctx->groups.size()) return fail(ctx, GGB_ERR_ARG, "group %d out of range", group);
  if (ctx->dims.precision != GGB_SPLIT_INT8)
    return fail(ctx, GGB_ERR_STATE, "ggb_set_theta_reuse applies to the split_int8 form only");
  if (ctx->prepared) return fail(ctx, GGB_ERR_STATE, "ggb_set_theta_reuse after the first ggb_step");
  ctx->groups[group].mixed.i8.theta_reuse = on != 0;
  return GGB_OK;
}

int ggb_launch_phase(ggb_ctx* ctx, int phase, void* stream) {
  if (!ctx) return GGB_ERR_ARG;
  if (phase < 0 || phase > 3) return fail(ctx, GGB_ERR_ARG, "phase %d outside 0..3", phase);
  if (!ctx->prepared) return fail(ctx, GGB_ERR_STATE, "ggb_launch_phase before the first ggb_step");
  cudaStream_t s = (cudaStream_t)stream;
  for (GroupHost& g : ctx->groups) {
    const GroupArgs& a = g.args;
    if (ctx->dims.precision == GGB_FP64) {
      if (phase == 0) launch_angular_fp64(a, 0, g.x_d, g.y_d, 0, s);
      if (phase == 1) launch_radial_fp64(a, g.W_d, g.y_d, g.x_d, s);
      if (phase == 2) launch_angular_fp64(a, 1, g.x_d, g.x_d, 1, s);
    } else {
      mixed_phase(g.mixed, a, phase, s);
    }
    if (phase == 3) {
      if (a.theta_tab) launch_theta_potentials(a, g.theta_args, g.x_d, s);
      launch_finalize(a, 2, s);
    }
  }
  CK(cudaGetLastError());
  return GGB_OK;
}

int ggb_get_step(ggb_ctx* ctx, int* step) {
  if (!ctx || !step) return GGB_ERR_ARG;
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(step, ctx->groups[0].step_d, sizeof(int), cudaMemcpyDeviceToHost));
  return GGB_OK;
}

int ggb_get_observables(ggb_ctx* ctx, int run, double* dip, double* acc, double* norm, int per_l, int n_steps) {
  if (!ctx) return GGB_ERR_ARG;
  if (run < 0 || run >= (int)ctx->runs.size()) return fail(ctx, GGB_ERR_ARG, "bad run %d", run);
  if (n_steps < 0 || n_steps > ctx->dims.n_t) return fail(ctx, GGB_ERR_ARG, "n_steps %d outside 0..n_t", n_steps);
  if (per_l && !ctx->dims.per_l) return fail(ctx, GGB_ERR_ARG, "per-l observables were not requested at create");
  RunHost& r = ctx->runs[run];
  const int nl = ctx->groups[r.d.group].d.n_l, no = r.d.n_orb, nt = ctx->dims.n_t;
  CK(cudaDeviceSynchronize());
  const size_t row = (size_t)n_steps * sizeof(double2);
  if (per_l) {
    if (dip) CK(cudaMemcpy2D(dip, row, r.dip_d, (size_t)nt * sizeof(double2), row, (size_t)nl * no, cudaMemcpyDefault));
    if (acc) CK(cudaMemcpy2D(acc, row, r.acc_d, (size_t)nt * sizeof(double2), row, (size_t)nl * no, cudaMemcpyDefault));
  } else {
    if (dip) CK(cudaMemcpy2D(dip, row, r.dip_tot_d, (size_t)nt * sizeof(double2), row, no, cudaMemcpyDefault));
    if (acc) CK(cudaMemcpy2D(acc, row, r.acc_tot_d, (size_t)nt * sizeof(double2), row, no, cudaMemcpyDefault));
  }
  if (norm)
    CK(cudaMemcpy2D(norm, (size_t)n_steps * sizeof(double), r.norm_d, (size_t)nt * sizeof(double),
                    (size_t)n_steps * sizeof(double), no, cudaMemcpyDefault));
  return GGB_OK;
}

int ggb_get_orbitals(ggb_ctx* ctx, int run, double* x) {
  if (!ctx) return GGB_ERR_ARG;
  if (run < 0 || run >= (int)ctx->runs.size() || !x) return fail(ctx, GGB_ERR_ARG, "bad run/pointer");
  RunHost& r = ctx->runs[run];
  GroupHost& g = ctx->groups[r.d.group];
  const int no = r.d.n_orb, nr = g.d.n_r, nl = g.d.n_l;
  CK(cudaDeviceSynchronize());
  if (ctx->dims.precision != GGB_FP64 && ctx->prepared) {
    int rc = mixed_store_orbitals(g.mixed, g.args, g.x_d);
    if (rc) return fail(ctx, rc, "orbital conversion failed");
    CK(cudaDeviceSynchronize());
  }
  CK(cudaMemcpy2D(x, (size_t)no * nr * sizeof(double2), g.x_d + (size_t)r.col0 * nr,
                  (size_t)g.n_cols * nr * sizeof(double2), (size_t)no * nr * sizeof(double2), nl, cudaMemcpyDefault));
  return GGB_OK;
}

int ggb_get_potentials(ggb_ctx* ctx, int run, double* v, double* v0, double* vexc, double* vexc0) {
  if (!ctx) return GGB_ERR_ARG;
  if (run < 0 || run >= (int)ctx->runs.size()) return fail(ctx, GGB_ERR_ARG, "bad run %d", run);
  RunHost& r = ctx->runs[run];
  const int nr = ctx->groups[r.d.group].d.n_r;
  CK(cudaDeviceSynchronize());
  if (v) CK(cudaMemcpy(v, r.v_d, 4 * (size_t)nr * sizeof(double), cudaMemcpyDefault));
  const GroupHost& g = ctx->groups[r.d.group];
  if (v && g.args.theta_tab) {
    // the theta form with n_har > 4 keeps its multipoles L >= 1 in the exact-quadrature buffers
    const int ri = (int)(std::find(g.runs.begin(), g.runs.end(), run) - g.runs.begin());
    const int rows = std::min(g.theta_args.n_mp, 4) - 1;
    if (rows > 0)
      CK(cudaMemcpy(v + nr, g.theta_args.vmp + ((size_t)ri * g.theta_args.n_mp + 1) * nr, (size_t)rows * nr * sizeof(double),
                    cudaMemcpyDefault));
  }
  if (v0) CK(cudaMemcpy(v0, r.v0_d, nr * sizeof(double), cudaMemcpyDefault));
  if (vexc) CK(cudaMemcpy(vexc, r.vexc_d, nr * sizeof(double), cudaMemcpyDefault));
  if (vexc0) CK(cudaMemcpy(vexc0, r.vexc0_d, nr * sizeof(double), cudaMemcpyDefault));
  return GGB_OK;
}

int ggb_status(ggb_ctx* ctx, char* msg, int len) {
  if (!ctx) return GGB_ERR_ARG;
  unsigned st = 0;
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(&st, ctx->status_d, sizeof(unsigned), cudaMemcpyDeviceToHost);
  std::string m = ctx->err;
  if (e != cudaSuccess) m = std::string("CUDA error: ") + cudaGetErrorString(e);
  if (st & ST_NAN) m += (m.empty() ? "" : "; ") + std::string("NaN/Inf in observables");
  if (st & ST_STEP_OVERFLOW) m += (m.empty() ? "" : "; ") + std::string("step beyond the field length n_t");
  if (st & ST_NORM_GROWTH) m += (m.empty() ? "" : "; ") + std::string("orbital norm grew above its initial value");
  if (msg && len > 0) {
    strncpy(msg, m.c_str(), len - 1);
    msg[len - 1] = 0;
  }
  if (e != cudaSuccess) return GGB_ERR_CUDA;
  return (int)st;
}

void ggb_destroy(ggb_ctx* ctx) {
  if (!ctx) return;
  cudaDeviceSynchronize();
  if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
  if (ctx->graph1_exec) cudaGraphExecDestroy(ctx->graph1_exec);
  if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
  for (cudaStream_t gs : ctx->group_streams) cudaStreamDestroy(gs);
  for (cudaEvent_t e : ctx->group_done) cudaEventDestroy(e);
  if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
  for (GroupHost& g : ctx->groups) mixed_release(g.mixed);
  for (void* p : ctx->allocs) cudaFree(p);
  delete ctx;
}

}  // extern "C"
