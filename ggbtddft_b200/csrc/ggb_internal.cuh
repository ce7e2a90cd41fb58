// Internal device-side data structures and helpers of libggbtddft.
//
// Layout in HBM (per grid group g: runs that share N_r, N_l, the grid and W_l):
//   x, y     [N_l][n_cols][N_r]  orbitals; column = one orbital of one run of the group.
//            FP64 form: double2.  Split forms: float2.  For a single run this is the reference's
//            d_x[l][kso*N_r + r] (main.cu:356-369) without the pointer-array indirection.
//   W        radial propagators, FP64 form: double2 [N_l][N_r][N_r] = propagatorL%03d.bin.
//   mats     angular chain matrices, [n_mats][N_m][N_l][ldS] doubles, stored so that the kernel's
//            product is y[j] = sum_l S[l][j] x[l]  (S = A^T of the left multiplier A).
//   dph      angular eigenvalues D[c][m][j], [4][N_m][ldS].
//   coef     angular coefficient tables [COEF_N][N_m][N_l] (cu, cd, p, qu, qd, p3lm, f3lm).
//   dens     density partials per column [n_cols][4][N_r] (not yet occupation weighted).
//   obs      dipole/acceleration partials per column, l and r-tile [n_cols][N_l][n_tiles][2] double4
//            (double-double: high parts, then low parts).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ggb {

constexpr int TR = 32;            // radii per angular tile (one warp-width, coalesced along r)
constexpr int ANG_WARPS = 8;      // warps per angular CTA
constexpr int MAX_NL = 220;       // largest N_l: two [N_l][32] complex128 tiles fit in 227 KB of shared memory
constexpr int MAX_NR = 8192;      // largest N_r: three [N_r] FP64 rows of the potentials kernel
constexpr int FIN_OB = 32;         // observables blocks per run in k_finalize (slices of l)
constexpr int N_DEN = 4;          // density multipoles carried per column (L = 0..3)

// status bits (sticky, OR-ed on the device)
constexpr unsigned ST_NAN = 1u;
constexpr unsigned ST_STEP_OVERFLOW = 2u;
constexpr unsigned ST_NORM_GROWTH = 4u;

// PH_THETA: the theta form's one phase at the P coupling's nodes x_j,
//   (r E + v_1) x_j + v_2 P_2(x_j) + v_3 P_3(x_j) + (v_0 - v_0(t=0)) + (vxc - vxc(t=0))
enum PhaseKind { PH_NONE = 0, PH_P = 1, PH_FP = 2, PH_D = 3, PH_FF = 4, PH_THETA = 5 };
constexpr int RUN_FLAG_PW92 = 1;
constexpr int RUN_FLAG_THETA = 2;
constexpr int RUN_FLAG_XC_FROZEN = 4;

// P_2 and P_3 of the theta phase
__host__ __device__ __forceinline__ double legendre_p2(double x) { return 0.5 * (3.0 * x * x - 1.0); }
__host__ __device__ __forceinline__ double legendre_p3(double x) { return 0.5 * x * (5.0 * x * x - 3.0); }
enum Coef { CF_CU = 0, CF_CD = 1, CF_P = 2, CF_QU = 3, CF_QD = 4, CF_P3 = 5, CF_F3 = 6, COEF_N = 7 };

struct ChainOp {
  int mat;    // chain matrix index
  int phase;  // PhaseKind applied to this product's outputs
  int coupling;  // which eigenvalue set the phase uses (0..3)
};

// One half-step program: [S] (A_0, phase_0) (A_1, phase_1) ... (A_k) [S]
struct Chain {
  int n_ops;
  int pre_s;
  int post_s;
  ChainOp ops[9];
};

struct RunDev {
  const double* E;        // [n_t]
  double* v;              // [4][N_r] Hartree multipoles (real part of the reference's d_v)
  double* v0;             // [N_r]   t = 0 monopole
  double* vexc;           // [N_r]
  double* vexc0;          // [N_r]
  const double* rho_frozen;  // [N_r]
  double2* dip;           // per_l: [N_l][n_orb][n_t]
  double2* acc;
  double2* dip_tot;       // [n_orb][n_t]
  double2* acc_tot;
  double* norm;           // [n_orb][n_t]
  double* norm0;          // [n_orb] norm at t = 0 (for the growth watchdog)
  double* htab;           // theta form with n_har > 4: sum_{L>=1} v_L(r) P_L(x_j^m), [N_m][N_l][N_r]
  int col0;
  int n_orb;
  int n_t;
  int flags;
};

struct GroupArgs {
  int n_r, n_l, n_m, n_cols, n_tiles, ldS, n_runs;
  int theta;        // theta form (GGB_RUN_THETA): one phase per half-step at the P nodes
  int theta_tab;    // theta form with n_har > 4: the multipoles L >= 1 come from run.htab
  int hartree_on;   // USE_HARTREE == 1 && targetID > 0
  int p_hartree;    // P phase carries v_1 (USE_HARTREE && N_har > 1 && targetID > 0)
  int n_den;        // multipoles computed: min(N_har, 4) when hartree_on, else 0
  int per_l;
  double dt;
  double n_g_fac;   // N_g (N_g + 1) / 2
  double norm_tol;
  int obs_seg;      // radii per observables partial sum (32; 16 for the int8 form when N_l > 128)  // relative growth of an orbital norm above its initial value that raises ST_NORM_GROWTH
  const double* r;
  const double* drdx;
  const double* P;
  const double* mats;
  const double* dph;
  const double* coef;
  const int* col_run;   // [n_cols] run index within ctx
  const int* col_m;
  const int* col_occ;
  const int* runs_of_group;  // [n_runs] ctx run indices
  RunDev* runs;             // ctx-wide device array
  double* dens;
  double4* obs;
  int* step;                // ctx-wide step counter
  unsigned* status;
  unsigned* done;           // block counter for the last-block step increment
  unsigned* fin_cnt;        // [n_runs] finished observables blocks of the step (last-block totals)
  double* fin_scr;          // [n_cols][FIN_OB][8] slice totals of the observables (double-double)
  Chain chain[3];   // first half, second half, empty (initial partials)
};

// Exact multipoles L = 0 .. n_mp-1 of the theta form with n_har > 4 (ggb_theta.cu).  Fine
// Gauss-Legendre quadrature on 2 N_l nodes +-x_q (q < nq = N_l, x_q > 0), using the parity of the
// normalised associated Legendre functions Theta_l^m(-x) = (-1)^(l-m) Theta_l^m(x).
struct ThetaArgs {
  int n_mp;            // multipoles L = 0 .. n_mp-1 (<= 2 N_l - 1)
  int nq;              // positive fine nodes (= N_l)
  const double* T;     // [N_m][nq][N_l]  Theta_l^m(x_q)
  const double* wP;    // [n_mp][nq]      w_q P_L(x_q)
  const double* PLj;   // [N_m][n_mp][ldS] P_L(x_j^m) at the P coupling's nodes
  const double* rq;    // [n_mp+1][N_r]   (r_(a-1) / r_a)^L for a >= 1, 0 at a = 0
  double* fine;        // [n_runs][2][nq][N_r]  S_q = sum occ 2(|E|^2 + |O|^2), D_q = sum occ 4 Re(E conj O)
  double* rho;         // [n_runs][n_mp][N_r]
  double* vmp;         // [n_runs][n_mp][N_r]
};
void launch_theta_potentials(const GroupArgs& g, const ThetaArgs& t, const double2* x, cudaStream_t s);

__device__ __forceinline__ double2 cmul_conj_phase(double2 x, double eta) {
  // x * exp(-i eta) written as the reference's phase kernels do (couplingP.cuh:99-102)
  double s, c;
  sincos(eta, &s, &c);
  return make_double2(c * x.x + s * x.y, c * x.y - s * x.x);
}

// Double-double accumulation (Knuth TwoSum): used for the compensated Hartree prefix sums.
struct dd {
  double hi, lo;
};
__device__ __forceinline__ dd dd_add(dd a, dd b) {
  double s = a.hi + b.hi;
  double bp = s - a.hi;
  double e = (a.hi - (s - bp)) + (b.hi - bp);
  e += a.lo + b.lo;
  double h = s + e;
  return dd{h, e - (h - s)};
}
__device__ __forceinline__ dd dd_shfl_up(dd a, int d) {
  return dd{__shfl_up_sync(0xffffffffu, a.hi, d), __shfl_up_sync(0xffffffffu, a.lo, d)};
}

// launchers (ggb_kernels_fp64.cu)
void launch_angular_fp64(const GroupArgs& g, int half, const double2* xin, double2* xout, int do_obs,
                         cudaStream_t s);
void launch_radial_fp64(const GroupArgs& g, const double2* W, const double2* xin, double2* xout,
                        cudaStream_t s);
void launch_finalize(const GroupArgs& g, int mode, cudaStream_t s);
size_t angular_smem_fp64(int n_l);
cudaError_t configure_kernels_fp64(int n_l_max, int n_r_max);
cudaError_t set_max_dynamic_smem(const void* fn, int optin);

}  // namespace ggb
