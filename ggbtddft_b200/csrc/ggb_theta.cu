// Hartree potential of the theta form from every multipole L = 0 .. 2 l_max (GGB_RUN_THETA with
// n_har > 4; not in the reference, whose density multipoles stop at L = 3,
// hartreePotentialDensity.cuh:1-181, and whose Hartree sum is the O(N_r^2) loop of
// h_calculateHartreePotential.cuh:1-56).
//
// Per run and step, from the orbitals x[l][col][r] at the end of the step:
//  k_theta_fine     the density on a Gauss-Legendre grid of 2 N_l nodes +-x_q, exact for every
//                   multipole up to 2 l_max: per orbital f(+-x_q) = E_q +- O_q with E (O) the sum over
//                   l - m even (odd) of x_l Theta_l^m(x_q); summed over the run's orbitals,
//                   S_q = sum occ 2 (|E|^2 + |O|^2) = rho(x_q) + rho(-x_q) and
//                   D_q = sum occ 4 Re(E conj O)  = rho(x_q) - rho(-x_q).
//  k_theta_project  rho_L(r) = sum_q w_q P_L(x_q) (S_q for even L, D_q for odd L).
//  k_theta_hartree  v_L(r_a) = sum_b rho_L(b) r_<^L / r_>^(L+1) as two linear recurrences with ratios
//                   of radii (no power of r over- or underflows):
//                     A_a = (r_(a-1)/r_a)^L A_(a-1) + rho_a,  B_a = (r_a/r_(a+1))^(L+1) (B_(a+1) + rho_(a+1)),
//                     v_L(r_a) = (A_a + B_a) / r_a,
//                   each evaluated by a warp: sequential over a chunk of radii per lane, then a warp
//                   scan of the chunks' affine maps.
//  k_theta_table    htab[m][j][r] = sum_{L>=1} v_L(r) P_L(x_j^m): the multipoles' potential at the
//                   nodes of the angular phase (the monopole and exchange changes come from k_finalize
//                   and enter the phase as in the theta form with n_har <= 4).
#include <cuda_runtime.h>

#include "ggb_internal.cuh"

namespace ggb {

constexpr int TH_THREADS = 256;
constexpr int TH_WARPS = TH_THREADS / 32;
constexpr int TH_QB = 2;          // fine nodes per warp
constexpr int TH_ILP = 8;         // independent partial sums of the projection and table loops

// pairwise sum of the partial sums
__device__ __forceinline__ double sum_partials(const double (&a)[TH_ILP]) {
  return ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
}

// Work split of the three density/potential kernels: a warp owns 32 radii and a few fine nodes
// (k_theta_fine), one multipole (k_theta_project) or one node of the phase (k_theta_table), so that
// a single run (the helium configuration: 13 tiles of 32 radii) still spreads over ~100 blocks; the
// radii are the lanes, so every load of an orbital, a density or a potential row is coalesced.

// blocks (run, 32 radii, TH_WARPS * TH_QB fine nodes): S and D of the run's orbitals at the block's
// positive fine nodes, accumulated over the run's orbitals in order in registers
__global__ void __launch_bounds__(TH_THREADS) k_theta_fine(GroupArgs g, ThetaArgs t, const double2* __restrict__ x) {
  const int tiles = (g.n_r + 31) / 32;
  const int nq = t.nq, n_l = g.n_l;
  const int qsplit = (nq + TH_WARPS * TH_QB - 1) / (TH_WARPS * TH_QB);
  const int ri = blockIdx.x / (tiles * qsplit);
  const int rest = blockIdx.x - ri * tiles * qsplit;
  const int tile = rest / qsplit, qs = rest - tile * qsplit;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r = tile * 32 + lane;
  const int q0 = (qs * TH_WARPS + warp) * TH_QB;
  if (r >= g.n_r || q0 >= nq) return;
  const RunDev run = g.runs[g.runs_of_group[ri]];
  double S[TH_QB], D[TH_QB];
#pragma unroll
  for (int u = 0; u < TH_QB; ++u) S[u] = D[u] = 0.0;
  for (int k = 0; k < run.n_orb; ++k) {
    const int col = run.col0 + k;
    const int m = g.col_m[col];
    const double occ = (double)g.col_occ[col];
    const double* Tm = t.T + (size_t)m * nq * n_l;
    double2 e[TH_QB], o[TH_QB];
#pragma unroll
    for (int u = 0; u < TH_QB; ++u) e[u] = o[u] = make_double2(0.0, 0.0);
    for (int l = m; l < n_l; ++l) {
      const double2 xv = x[((size_t)l * g.n_cols + col) * g.n_r + r];
      const bool odd = ((l - m) & 1) != 0;
#pragma unroll
      for (int u = 0; u < TH_QB; ++u) {
        const int q = q0 + u;
        const double tv = q < nq ? __ldg(Tm + (size_t)q * n_l + l) : 0.0;
        if (odd) {
          o[u].x = fma(tv, xv.x, o[u].x);
          o[u].y = fma(tv, xv.y, o[u].y);
        } else {
          e[u].x = fma(tv, xv.x, e[u].x);
          e[u].y = fma(tv, xv.y, e[u].y);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < TH_QB; ++u) {
      S[u] += occ * 2.0 * (e[u].x * e[u].x + e[u].y * e[u].y + o[u].x * o[u].x + o[u].y * o[u].y);
      D[u] += occ * 4.0 * (e[u].x * o[u].x + e[u].y * o[u].y);
    }
  }
  double* f = t.fine + (size_t)ri * 2 * nq * g.n_r;
#pragma unroll
  for (int u = 0; u < TH_QB; ++u) {
    const int q = q0 + u;
    if (q < nq) {
      f[(size_t)q * g.n_r + r] = S[u];
      f[((size_t)nq + q) * g.n_r + r] = D[u];
    }
  }
}

// blocks (run, 32 radii, TH_WARPS multipoles): rho_L(r) for the warp's L, TH_ILP partial sums over
// the fine nodes
__global__ void __launch_bounds__(TH_THREADS) k_theta_project(GroupArgs g, ThetaArgs t) {
  const int tiles = (g.n_r + 31) / 32;
  const int lsplit = (t.n_mp + TH_WARPS - 1) / TH_WARPS;
  const int ri = blockIdx.x / (tiles * lsplit);
  const int rest = blockIdx.x - ri * tiles * lsplit;
  const int tile = rest / lsplit, ls = rest - tile * lsplit;
  const int r = tile * 32 + (threadIdx.x & 31);
  const int L = ls * TH_WARPS + (threadIdx.x >> 5);
  if (r >= g.n_r || L >= t.n_mp) return;
  const int nq = t.nq, n_r = g.n_r;
  const double* src = t.fine + ((size_t)ri * 2 + (L & 1)) * nq * n_r + r;
  const double* w = t.wP + (size_t)L * nq;
  double acc[TH_ILP];
#pragma unroll
  for (int u = 0; u < TH_ILP; ++u) acc[u] = 0.0;
  int q = 0;
  for (; q + TH_ILP - 1 < nq; q += TH_ILP)
#pragma unroll
    for (int u = 0; u < TH_ILP; ++u) acc[u] = fma(__ldg(w + q + u), src[(size_t)(q + u) * n_r], acc[u]);
  for (; q < nq; ++q) acc[0] = fma(__ldg(w + q), src[(size_t)q * n_r], acc[0]);
  t.rho[((size_t)ri * t.n_mp + L) * n_r + r] = sum_partials(acc);
}

// affine map a -> mul a + add, composed in the order of the recurrence
struct Aff {
  double mul, add;
};
__device__ __forceinline__ Aff aff_then(Aff first, Aff second) {
  return Aff{second.mul * first.mul, fma(second.mul, first.add, second.add)};
}

// one warp per (run, L >= 1)
__global__ void __launch_bounds__(TH_THREADS) k_theta_hartree(GroupArgs g, ThetaArgs t) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int per_run = (t.n_mp - 1 + TH_WARPS - 1) / TH_WARPS;
  const int ri = blockIdx.x / per_run;
  const int L = 1 + (blockIdx.x - ri * per_run) * TH_WARPS + warp;
  if (L >= t.n_mp) return;
  const int n = g.n_r;
  const double* rho = t.rho + ((size_t)ri * t.n_mp + L) * n;
  double* v = t.vmp + ((size_t)ri * t.n_mp + L) * n;
  const int C = (n + 31) / 32;
  const int a0 = lane * C, a1 = min(n, a0 + C);
  // forward: A_a = f_a A_(a-1) + rho_a, f_a = (r_(a-1)/r_a)^L (the grid's table), f_0 = 0
  const double* fL = t.rq + (size_t)L * n;
  const double* gL = t.rq + (size_t)(L + 1) * n;
  Aff mine{1.0, 0.0};
  for (int a = a0; a < a1; ++a) {
    const double f = a == 0 ? 0.0 : fL[a];
    mine = Aff{f * mine.mul, fma(f, mine.add, rho[a])};
  }
  Aff inc = mine;                       // inclusive scan of the lanes' maps, in lane order
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const Aff o{__shfl_up_sync(0xffffffffu, inc.mul, d), __shfl_up_sync(0xffffffffu, inc.add, d)};
    if (lane >= d) inc = aff_then(o, inc);
  }
  double A = __shfl_up_sync(0xffffffffu, inc.add, 1);   // A_(a0 - 1): the previous lanes' maps applied to 0
  if (lane == 0) A = 0.0;
  for (int a = a0; a < a1; ++a) {
    const double f = a == 0 ? 0.0 : fL[a];
    A = fma(f, A, rho[a]);
    v[a] = A;
  }
  // backward: B_a = g_a (B_(a+1) + rho_(a+1)), g_a = (r_a/r_(a+1))^(L+1), B_(n-1) = 0;
  // lane order reversed: the last chunk first
  const int bl = 31 - lane;
  const int b0 = bl * C, b1 = min(n, b0 + C);
  Aff mb{1.0, 0.0};
  for (int a = b1 - 1; a >= b0; --a) {
    const double gg = a == n - 1 ? 0.0 : gL[a + 1];
    const double rn = a == n - 1 ? 0.0 : rho[a + 1];
    mb = Aff{gg * mb.mul, gg * (mb.add + rn)};
  }
  Aff ib = mb;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const Aff o{__shfl_up_sync(0xffffffffu, ib.mul, d), __shfl_up_sync(0xffffffffu, ib.add, d)};
    if (lane >= d) ib = aff_then(o, ib);
  }
  double B = __shfl_up_sync(0xffffffffu, ib.add, 1);
  if (lane == 0) B = 0.0;
  __syncwarp();
  for (int a = b1 - 1; a >= b0; --a) {
    const double gg = a == n - 1 ? 0.0 : gL[a + 1];
    const double rn = a == n - 1 ? 0.0 : rho[a + 1];
    B = gg * (B + rn);
    v[a] = (v[a] + B) / g.r[a];
  }
}

// blocks (run, 32 radii, TH_WARPS nodes (m, j)): htab[m][j][r] = sum_{L>=1} v_L(r) P_L(x_j^m),
// TH_ILP partial sums over L
__global__ void __launch_bounds__(TH_THREADS) k_theta_table(GroupArgs g, ThetaArgs t) {
  const int tiles = (g.n_r + 31) / 32;
  const int n_mj = g.n_m * g.n_l;
  const int jsplit = (n_mj + TH_WARPS - 1) / TH_WARPS;
  const int ri = blockIdx.x / (tiles * jsplit);
  const int rest = blockIdx.x - ri * tiles * jsplit;
  const int tile = rest / jsplit, js = rest - tile * jsplit;
  const int r = tile * 32 + (threadIdx.x & 31);
  const int mj = js * TH_WARPS + (threadIdx.x >> 5);
  if (r >= g.n_r || mj >= n_mj) return;
  const RunDev run = g.runs[g.runs_of_group[ri]];
  const int n_r = g.n_r, n_mp = t.n_mp;
  const double* v = t.vmp + (size_t)ri * n_mp * n_r + r;
  const int m = mj / g.n_l, j = mj - m * g.n_l;
  // TH_ILP independent partial sums: the loop is bound by the latency of its loads
  double acc[TH_ILP];
#pragma unroll
  for (int u = 0; u < TH_ILP; ++u) acc[u] = 0.0;
  if (j >= m) {
    const double* pl = t.PLj + (size_t)m * n_mp * g.ldS + j;
    int L = 1;
    for (; L + TH_ILP - 1 < n_mp; L += TH_ILP)
#pragma unroll
      for (int u = 0; u < TH_ILP; ++u)
        acc[u] = fma(v[(size_t)(L + u) * n_r], __ldg(pl + (size_t)(L + u) * g.ldS), acc[u]);
    for (; L < n_mp; ++L) acc[0] = fma(v[(size_t)L * n_r], __ldg(pl + (size_t)L * g.ldS), acc[0]);
  }
  run.htab[(size_t)mj * n_r + r] = sum_partials(acc);
}

void launch_theta_potentials(const GroupArgs& g, const ThetaArgs& t, const double2* x, cudaStream_t s) {
  const int tiles = (g.n_r + 31) / 32;
  const int qsplit = (t.nq + TH_WARPS * TH_QB - 1) / (TH_WARPS * TH_QB);
  const int lsplit = (t.n_mp + TH_WARPS - 1) / TH_WARPS;
  const int jsplit = (g.n_m * g.n_l + TH_WARPS - 1) / TH_WARPS;
  k_theta_fine<<<g.n_runs * tiles * qsplit, TH_THREADS, 0, s>>>(g, t, x);
  k_theta_project<<<g.n_runs * tiles * lsplit, TH_THREADS, 0, s>>>(g, t);
  const int per_run = (t.n_mp - 1 + TH_WARPS - 1) / TH_WARPS;
  if (per_run > 0) k_theta_hartree<<<g.n_runs * per_run, TH_THREADS, 0, s>>>(g, t);
  k_theta_table<<<g.n_runs * tiles * jsplit, TH_THREADS, 0, s>>>(g, t);
}

}  // namespace ggb
