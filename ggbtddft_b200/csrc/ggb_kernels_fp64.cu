// FP64 (parity form) kernels of the split-operator step.
//
//  k_angular_fp64  one half of the angular step for a tile of 16 radii of one orbital column:
//                  the whole l-vector of every radius is held in shared memory while the chain
//                  (rotate -> phase -> [pre-multiplied rotate pair] -> phase ... -> rotate back,
//                  plus the l-diagonal S phase) is applied, each product on the FP64 tensor cores
//                  (mma.sync m8n8k4).  Replaces, per half-step, the 3 launches of each of
//                  h_couplingFF/FP/D/P (couplingP.cuh:108-125, couplingD.cuh, couplingF.cuh) and
//                  h_couplingS (couplingS.cuh:43-57).  The second half also produces the
//                  density-multipole and dipole/acceleration partial sums of the new orbitals
//                  (hartreePotentialDensity.cuh:1-181, dipoleMoment.cuh:1-75,
//                  dipoleAcceleration.cuh:1-71), so the orbitals are read once per half-step.
//  k_radial_fp64   x_l <- A_l x_l for every l with A_l(a,b) = W[l][b][a]: the batched ZGEMM of
//                  h_propagationH0 (h_timePropagation.cuh:1-30), out of place.  Persistent, two CTAs
//                  per SM; a producer warp streams the W rows and x segments of each 16-wide k chunk
//                  into a 3-stage shared-memory ring with cp.async.bulk (mbarrier transaction
//                  counts), so that ~200 KB per SM are in flight whatever the occupancy; four
//                  consumer warps (one output radius per thread, TC orbital columns in registers)
//                  run the FP64 FMAs from shared memory.
//  k_finalize      per run: observables of the step from the partials, density multipoles
//                  (occupation-weighted sum over orbitals), Hartree potentials by compensated
//                  prefix scans (h_calculateHartreePotential.cuh:1-136), LDA exchange
//                  (h_calculateExchangeCorrelationPotential.cuh:1-56), step counter.
#include <algorithm>
#include <cstdio>
#include "ggb_internal.cuh"
#include "ggb_angular.cuh"
#include "ggb_mixed.cuh"
#include "ggb_tc_common.cuh"

namespace ggb {

// ---------------------------------------------------------------------------------------------
// angular chain
// ---------------------------------------------------------------------------------------------

// A tile is RT radii of one orbital column (RT = the group's observables segment: 16 for the FP64
// form, 16 or 32 for the initial partials of the int8 form): the whole l-vector of each radius sits
// in shared memory as a [rows][2 RT + 8] FP64 matrix (column 2 rad + 0/1 = real/imaginary part of
// radius rad; rows N_l rounded up to 8, zero beyond N_l), and every product of the chain
// y_j = sum_l S[l][j] x_l is a small real GEMM  Y (N_l x 2 RT) = S^T (N_l x N_l) X (N_l x 2 RT)  on
// the FP64 tensor cores: mma.sync m8n8k4 (8 channels x 8 columns x 4 l per instruction).  Each warp
// owns pairs of 8-channel tiles (16 j) over all 2 RT columns; its S fragments come from L2
// (read-only path), prefetched one chunk of AM_KU k-steps ahead; its X fragments from shared
// memory.  The phases are applied to the accumulators in registers (each thread holds whole complex
// numbers: the real and imaginary column of one radius), then written to the other buffer for the
// next product.
constexpr int AM_WARPS = 4;
constexpr int AM_KU = 4;                    // k-steps (4 l each) per prefetch chunk
// row stride in doubles: +8 puts the 4 rows of an X fragment on alternating bank halves
__host__ __device__ constexpr int angular_ldx(int rt) { return 2 * rt + 8; }

__host__ __device__ constexpr int angular_rows_mma(int n_l) {
  // N_l rounded up to 8 (the channel tiles), and at least 16 rows: the free buffer holds the
  // AM_NSUB x N_DEN x AM_RT density partials of the epilogue
  return ((n_l + 7) / 8 * 8) > 16 ? (n_l + 7) / 8 * 8 : 16;
}

__device__ __forceinline__ void mma_f64_8x8x4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// One half of the angular step (or, with the empty chain of half 2, only the epilogue): replaces,
// per half-step, the 3 launches of each of h_couplingFF/FP/D/P (couplingP.cuh:108-125,
// couplingD.cuh, couplingF.cuh) and h_couplingS (couplingS.cuh:43-57); the second half also
// produces the density-multipole and dipole/acceleration partial sums of the new orbitals
// (hartreePotentialDensity.cuh:1-181, dipoleMoment.cuh:1-75, dipoleAcceleration.cuh:1-71).
template <int RT>
__global__ void __launch_bounds__(AM_WARPS * 32)
k_angular_fp64(GroupArgs g, int half, const double2* __restrict__ xin, double2* xout, int do_obs) {
  constexpr int AM_RT = RT;
  constexpr int AM_LDX = angular_ldx(RT);
  constexpr int AM_NT = 2 * RT / 8;                  // 8-column tiles per row
  constexpr int AM_NSUB = AM_WARPS * 32 / RT;        // lane groups of RT threads (epilogue)
  extern __shared__ double smd[];
  __shared__ double s_rr[RT], s_rE[RT], s_v1[RT], s_v2[RT], s_v3[RT], s_sb[RT];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int gid = lane >> 2;      // fragment row group
  const int q = lane & 3;         // fragment thread in group
  const int n_l = g.n_l;
  const int rows = angular_rows_mma(n_l);
  const int tilesN = (g.n_r + AM_RT - 1) / AM_RT;
  const int col = blockIdx.x / tilesN;
  const int tile = blockIdx.x - col * tilesN;
  const int r0 = tile * AM_RT;
  double* xs = smd;
  double* ys = smd + (size_t)rows * AM_LDX;
  const int m = g.col_m[col];
  const RunDev run = g.runs[g.col_run[col]];
  int step = *g.step;
  if (step >= run.n_t) step = run.n_t - 1;  // overflow is flagged by k_finalize

  // the tile's orbitals (zero beyond N_l and beyond N_r), zero padding rows in both buffers
  for (int i = tid; i < rows * AM_RT; i += blockDim.x) {
    const int l = i / AM_RT, rad = i - l * AM_RT, r = r0 + rad;
    const double2 v = (l < n_l && r < g.n_r) ? xin[((size_t)l * g.n_cols + col) * g.n_r + r]
                                             : make_double2(0.0, 0.0);
    *reinterpret_cast<double2*>(xs + (size_t)l * AM_LDX + 2 * rad) = v;
    if (l >= n_l) *reinterpret_cast<double2*>(ys + (size_t)l * AM_LDX + 2 * rad) = make_double2(0.0, 0.0);
  }
  // per-radius potentials
  if (tid < AM_RT) {
    const int r = r0 + tid;
    const bool rv = r < g.n_r;
    const int rc = rv ? r : 0;
    const double rr = rv ? g.r[r] : 1.0;
    double v1 = 0.0, v2 = 0.0, v3 = 0.0, sbase = 0.0;
    if (g.hartree_on) {
      v1 = run.v[1 * g.n_r + rc];
      v2 = run.v[2 * g.n_r + rc];
      v3 = run.v[3 * g.n_r + rc];
      // couplingS.cuh:20-21, evaluated left to right
      sbase = run.v[rc] - run.v0[rc] + run.vexc[rc] - run.vexc0[rc];
    }
    s_rr[tid] = rr;
    s_rE[tid] = rr * run.E[step];
    s_v1[tid] = v1;
    s_v2[tid] = v2;
    s_v3[tid] = v3;
    s_sb[tid] = sbase;
  }
  const double hdt = 0.5 * g.dt;
  const double* pco = g.coef + ((size_t)CF_P * g.n_m + m) * n_l;
  __syncthreads();

  const Chain& ch = g.chain[half];
  if (ch.pre_s) {
    for (int i = tid; i < n_l * AM_RT; i += blockDim.x) {
      const int l = i / AM_RT, rad = i - l * AM_RT;
      double eta = s_sb[rad] + pco[l] * s_v2[rad];
      eta *= hdt;
      double2* p = reinterpret_cast<double2*>(xs + (size_t)l * AM_LDX + 2 * rad);
      *p = cmul_conj_phase(*p, eta);
    }
    __syncthreads();
  }

  const int k_steps = (n_l + 3) / 4;
  const int n_pairs = ((n_l + 7) / 8 + 1) / 2;
  for (int o = 0; o < ch.n_ops; ++o) {
    const ChainOp op = ch.ops[o];
    const double* S = g.mats + ((size_t)op.mat * g.n_m + m) * (size_t)n_l * g.ldS;
    const bool last = (o == ch.n_ops - 1);
    const double* Dv = g.dph + ((size_t)op.coupling * g.n_m + m) * g.ldS;
    for (int pr = warp; pr < n_pairs; pr += AM_WARPS) {
      const int ja = pr * 16 + gid, jb = ja + 8;
      const bool va = ja < n_l, vb = jb < n_l;
      double acc[2][AM_NT][2];
#pragma unroll
      for (int t = 0; t < 2; ++t)
#pragma unroll
        for (int nt = 0; nt < AM_NT; ++nt) acc[t][nt][0] = acc[t][nt][1] = 0.0;
      // S fragments (A = S^T: row j, column l) of AM_KU k-steps; rows l < m are skipped, as the
      // reference's couplings start at l = m
      double fa[AM_KU][2], fn[AM_KU][2];
      auto load_a = [&](int ks0, double (&dst)[AM_KU][2]) {
#pragma unroll
        for (int u = 0; u < AM_KU; ++u) {
          const int l = (ks0 + u) * 4 + q;
          const bool lv = l >= m && l < n_l;
          dst[u][0] = (lv && va) ? __ldg(S + (size_t)l * g.ldS + ja) : 0.0;
          dst[u][1] = (lv && vb) ? __ldg(S + (size_t)l * g.ldS + jb) : 0.0;
        }
      };
      load_a(0, fa);
      for (int ks0 = 0; ks0 < k_steps; ks0 += AM_KU) {
        load_a(ks0 + AM_KU, fn);   // past the last k-step it loads nothing (l >= N_l)
#pragma unroll
        for (int u = 0; u < AM_KU; ++u) {
          if (ks0 + u < k_steps) {
            const double* xr = xs + (size_t)((ks0 + u) * 4 + q) * AM_LDX + gid;
            double fb[AM_NT];
#pragma unroll
            for (int nt = 0; nt < AM_NT; ++nt) fb[nt] = xr[nt * 8];
#pragma unroll
            for (int nt = 0; nt < AM_NT; ++nt) {
              mma_f64_8x8x4(acc[0][nt][0], acc[0][nt][1], fa[u][0], fb[nt]);
              mma_f64_8x8x4(acc[1][nt][0], acc[1][nt][1], fa[u][1], fb[nt]);
            }
          }
        }
#pragma unroll
        for (int u = 0; u < AM_KU; ++u) { fa[u][0] = fn[u][0]; fa[u][1] = fn[u][1]; }
      }
      // phases on the accumulators: thread (gid, q) holds channel j = pair base + 8 t + gid, radius
      // 4 nt + q, real and imaginary part (couplingP.cuh:61-106 and twins)
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int j = pr * 16 + 8 * t + gid;
        if (j >= n_l) continue;
        const double dj = Dv[j];
#pragma unroll
        for (int nt = 0; nt < AM_NT; ++nt) {
          const int rad = 4 * nt + q;
          double2 y = make_double2(acc[t][nt][0], acc[t][nt][1]);
          if (op.phase == PH_THETA && j >= m) {
            // the theta form: the whole angular potential at node x_j
            double eta = (s_rE[rad] + s_v1[rad]) * dj + s_v2[rad] * legendre_p2(dj) +
                         s_v3[rad] * legendre_p3(dj) + s_sb[rad];
            // n_har > 4: the multipoles L >= 1 at this node come from the exact-quadrature table
            if (g.theta_tab && r0 + rad < g.n_r) eta += run.htab[((size_t)m * n_l + j) * g.n_r + r0 + rad];
            eta *= hdt;
            y = cmul_conj_phase(y, eta);
          } else if (op.phase != PH_NONE && j >= m) {
            double eta;
            if (op.phase == PH_P) eta = g.p_hartree ? (s_rE[rad] + s_v1[rad]) : s_rE[rad];
            else if (op.phase == PH_D) eta = s_v2[rad];
            else eta = s_v3[rad];   // FP and FF
            eta *= hdt * dj;
            y = cmul_conj_phase(y, eta);
          }
          if (last && ch.post_s) {
            double eta = s_sb[rad] + pco[j] * s_v2[rad];
            eta *= hdt;
            y = cmul_conj_phase(y, eta);
          }
          *reinterpret_cast<double2*>(ys + (size_t)j * AM_LDX + 2 * rad) = y;
        }
      }
    }
    __syncthreads();
    double* t = xs; xs = ys; ys = t;
  }

  const double2* x2 = reinterpret_cast<const double2*>(xs);
  if (xout)
    for (int i = tid; i < n_l * AM_RT; i += blockDim.x) {
      const int l = i / AM_RT, rad = i - l * AM_RT, r = r0 + rad;
      if (r < g.n_r) xout[((size_t)l * g.n_cols + col) * g.n_r + r] = x2[(size_t)l * (AM_LDX / 2) + rad];
    }

  if (do_obs) {
    // lane groups of AM_RT threads, one radius per thread
    const int lr = lane % AM_RT, sub = warp * (32 / AM_RT) + lane / AM_RT;
    const double rr = s_rr[lr];
    const double fr2 = (r0 + lr < g.n_r) ? pow(rr, -2.0) : 0.0;
    observables_tile<double2, AM_LDX / 2>(g, x2, col, m, r0, lr, sub, AM_NSUB, rr, fr2);
    // density multipoles: the literal l loops strided over the lane groups, then the groups summed
    // in order (the free buffer holds the AM_NSUB x N_DEN x AM_RT partials)
    const int n_den = g.n_den > 0 ? g.n_den : 1;  // L = 0 is always needed for the norm
    double d[N_DEN] = {0.0, 0.0, 0.0, 0.0};
    density_partials<double2, AM_LDX / 2>(n_den, m, n_l, x2, lr, g.coef + (size_t)m * n_l, sub, AM_NSUB, d,
                                          g.n_m * n_l);
#pragma unroll
    for (int L = 0; L < N_DEN; ++L) ys[(sub * N_DEN + L) * AM_RT + lr] = d[L];
    __syncthreads();
    if (tid < n_den * AM_RT) {
      const int L = tid / AM_RT, p = tid - L * AM_RT, rl = r0 + p;
      double sum = 0.0;
      for (int w = 0; w < AM_NSUB; ++w) sum += ys[(w * N_DEN + L) * AM_RT + p];
      if (rl < g.n_r) g.dens[((size_t)col * N_DEN + L) * g.n_r + rl] = sum;
    }
  }
}

static size_t angular_smem_rt(int n_l, int rt) {
  return 2 * (size_t)angular_rows_mma(n_l) * angular_ldx(rt) * sizeof(double);
}
// the largest launch for groups of up to n_l channels: 32-radius tiles only for N_l <= 128 (the int8
// form's initial partials), 16-radius tiles otherwise
size_t angular_smem_fp64(int n_l) {
  return std::max(angular_smem_rt(std::min(n_l, 128), TR), angular_smem_rt(n_l, 16));
}

void launch_angular_fp64(const GroupArgs& g, int half, const double2* xin, double2* xout, int do_obs,
                         cudaStream_t s) {
  if (g.obs_seg == 16) {
    const int tiles = g.n_cols * ((g.n_r + 15) / 16);
    k_angular_fp64<16><<<tiles, AM_WARPS * 32, angular_smem_rt(g.n_l, 16), s>>>(g, half, xin, xout, do_obs);
  } else {
    const int tiles = g.n_cols * ((g.n_r + TR - 1) / TR);
    k_angular_fp64<TR><<<tiles, AM_WARPS * 32, angular_smem_rt(g.n_l, TR), s>>>(g, half, xin, xout, do_obs);
  }
}

// ---------------------------------------------------------------------------------------------
// radial propagator, FP64
// ---------------------------------------------------------------------------------------------

constexpr int RAD_CW = 4;                 // consumer warps: one output radius per thread
constexpr int RAD_TI = 32 * RAD_CW;       // rows (output radii) per tile
constexpr int RAD_KC = 16;                // k per stage (3 stages of ~35 KB: two CTAs per SM)
constexpr int RAD_STAGES = 3;
constexpr int RAD_THREADS = 32 * (RAD_CW + 1);

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Tiles (l, radius tile, column tile), the column tile fastest so that CTAs running side by side
// read the same W rows (one HBM read, the others from L2).
template <int TC>
__global__ void __launch_bounds__(RAD_THREADS, 2)
k_radial_fp64(int n_r, int n_cols, int n_l, const double2* __restrict__ W, const double2* __restrict__ xin,
              double2* __restrict__ xout, unsigned* status) {
  constexpr int W_STAGE = RAD_KC * RAD_TI;        // double2 per stage: [k][row]
  constexpr int X_STAGE = TC * RAD_KC;            // [col][k]
  extern __shared__ __align__(128) double2 rsm[];
  __shared__ uint64_t full_bar[RAD_STAGES], empty_bar[RAD_STAGES];
  __shared__ int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_it = (n_r + RAD_TI - 1) / RAD_TI, n_ct = (n_cols + TC - 1) / TC;
  const int total = n_it * n_ct * n_l;
  const int n_kc = (n_r + RAD_KC - 1) / RAD_KC;
  if (threadIdx.x == 0) {
    for (int s = 0; s < RAD_STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], RAD_CW);
    }
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  volatile int* abort_p = &abort_flag;
  if (warp == RAD_CW) {
    // producer: one thread issues the bulk copies of every stage
    if (lane == 0) {
      int it = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < total && ok; tile += gridDim.x) {
        const int ct = tile % n_ct, rest = tile / n_ct, itile = rest % n_it, l = rest / n_it;
        const int i0 = itile * RAD_TI, rows = min(RAD_TI, n_r - i0);
        const int c0 = ct * TC, nc = min(TC, n_cols - c0);
        const double2* Wl = W + (size_t)l * n_r * n_r;
        const double2* Xl = xin + (size_t)l * n_cols * n_r;
        for (int kc = 0; kc < n_kc; ++kc, ++it) {
          const int s = it % RAD_STAGES;
          if (it >= RAD_STAGES && !mbar_wait(&empty_bar[s], ((it / RAD_STAGES) & 1) ^ 1, abort_p)) {
            ok = false;
            break;
          }
          const int k0 = kc * RAD_KC, kn = min(RAD_KC, n_r - k0);
          double2* ws = rsm + (size_t)s * (W_STAGE + X_STAGE);
          double2* xs = ws + W_STAGE;
          mbar_expect_tx(&full_bar[s], (uint32_t)(kn * rows + nc * kn) * 16u);
          for (int kk = 0; kk < kn; ++kk)
            bulk_g2s(ws + kk * RAD_TI, Wl + (size_t)(k0 + kk) * n_r + i0, (uint32_t)rows * 16u, &full_bar[s]);
          for (int c = 0; c < nc; ++c)
            bulk_g2s(xs + c * RAD_KC, Xl + (size_t)(c0 + c) * n_r + k0, (uint32_t)kn * 16u, &full_bar[s]);
        }
      }
      if (!ok) {
        // let the copies already issued land before the CTA exits
        for (int q = (it > RAD_STAGES ? it - RAD_STAGES : 0); q < it; ++q)
          mbar_drain(&full_bar[q % RAD_STAGES], (q / RAD_STAGES) & 1);
      }
    }
  } else {
    // consumers on the FP64 tensor cores: warp w computes output radii i0 + 32 w .. + 31 (four 8-row
    // MMA tiles) for the tile's TC columns.  Real form of the complex product, columns interleaved
    // (2 c + 0/1 = real/imaginary part of column c):  [Yr Yi] = Wr B + Wi B'  with B = [Xr Xi] and
    // B' = [-Xi Xr] per column, so that a thread's two accumulators of an 8-column tile are one
    // complex output.  A (i, k) = W[l][k][i] from the W rows in shared memory (one 16-byte load
    // gives the Wr and Wi fragments), B and B' from one 16-byte load of x.  k beyond the row (the
    // last chunk) contributes zero on both sides.
    constexpr int NT = (2 * TC + 7) / 8;            // 8-column MMA tiles
    const int g8 = lane >> 2, q = lane & 3;
    int it = 0;
    for (int tile = blockIdx.x; tile < total; tile += gridDim.x) {
      const int ct = tile % n_ct, rest = tile / n_ct, itile = rest % n_it, l = rest / n_it;
      const int i0 = itile * RAD_TI;
      const int c0 = ct * TC, nc = min(TC, n_cols - c0);
      // separate accumulators for the Wr and Wi products (up to 24 columns; beyond, the registers
      // would spill): the 2 x 4 x NT MMAs of a k step are independent, where one accumulator chain
      // makes every second MMA wait for the first
      constexpr bool SPLIT = NT <= 3;
      double acc[4][NT][2], acd[4][NT][2];
      auto& adst = SPLIT ? acd : acc;
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = acd[mt][nt][0] = acd[mt][nt][1] = 0.0;
      bool ok = true;
      for (int kc = 0; kc < n_kc; ++kc, ++it) {
        const int s = it % RAD_STAGES;
        if (!mbar_wait(&full_bar[s], (it / RAD_STAGES) & 1, abort_p)) {
          ok = false;
          break;
        }
        const int kn = min(RAD_KC, n_r - kc * RAD_KC);
        const double2* ws = rsm + (size_t)s * (W_STAGE + X_STAGE);
        const double2* xs = ws + W_STAGE;
#pragma unroll
        for (int ks = 0; ks < RAD_KC / 4; ++ks) {
          const int kk = 4 * ks + q;
          const bool kv = kk < kn;
          double ar[4], ai[4], bp[NT], bq[NT];
#pragma unroll
          for (int mt = 0; mt < 4; ++mt) {
            const double2 w = kv ? ws[kk * RAD_TI + 32 * warp + 8 * mt + g8] : make_double2(0.0, 0.0);
            ar[mt] = w.x;
            ai[mt] = w.y;
          }
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) {
            const int c = 4 * nt + (g8 >> 1);
            const double2 x = (kv && c < TC) ? xs[c * RAD_KC + kk] : make_double2(0.0, 0.0);
            bp[nt] = (g8 & 1) ? x.y : x.x;
            bq[nt] = (g8 & 1) ? x.x : -x.y;
          }
#pragma unroll
          for (int mt = 0; mt < 4; ++mt)
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
              mma_f64_8x8x4(acc[mt][nt][0], acc[mt][nt][1], ar[mt], bp[nt]);
              mma_f64_8x8x4(adst[mt][nt][0], adst[mt][nt][1], ai[mt], bq[nt]);
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty_bar[s]);
      }
      if (!ok) break;
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const int i = i0 + 32 * warp + 8 * mt + g8;
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          const int c = 4 * nt + q;
          if (i < n_r && c < nc)
            xout[((size_t)l * n_cols + c0 + c) * n_r + i] =
                make_double2(acc[mt][nt][0] + acd[mt][nt][0], acc[mt][nt][1] + acd[mt][nt][1]);
        }
      }
    }
  }
  __syncthreads();
  if (abort_flag && threadIdx.x == 0) atomicOr(status, ST_TC_TIMEOUT);
}

template <int TC>
static constexpr size_t radial_fp64_smem() {
  return (size_t)RAD_STAGES * (RAD_KC * RAD_TI + TC * RAD_KC) * sizeof(double2);
}

static int g_radial_sms = 0;

void launch_radial_fp64(const GroupArgs& g, const double2* W, const double2* xin, double2* xout, cudaStream_t s) {
  const int nc = g.n_cols;
  int tc = nc >= 16 ? 16 : nc;
  static const int opts[] = {1, 2, 3, 4, 6, 8, 9, 12, 16};
  for (int o : opts)
    if (o >= tc) { tc = o; break; }
  const int tiles = ((g.n_r + RAD_TI - 1) / RAD_TI) * ((nc + tc - 1) / tc) * g.n_l;
  const int ctas = std::min(tiles, 2 * g_radial_sms);
#define GGB_RAD_CASE(C)                                                                                     \
  case C:                                                                                                   \
    k_radial_fp64<C><<<ctas, RAD_THREADS, radial_fp64_smem<C>(), s>>>(g.n_r, nc, g.n_l, W, xin, xout, g.status); \
    break;
  switch (tc) {
    GGB_RAD_CASE(1) GGB_RAD_CASE(2) GGB_RAD_CASE(3) GGB_RAD_CASE(4) GGB_RAD_CASE(6)
    GGB_RAD_CASE(8) GGB_RAD_CASE(9) GGB_RAD_CASE(12) GGB_RAD_CASE(16)
    default: break;
  }
#undef GGB_RAD_CASE
}

static cudaError_t configure_radial_fp64() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&g_radial_sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
#define GGB_RAD_ATTR(C)                                                                                   \
  e = cudaFuncSetAttribute((const void*)k_radial_fp64<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                           (int)radial_fp64_smem<C>());                                                   \
  if (e != cudaSuccess) return e;
  GGB_RAD_ATTR(1) GGB_RAD_ATTR(2) GGB_RAD_ATTR(3) GGB_RAD_ATTR(4) GGB_RAD_ATTR(6)
  GGB_RAD_ATTR(8) GGB_RAD_ATTR(9) GGB_RAD_ATTR(12) GGB_RAD_ATTR(16)
#undef GGB_RAD_ATTR
  return cudaSuccess;
}

// ---------------------------------------------------------------------------------------------
// finalize: observables, Hartree multipoles (compensated scans), exchange, step counter
// ---------------------------------------------------------------------------------------------

constexpr int FIN_THREADS = 256;

// Inclusive (forward) or suffix-exclusive (backward) compensated scan of t[0..n) in shared memory.
// forward:  out[a] = sum_{b <= a} t[b]      backward: out[a] = sum_{b > a} t[b]
__device__ void block_scan_dd(const double* t, double* out, int n, bool backward, dd* wsum) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = FIN_THREADS / 32;
  const int per = (n + FIN_THREADS - 1) / FIN_THREADS;
  const int b0 = tid * per;
  // local inclusive sums in the scan direction
  dd loc{0.0, 0.0};
  for (int q = 0; q < per; ++q) {
    const int k = b0 + q;
    if (k < n) loc = dd_add(loc, dd{t[backward ? n - 1 - k : k], 0.0});
  }
  // warp inclusive scan of thread totals
  dd inc = loc;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    dd o = dd_shfl_up(inc, d);
    if (lane >= d) inc = dd_add(o, inc);
  }
  if (lane == 31) wsum[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    dd w = lane < nw ? wsum[lane] : dd{0.0, 0.0};
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      dd o = dd_shfl_up(w, d);
      if (lane >= d) w = dd_add(o, w);
    }
    if (lane < nw) wsum[lane] = w;
  }
  __syncthreads();
  // exclusive prefix of this thread = inclusive value of the previous lane + earlier warps
  const dd prev = dd_shfl_up(inc, 1);
  dd run = lane == 0 ? dd{0.0, 0.0} : prev;
  if (warp > 0) run = dd_add(wsum[warp - 1], run);
  for (int q = 0; q < per; ++q) {
    const int k = b0 + q;
    if (k < n) {
      const int idx = backward ? n - 1 - k : k;
      const double tv = t[idx];
      if (backward) {
        out[idx] = run.hi + run.lo;                 // exclusive (sum over b > a)
        run = dd_add(run, dd{tv, 0.0});
      } else {
        run = dd_add(run, dd{tv, 0.0});
        out[idx] = run.hi + run.lo;                 // inclusive (sum over b <= a)
      }
    }
  }
  __syncthreads();
}

__device__ __forceinline__ dd warp_sum_dd2(dd a) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const dd b{__shfl_xor_sync(0xffffffffu, a.hi, o), __shfl_xor_sync(0xffffffffu, a.lo, o)};
    a = dd_add(a, b);
  }
  return a;
}

__device__ __forceinline__ double ipow(double x, int L) {
  double p = 1.0;
  for (int i = 0; i < L; ++i) p *= x;
  return p;
}

// Blocks: for each run of the group, n_den Hartree blocks (L = 0..n_den-1; block L = 0 also does
// the exchange potential) + FIN_OB observables blocks.  mode 0 = initial potentials (no observables,
// no step increment), mode 1 = end of step, mode 2 = end of step without the step increment and the
// watchdog checks (the per-phase timing).
//
// Observables: observables block ob sums the partials of a slice of l (one warp per orbital, lanes
// striding over the tiles, double-double), writes the per-l series and its slice's totals to a
// scratch row; the last of the run's FIN_OB blocks to finish (a per-run counter) adds the slices in
// order, writes the totals and the norm and runs the NaN / norm-growth watchdog.
__global__ void __launch_bounds__(FIN_THREADS) k_finalize(GroupArgs g, int mode) {
  extern __shared__ double fsm[];  // [3][N_r]
  __shared__ dd wsum[FIN_THREADS / 32];
  __shared__ int s_last;
  const int nb = g.n_den + FIN_OB;
  const int ri = blockIdx.x / nb;
  const int role = blockIdx.x - ri * nb;  // < n_den: Hartree L = role; >= n_den: observables slice
  const int run_idx = g.runs_of_group[ri];
  RunDev run = g.runs[run_idx];
  const int n_r = g.n_r, n_l = g.n_l, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int step = *g.step;
  const bool obs_block = role >= g.n_den;
  const int ob = role - g.n_den;

  if (obs_block && mode != 0) {
    if (step >= run.n_t) {
      if (mode == 1 && ob == 0 && tid == 0) atomicOr(g.status, ST_STEP_OVERFLOW);
    } else {
      const int n_orb = run.n_orb;
      const int l0 = ob * n_l / FIN_OB, l1 = (ob + 1) * n_l / FIN_OB;
      for (int k = warp; k < n_orb; k += FIN_THREADS / 32) {
        dd tx{0.0, 0.0}, ty{0.0, 0.0}, tz{0.0, 0.0}, tw{0.0, 0.0};
        for (int l = l0; l < l1; ++l) {
          const double4* p = g.obs + 2 * (((size_t)(run.col0 + k) * n_l + l) * g.n_tiles);
          dd sx{0.0, 0.0}, sy{0.0, 0.0}, sz{0.0, 0.0}, sw{0.0, 0.0};
          for (int t = lane; t < g.n_tiles; t += 32) {
            const double4 h = p[2 * t], lo = p[2 * t + 1];
            sx = dd_add(sx, dd{h.x, lo.x}); sy = dd_add(sy, dd{h.y, lo.y});
            sz = dd_add(sz, dd{h.z, lo.z}); sw = dd_add(sw, dd{h.w, lo.w});
          }
          sx = warp_sum_dd2(sx); sy = warp_sum_dd2(sy); sz = warp_sum_dd2(sz); sw = warp_sum_dd2(sw);
          if (lane == 0 && g.per_l) {
            run.dip[((size_t)l * n_orb + k) * run.n_t + step] = make_double2(sx.hi + sx.lo, sy.hi + sy.lo);
            run.acc[((size_t)l * n_orb + k) * run.n_t + step] = make_double2(sz.hi + sz.lo, sw.hi + sw.lo);
          }
          tx = dd_add(tx, sx); ty = dd_add(ty, sy); tz = dd_add(tz, sz); tw = dd_add(tw, sw);
        }
        if (lane == 0) {
          double* o = g.fin_scr + ((size_t)(run.col0 + k) * FIN_OB + ob) * 8;
          o[0] = tx.hi; o[1] = tx.lo; o[2] = ty.hi; o[3] = ty.lo;
          o[4] = tz.hi; o[5] = tz.lo; o[6] = tw.hi; o[7] = tw.lo;
        }
      }
      __syncthreads();
      if (tid == 0) {
        __threadfence();
        s_last = atomicAdd(g.fin_cnt + ri, 1u) == (unsigned)(FIN_OB - 1);
      }
      __syncthreads();
      if (s_last) {
        __threadfence();
        // totals over l (the slices in order), the norm; one warp per orbital
        for (int k = warp; k < n_orb; k += FIN_THREADS / 32) {
          dd sx{0.0, 0.0}, sy{0.0, 0.0}, sz{0.0, 0.0}, sw{0.0, 0.0};
          for (int b = 0; b < FIN_OB; ++b) {
            const double* o = g.fin_scr + ((size_t)(run.col0 + k) * FIN_OB + b) * 8;
            sx = dd_add(sx, dd{__ldcg(o + 0), __ldcg(o + 1)}); sy = dd_add(sy, dd{__ldcg(o + 2), __ldcg(o + 3)});
            sz = dd_add(sz, dd{__ldcg(o + 4), __ldcg(o + 5)}); sw = dd_add(sw, dd{__ldcg(o + 6), __ldcg(o + 7)});
          }
          const double* dn = g.dens + (size_t)(run.col0 + k) * N_DEN * n_r;  // L = 0 row
          dd nd{0.0, 0.0};
          for (int q = lane; q < n_r; q += 32) nd = dd_add(nd, dd{dn[q], 0.0});
          nd = warp_sum_dd2(nd);
          const double nrm = nd.hi + nd.lo;
          if (lane == 0) {
            run.dip_tot[(size_t)k * run.n_t + step] = make_double2(sx.hi + sx.lo, sy.hi + sy.lo);
            run.acc_tot[(size_t)k * run.n_t + step] = make_double2(sz.hi + sz.lo, sw.hi + sw.lo);
            run.norm[(size_t)k * run.n_t + step] = nrm;
            if (mode == 1) {
              if (!(nrm == nrm) || isinf(nrm) || !(sx.hi == sx.hi) || !(sz.hi == sz.hi)) atomicOr(g.status, ST_NAN);
              if (nrm > run.norm0[k] * (1.0 + g.norm_tol) + 1e-300) atomicOr(g.status, ST_NORM_GROWTH);
            }
          }
        }
        if (tid == 0) g.fin_cnt[ri] = 0u;   // for the next launch (stream-ordered after this one)
      }
    }
  } else if (obs_block && mode == 0 && ob == 0) {
    // initial norm for the growth watchdog
    for (int k = warp; k < run.n_orb; k += FIN_THREADS / 32) {
      const double* dn = g.dens + (size_t)(run.col0 + k) * N_DEN * n_r;
      dd nd{0.0, 0.0};
      for (int q = lane; q < n_r; q += 32) nd = dd_add(nd, dd{dn[q], 0.0});
      nd = warp_sum_dd2(nd);
      if (lane == 0) run.norm0[k] = nd.hi + nd.lo;
    }
  }

  if (!obs_block) {
    const int L = role;
    double* rho = fsm;            // [N_r]
    double* F = fsm + n_r;        // forward partial sums
    double* G = fsm + 2 * n_r;    // backward partial sums
    // rho_L(r) = sum_kso occ * density_kso (hartreePotentialDensity.cuh:58-60, orbital order)
    for (int q = tid; q < n_r; q += FIN_THREADS) {
      double s = 0.0;
      for (int k = 0; k < run.n_orb; ++k)
        s += (double)g.col_occ[run.col0 + k] * g.dens[((size_t)(run.col0 + k) * N_DEN + L) * n_r + q];
      rho[q] = s;
    }
    __syncthreads();
    // v_L(r_a) = r_a^-(L+1) sum_{b<=a} rho(b) r_b^L + r_a^L sum_{b>a} rho(b) r_b^-(L+1)
    for (int q = tid; q < n_r; q += FIN_THREADS) {
      const double rb = g.r[q];
      F[q] = rho[q] * ipow(rb, L);
      G[q] = rho[q] / ipow(rb, L + 1);
    }
    __syncthreads();
    block_scan_dd(F, F, n_r, false, wsum);
    block_scan_dd(G, G, n_r, true, wsum);
    for (int q = tid; q < n_r; q += FIN_THREADS) {
      const double ra = g.r[q];
      const double v = F[q] / ipow(ra, L + 1) + ipow(ra, L) * G[q];
      run.v[(size_t)L * n_r + q] = v;
      if (mode == 0 && L == 0) run.v0[q] = v;
    }
  }

  // exchange (block L = 0, or the first observables block when Hartree is off)
  const bool xc_block = (g.n_den > 0) ? (role == 0) : (ob == 0);
  if (xc_block) {
    const bool pw92 = (run.flags & RUN_FLAG_PW92) != 0;
    for (int q = tid; q < n_r; q += FIN_THREADS) {
      double rho0 = 0.0;
      if (g.n_den > 0) rho0 = fsm[q];
      // h_calculateExchangeCorrelationPotential.cuh:33-44
      double den = g.n_g_fac * (rho0 / 4.0 / M_PI + run.rho_frozen[q]) / g.drdx[q] * pow(g.P[q], 2.0);
      const double rq = g.r[q];
      if (mode == 0) {
        double vx0 = -pow(3.0 / M_PI * den, 1.0 / 3.0);
        vx0 /= pow(rq, 2.0 / 3.0);
        if (pw92) {
          // PW92 correlation of n = den / r^2 (not in the reference)
          const double n = fmax(den / (rq * rq), 1e-300);
          const double a = 0.031091, a1 = 0.21370, b1 = 7.5957, b2 = 3.5876, b3 = 1.6382, b4 = 0.49294;
          const double rs = cbrt(3.0 / (4.0 * M_PI * n)), srs = sqrt(rs);
          const double q0 = -2.0 * a * (1.0 + a1 * rs);
          const double q1 = 2.0 * a * (b1 * srs + b2 * rs + b3 * rs * srs + b4 * rs * rs);
          const double q1p = a * (b1 / srs + 2.0 * b2 + 3.0 * b3 * srs + 4.0 * b4 * rs);
          const double lg = log1p(1.0 / q1);
          vx0 += q0 * lg - rs / 3.0 * (-2.0 * a * a1 * lg - q0 * q1p / (q1 * q1 + q1));
        }
        run.vexc0[q] = vx0;
      }
      if (den < 0.0) den = 0.0;
      double vx = -pow(3.0 / M_PI * den, 1.0 / 3.0);
      vx /= pow(rq, 2.0 / 3.0);
      if (pw92) {
        const double n = fmax(den / (rq * rq), 1e-300);
        const double a = 0.031091, a1 = 0.21370, b1 = 7.5957, b2 = 3.5876, b3 = 1.6382, b4 = 0.49294;
        const double rs = cbrt(3.0 / (4.0 * M_PI * n)), srs = sqrt(rs);
        const double q0 = -2.0 * a * (1.0 + a1 * rs);
        const double q1 = 2.0 * a * (b1 * srs + b2 * rs + b3 * rs * srs + b4 * rs * rs);
        const double q1p = a * (b1 / srs + 2.0 * b2 + 3.0 * b3 * srs + 4.0 * b4 * rs);
        const double lg = log1p(1.0 / q1);
        vx += q0 * lg - rs / 3.0 * (-2.0 * a * a1 * lg - q0 * q1p / (q1 * q1 + q1));
      }
      // GGB_RUN_XC_FROZEN: the exchange-correlation potential stays at its t = 0 value
      run.vexc[q] = (run.flags & RUN_FLAG_XC_FROZEN) ? run.vexc0[q] : vx;
    }
  }

  // last block of a step advances the shared step counter
  if (mode == 1) {
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      const unsigned total = gridDim.x;
      const unsigned prev = atomicAdd(g.done, 1u);
      if (prev == total - 1) {
        *g.done = 0u;
        __threadfence();
        atomicAdd(g.step, 1);
      }
    }
  }
}

void launch_finalize(const GroupArgs& g, int mode, cudaStream_t s) {
  const dim3 grid(g.n_runs * (g.n_den + FIN_OB)), block(FIN_THREADS);
  const size_t smem = 3 * (size_t)g.n_r * sizeof(double);
  k_finalize<<<grid, block, smem, s>>>(g, mode);
}

// Allow a kernel the largest dynamic shared memory the device offers beyond its static part.
cudaError_t set_max_dynamic_smem(const void* fn, int optin) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, fn);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

cudaError_t configure_kernels_fp64(int n_l_max, int n_r_max) {
  // The attribute is global per function: set it to the device's opt-in maximum once, so that
  // contexts of different sizes can coexist.  Callers check their own sizes against it.
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  if (angular_smem_fp64(n_l_max) > (size_t)optin || 3 * (size_t)n_r_max * sizeof(double) > (size_t)optin)
    return cudaErrorInvalidValue;
  e = set_max_dynamic_smem((const void*)k_angular_fp64<16>, optin);
  if (e != cudaSuccess) return e;
  e = set_max_dynamic_smem((const void*)k_angular_fp64<TR>, optin);
  if (e != cudaSuccess) return e;
  e = configure_radial_fp64();
  if (e != cudaSuccess) return e;
  return set_max_dynamic_smem((const void*)k_finalize, optin);
}

}  // namespace ggb
