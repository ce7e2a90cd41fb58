// FP64 (parity form) kernels of the split-operator step.
//
//  k_angular_fp64  one half of the angular step for a tile of 32 radii of one orbital column:
//                  the whole l-vector of every radius is held in shared memory while the chain
//                  (rotate -> phase -> [pre-multiplied rotate pair] -> phase ... -> rotate back,
//                  plus the l-diagonal S phase) is applied.  Replaces, per half-step, the 3
//                  launches of each of h_couplingFF/FP/D/P (couplingP.cuh:108-125, couplingD.cuh,
//                  couplingF.cuh) and h_couplingS (couplingS.cuh:43-57).  The second half also
//                  produces the density-multipole and dipole/acceleration partial sums of the new
//                  orbitals (hartreePotentialDensity.cuh:1-181, dipoleMoment.cuh:1-75,
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
#include <cooperative_groups.h>

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

constexpr int ANG_JB = 8;   // eigen-channels j per register block

// RT radii per CTA (32, or 16 with the two half-warps on different eigen-channel blocks): lane % RT is
// the radius, lane / RT picks the half; the group's observables partials cover RT radii each.
// CL = 2: a cluster of two CTAs shares one tile: each computes half of the eigen-channels of every
// product (reading half of the chain matrix) and writes its half into both CTAs' shared memory
// (distributed shared memory), a cluster barrier between products; the same arithmetic as CL = 1,
// with twice the CTAs for runs too small to fill the GPU.
template <int RT, int CL>
__global__ void __launch_bounds__(ANG_WARPS * 32)
k_angular_fp64(GroupArgs g, int half, const double2* __restrict__ xin, double2* __restrict__ xout, int do_obs) {
  namespace cg = cooperative_groups;
  constexpr int SUB = 32 / RT;                    // lanes groups per warp (1 or 2)
  constexpr int NSUB = ANG_WARPS * SUB;           // thread groups that stride l and j in one CTA
  extern __shared__ double2 sm[];  // two [N_l][RT] buffers
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int lr = lane % RT;                       // radius of this lane
  const int sub = warp * SUB + lane / RT;         // this thread's group
  const int crank = CL == 2 ? (int)cg::this_cluster().block_rank() : 0;
  const int gsub = crank * NSUB + sub;            // this thread's group across the cluster
  const int tilesN = (g.n_r + RT - 1) / RT;
  const int bt = blockIdx.x / CL;                 // the tile of this CTA (or CTA pair)
  const int col = bt / tilesN;
  const int tile = bt - col * tilesN;
  const int r = tile * RT + lr;
  const bool rv = r < g.n_r;
  const int n_l = g.n_l;
  double2* xs = sm;
  double2* ys = sm + (size_t)n_l * RT;
  const int m = g.col_m[col];
  const RunDev run = g.runs[g.col_run[col]];
  int step = *g.step;
  if (step >= run.n_t) step = run.n_t - 1;  // overflow is flagged by k_finalize

  for (int l = sub; l < n_l; l += NSUB)
    xs[l * RT + lr] = rv ? xin[((size_t)l * g.n_cols + col) * g.n_r + r] : make_double2(0.0, 0.0);

  // per-radius potentials
  const double rr = rv ? g.r[r] : 1.0;
  const int rc = rv ? r : 0;
  const double E = run.E[step];
  double v1 = 0.0, v2 = 0.0, v3 = 0.0, sbase = 0.0;
  if (g.hartree_on) {
    v1 = run.v[1 * g.n_r + rc];
    v2 = run.v[2 * g.n_r + rc];
    v3 = run.v[3 * g.n_r + rc];
    // couplingS.cuh:20-21, evaluated left to right
    sbase = run.v[rc] - run.v0[rc] + run.vexc[rc] - run.vexc0[rc];
  }
  const double hdt = 0.5 * g.dt;
  const double* pco = g.coef + ((size_t)CF_P * g.n_m + m) * n_l;
  if constexpr (CL == 2) cg::this_cluster().sync();   // both CTAs running before any remote write
  else __syncthreads();

  const Chain& ch = g.chain[half];
  if (ch.pre_s) {
    for (int l = sub; l < n_l; l += NSUB) {
      double eta = sbase + pco[l] * v2;
      eta *= hdt;
      xs[l * RT + lr] = cmul_conj_phase(xs[l * RT + lr], eta);
    }
    __syncthreads();
  }

  for (int o = 0; o < ch.n_ops; ++o) {
    const ChainOp op = ch.ops[o];
    const double* S = g.mats + ((size_t)op.mat * g.n_m + m) * (size_t)n_l * g.ldS;
    const bool last = (o == ch.n_ops - 1);
    double base = 0.0;
    if (op.phase == PH_P) base = g.p_hartree ? (rr * E + v1) : (rr * E);
    else if (op.phase == PH_D) base = v2;
    else if (op.phase != PH_NONE) base = v3;  // FP and FF
    const double* Dv = g.dph + ((size_t)op.coupling * g.n_m + m) * g.ldS;
    double2* ys_peer = ys;
    if constexpr (CL == 2) ys_peer = cg::this_cluster().map_shared_rank(ys, crank ^ 1);
    for (int j0 = gsub * ANG_JB; j0 < n_l; j0 += CL * NSUB * ANG_JB) {
      double2 acc[ANG_JB];
#pragma unroll
      for (int q = 0; q < ANG_JB; ++q) acc[q] = make_double2(0.0, 0.0);
      const double* Sc = S + j0;
      int l = m;
      // four l rows per iteration: 16 independent 16-byte loads of S in flight per thread
      for (; l + 4 <= n_l; l += 4) {
        double2 sv[4][ANG_JB / 2];
        double2 xv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          xv[u] = xs[(l + u) * RT + lr];
          const double2* Srow = reinterpret_cast<const double2*>(Sc + (size_t)(l + u) * g.ldS);
#pragma unroll
          for (int h = 0; h < ANG_JB / 2; ++h) sv[u][h] = __ldg(Srow + h);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int h = 0; h < ANG_JB / 2; ++h) {
            acc[2 * h].x += sv[u][h].x * xv[u].x;     acc[2 * h].y += sv[u][h].x * xv[u].y;
            acc[2 * h + 1].x += sv[u][h].y * xv[u].x; acc[2 * h + 1].y += sv[u][h].y * xv[u].y;
          }
      }
      for (; l < n_l; ++l) {
        const double2 xv = xs[l * RT + lr];
        const double2* Srow = reinterpret_cast<const double2*>(Sc + (size_t)l * g.ldS);
#pragma unroll
        for (int h = 0; h < ANG_JB / 2; ++h) {
          const double2 sv = __ldg(Srow + h);
          acc[2 * h].x += sv.x * xv.x;     acc[2 * h].y += sv.x * xv.y;
          acc[2 * h + 1].x += sv.y * xv.x; acc[2 * h + 1].y += sv.y * xv.y;
        }
      }
#pragma unroll
      for (int q = 0; q < ANG_JB; ++q) {
        const int j = j0 + q;
        if (j < n_l) {
          double2 y = acc[q];
          // phase in the eigenbasis (couplingP.cuh:61-106 and twins)
          if (op.phase == PH_THETA && j >= m) {
            // the theta form: the whole angular potential at node x_j
            const double xj = Dv[j];
            double eta = (rr * E + v1) * xj + v2 * legendre_p2(xj) + v3 * legendre_p3(xj) + sbase;
            // n_har > 4: the multipoles L >= 1 at this node come from the exact-quadrature table
            if (g.theta_tab && rv) eta += run.htab[((size_t)m * n_l + j) * g.n_r + r];
            eta *= hdt;
            y = cmul_conj_phase(y, eta);
          } else if (op.phase != PH_NONE && j >= m) {
            double eta = base;
            eta *= hdt * Dv[j];
            y = cmul_conj_phase(y, eta);
          }
          if (last && ch.post_s) {
            double eta = sbase + pco[j] * v2;
            eta *= hdt;
            y = cmul_conj_phase(y, eta);
          }
          ys[j * RT + lr] = y;
          if constexpr (CL == 2) ys_peer[j * RT + lr] = y;
        }
      }
    }
    if constexpr (CL == 2) cg::this_cluster().sync();
    else __syncthreads();
    double2* t = xs; xs = ys; ys = t;
  }

  // both CTAs of a pair hold the whole result: each writes and reduces its share of l
  if (rv && xout)
    for (int l = gsub; l < n_l; l += CL * NSUB) xout[((size_t)l * g.n_cols + col) * g.n_r + r] = xs[l * RT + lr];

  if (do_obs) {
    const double fr2 = rv ? pow(rr, -2.0) : 0.0;
    observables_tile<double2, RT>(g, xs, col, m, tile * RT, lr, gsub, CL * NSUB, rr, fr2);
    const int n_den = g.n_den > 0 ? g.n_den : 1;  // L = 0 is always needed for the norm
    for (int L = gsub; L < n_den; L += CL * NSUB) {
      const double d = density_multipole<double2, RT>(L, m, n_l, xs, lr, g.coef, g.n_m);
      if (rv) g.dens[((size_t)col * N_DEN + L) * g.n_r + r] = d;
    }
  }
}

size_t angular_smem_fp64(int n_l) { return 2 * (size_t)n_l * TR * sizeof(double2); }

static int g_angular_sms = 148;

template <int RT>
static void launch_angular_rt(const GroupArgs& g, int half, const double2* xin, double2* xout, int do_obs,
                              cudaStream_t s) {
  const int tiles = g.n_cols * ((g.n_r + RT - 1) / RT);
  const size_t smem = 2 * (size_t)g.n_l * RT * sizeof(double2);
  if (tiles >= 2 * g_angular_sms) {
    k_angular_fp64<RT, 1><<<tiles, ANG_WARPS * 32, smem, s>>>(g, half, xin, xout, do_obs);
    return;
  }
  // too few tiles to fill the GPU: a CTA pair per tile
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2 * tiles);
  cfg.blockDim = dim3(ANG_WARPS * 32);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k_angular_fp64<RT, 2>, g, half, xin, xout, do_obs);
}

void launch_angular_fp64(const GroupArgs& g, int half, const double2* xin, double2* xout, int do_obs,
                         cudaStream_t s) {
  if (g.obs_seg == 16) launch_angular_rt<16>(g, half, xin, xout, do_obs, s);
  else launch_angular_rt<TR>(g, half, xin, xout, do_obs, s);
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
    // consumers: thread t computes output radius i0 + t for the tile's TC columns
    const int t = threadIdx.x;
    int it = 0;
    for (int tile = blockIdx.x; tile < total; tile += gridDim.x) {
      const int ct = tile % n_ct, rest = tile / n_ct, itile = rest % n_it, l = rest / n_it;
      const int i0 = itile * RAD_TI;
      const int c0 = ct * TC, nc = min(TC, n_cols - c0);
      double2 acc[TC];
#pragma unroll
      for (int c = 0; c < TC; ++c) acc[c] = make_double2(0.0, 0.0);
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
        if (kn == RAD_KC) {
#pragma unroll 4
          for (int kk = 0; kk < RAD_KC; ++kk) {
            const double2 w = ws[kk * RAD_TI + t];
#pragma unroll
            for (int c = 0; c < TC; ++c) {
              const double2 x = xs[c * RAD_KC + kk];
              acc[c].x = fma(w.x, x.x, fma(-w.y, x.y, acc[c].x));
              acc[c].y = fma(w.x, x.y, fma(w.y, x.x, acc[c].y));
            }
          }
        } else {
          for (int kk = 0; kk < kn; ++kk) {
            const double2 w = ws[kk * RAD_TI + t];
#pragma unroll
            for (int c = 0; c < TC; ++c) {
              const double2 x = xs[c * RAD_KC + kk];
              acc[c].x = fma(w.x, x.x, fma(-w.y, x.y, acc[c].x));
              acc[c].y = fma(w.x, x.y, fma(w.y, x.x, acc[c].y));
            }
          }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty_bar[s]);
      }
      if (!ok) break;
      const int i = i0 + t;
      if (i < n_r)
#pragma unroll
        for (int c = 0; c < TC; ++c)
          if (c < nc) xout[((size_t)l * n_cols + c0 + c) * n_r + i] = acc[c];
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
// the exchange potential) + 1 observables block.  mode 0 = initial potentials (no observables,
// no step increment), mode 1 = end of step, mode 2 = end of step without observables or step
// increment (profiling).
__global__ void __launch_bounds__(FIN_THREADS) k_finalize(GroupArgs g, int mode) {
  extern __shared__ double fsm[];  // [3][N_r]
  __shared__ dd wsum[FIN_THREADS / 32];
  const int nb = g.n_den + 1;
  const int ri = blockIdx.x / nb;
  const int role = blockIdx.x - ri * nb;  // < n_den: Hartree L = role; == n_den: observables
  const int run_idx = g.runs_of_group[ri];
  RunDev run = g.runs[run_idx];
  const int n_r = g.n_r, n_l = g.n_l, tid = threadIdx.x;
  const int step = *g.step;
  const bool obs_block = (role == g.n_den);

  if (obs_block && mode == 1) {
    if (step >= run.n_t) {
      if (tid == 0) atomicOr(g.status, ST_STEP_OVERFLOW);
    } else {
      const int n_orb = run.n_orb;
      // per (l, orbital): compensated sum over r tiles
      for (int idx = tid; idx < n_l * n_orb; idx += FIN_THREADS) {
        const int l = idx / n_orb, k = idx - l * n_orb;
        const double4* p = g.obs + 2 * (((size_t)(run.col0 + k) * n_l + l) * g.n_tiles);
        dd sx{0.0, 0.0}, sy{0.0, 0.0}, sz{0.0, 0.0}, sw{0.0, 0.0};
        for (int t = 0; t < g.n_tiles; ++t) {
          const double4 h = p[2 * t], lo = p[2 * t + 1];
          sx = dd_add(sx, dd{h.x, lo.x}); sy = dd_add(sy, dd{h.y, lo.y});
          sz = dd_add(sz, dd{h.z, lo.z}); sw = dd_add(sw, dd{h.w, lo.w});
        }
        if (g.per_l) {
          run.dip[((size_t)l * n_orb + k) * run.n_t + step] = make_double2(sx.hi + sx.lo, sy.hi + sy.lo);
          run.acc[((size_t)l * n_orb + k) * run.n_t + step] = make_double2(sz.hi + sz.lo, sw.hi + sw.lo);
        }
      }
      // per orbital: totals over l and the norm; one warp per orbital
      const int lane = tid & 31, warp = tid >> 5;
      for (int k = warp; k < n_orb; k += FIN_THREADS / 32) {
        const double4* p = g.obs + 2 * ((size_t)(run.col0 + k) * n_l * g.n_tiles);
        dd sx{0.0, 0.0}, sy{0.0, 0.0}, sz{0.0, 0.0}, sw{0.0, 0.0};
        for (int q = lane; q < n_l * g.n_tiles; q += 32) {
          const double4 h = p[2 * q], lo = p[2 * q + 1];
          sx = dd_add(sx, dd{h.x, lo.x}); sy = dd_add(sy, dd{h.y, lo.y});
          sz = dd_add(sz, dd{h.z, lo.z}); sw = dd_add(sw, dd{h.w, lo.w});
        }
        sx = warp_sum_dd2(sx); sy = warp_sum_dd2(sy); sz = warp_sum_dd2(sz); sw = warp_sum_dd2(sw);
        const double* dn = g.dens + (size_t)(run.col0 + k) * N_DEN * n_r;  // L = 0 row
        dd nd{0.0, 0.0};
        for (int q = lane; q < n_r; q += 32) nd = dd_add(nd, dd{dn[q], 0.0});
        nd = warp_sum_dd2(nd);
        const double nrm = nd.hi + nd.lo;
        if (lane == 0) {
          run.dip_tot[(size_t)k * run.n_t + step] = make_double2(sx.hi + sx.lo, sy.hi + sy.lo);
          run.acc_tot[(size_t)k * run.n_t + step] = make_double2(sz.hi + sz.lo, sw.hi + sw.lo);
          run.norm[(size_t)k * run.n_t + step] = nrm;
          if (!(nrm == nrm) || isinf(nrm) || !(sx.hi == sx.hi) || !(sz.hi == sz.hi)) atomicOr(g.status, ST_NAN);
          if (nrm > run.norm0[k] * (1.0 + g.norm_tol) + 1e-300) atomicOr(g.status, ST_NORM_GROWTH);
        }
      }
    }
  } else if (obs_block && mode == 0) {
    // initial norm for the growth watchdog
    const int lane = tid & 31, warp = tid >> 5;
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

  // exchange (block L = 0, or the observables block when Hartree is off)
  const bool xc_block = (g.n_den > 0) ? (role == 0) : obs_block;
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
  const dim3 grid(g.n_runs * (g.n_den + 1)), block(FIN_THREADS);
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
  e = set_max_dynamic_smem((const void*)k_angular_fp64<TR, 1>, optin);
  if (e != cudaSuccess) return e;
  e = set_max_dynamic_smem((const void*)k_angular_fp64<16, 1>, optin);
  if (e != cudaSuccess) return e;
  e = set_max_dynamic_smem((const void*)k_angular_fp64<TR, 2>, optin);
  if (e != cudaSuccess) return e;
  e = set_max_dynamic_smem((const void*)k_angular_fp64<16, 2>, optin);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&g_angular_sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  e = configure_radial_fp64();
  if (e != cudaSuccess) return e;
  return set_max_dynamic_smem((const void*)k_finalize, optin);
}

}  // namespace ggb
