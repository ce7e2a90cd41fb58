// Angular half-step on tcgen05 tensor cores (split-precision form).
//
// One CTA owns 64 radii (points) of one orbital column and keeps the whole l-vector of each point
// resident in shared memory as the K-major B operand: two BF16 planes (hi, lo) of 128 rows, rows
// 0-63 the real parts of the 64 points and rows 64-127 their imaginary parts, so that one MMA with
// N = 128 produces Re and Im together.  Every product of the chain (rotate into a coupling's
// eigenbasis, pre-multiplied rotation pairs, rotate back; see k_angular_fp64) is
//     D[j][n] = sum_l S^T[j][l] X[n][l]          (M = j, N = 128 = 64 points x {Re, Im}, K = l)
// with A = S^T streamed by TMA (three BF16 planes hi/mid/lo, one plane per pipeline stage, 128-byte
// swizzle, L2 resident: every CTA of the group reads the same matrices) and the Re/Im accumulators
// in tensor memory; the split products S_h X_h + S_h X_l + S_m X_h + S_m X_l + S_l X_h are
// accumulated in FP32 (a three-term S keeps the fixed non-unitarity of the rounded chain matrices,
// which compounds step after step, at ~2^-25).  The epilogue warps read the
// accumulators (one TMEM lane = one eigen-channel j), apply the coupling's phase
// exp(-i eta(r) dt/2 D[j]) (and the l-diagonal S phase after the last product of the first half),
// split the result into BF16 hi/lo and write it back as the next product's operand.  The last
// product is staged in FP32 in shared memory and stored coalesced: as the radial B operand planes
// (first half) or as complex64 orbitals (second half; the FP64 density and dipole partial sums of the
// new orbitals are taken by the light k_angular_f32 pass that follows, so this kernel stays small
// enough for two CTAs per SM, one CTA's epilogue overlapping the other's MMAs).
//
// Warp roles: warp 0 TMA producer, warp 1 MMA issuer (+ TMEM allocation), warps 2-9 epilogue.
#include <cuda_bf16.h>

#include "ggb_angular.cuh"
#include "ggb_mixed.cuh"
#include "ggb_tc_common.cuh"

namespace ggb {

constexpr int AT_NP = 64;               // points per CTA (MMA N)
constexpr int AT_THREADS = 320;         // 10 warps
constexpr int AT_EPI_WARP0 = 2;
constexpr int AT_KATOM = 64;            // BF16 elements per 128-byte swizzled row
constexpr int AT_A_TILE = 128 * 128;    // bytes of one 128-row x 64-k plane tile of S^T (one stage)
constexpr int AT_S_PLANES = 3;          // S^T hi, mid, lo
constexpr int AT_NB = 2 * AT_NP;        // B rows: Re of 64 points, then Im
constexpr int AT_B_TILE = AT_NB * 128;  // bytes of one 128-row x 64-k plane tile of x

struct AngTcArgs {
  CUtensorMap tmS;        // S^T planes: dims (l, j, plane, m, mat)
  int k_atoms;            // K extent / 64
  int m_tiles;            // ceil(N_l / 128)
  int k_slices;           // ceil(N_l / 16): 16-wide K slices that carry data
  int stages;
  int k_pad;              // radial B operand row length
  int cols_pad;
  __nv_bfloat16* xsp;     // radial B operand (first-half output)
};

// byte offset of element (row p, k) inside a K-major 128-byte-swizzled tile of 64-element rows
__device__ __forceinline__ uint32_t sw128_off(int p, int k) {
  const int chunk = ((k & 63) >> 3) ^ (p & 7);
  return (uint32_t)(p * 128 + chunk * 16 + (k & 7) * 2);
}

// x * exp(-i eta) with the accurate FP32 sine and cosine: their rounding is not correlated from one
// step to the next, whereas the systematic error of the SFU approximation makes |exp(-i eta)| != 1
// in the same direction every step and compounds.
__device__ __noinline__ void sincos_acc(float e, float* s, float* c) { sincosf(e, s, c); }

__device__ __forceinline__ float2 rot(float2 x, float e) {
  float s, c;
  sincos_acc(e, &s, &c);
  return make_float2(c * x.x + s * x.y, c * x.y - s * x.x);
}

// Store x_k(p) as BF16 hi/lo: Re in row p, Im in row 64 + p of the hi plane and of the lo plane.
__device__ __forceinline__ void split_put(uint8_t* xb, int k_atoms, int p, int k, float2 v) {
  const __nv_bfloat16 rh = __float2bfloat16_rn(v.x), ih = __float2bfloat16_rn(v.y);
  const __nv_bfloat16 rl = __float2bfloat16_rn(v.x - __bfloat162float(rh));
  const __nv_bfloat16 il = __float2bfloat16_rn(v.y - __bfloat162float(ih));
  const uint32_t atom = (uint32_t)(k >> 6) * AT_B_TILE;
  const uint32_t o_re = atom + sw128_off(p, k), o_im = atom + sw128_off(p + AT_NP, k);
  const uint32_t plane = (uint32_t)k_atoms * AT_B_TILE;
  *reinterpret_cast<__nv_bfloat16*>(xb + o_re) = rh;
  *reinterpret_cast<__nv_bfloat16*>(xb + o_im) = ih;
  *reinterpret_cast<__nv_bfloat16*>(xb + plane + o_re) = rl;
  *reinterpret_cast<__nv_bfloat16*>(xb + plane + o_im) = il;
}

template <bool SECOND_HALF>
__global__ void __launch_bounds__(AT_THREADS, 2)
k_angular_tc(const __grid_constant__ CUtensorMap tmS, GroupArgs g, AngTcArgs t, const float2* __restrict__ xin,
             float2* __restrict__ xout) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ uint64_t full_bar[4], empty_bar[4], acc_bar, xb_bar, drain_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  __shared__ float pbase[5][AT_NP];     // per point: r, (r E + v1 or r E) dt/2, v2 dt/2, v3 dt/2, S base dt/2
  // aligned by an offset from the __shared__ array itself, so that the compiler keeps the shared
  // address space (shared loads and stores, not generic ones) for every access through it
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint8_t* xb = smem;                                            // 2 planes x k_atoms x 16 KB
  uint8_t* sst = smem + (size_t)2 * t.k_atoms * AT_B_TILE;       // stages x 32 KB (later: FP32 staging)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_l = g.n_l;
  const int tiles64 = (g.n_r + AT_NP - 1) / AT_NP;
  const int col = blockIdx.x / tiles64;
  const int r0 = (blockIdx.x - col * tiles64) * AT_NP;
  const int m = g.col_m[col];
  const RunDev run = g.runs[g.col_run[col]];
  const Chain& ch = g.chain[SECOND_HALF ? 1 : 0];
  const int n_ops = ch.n_ops;
  const int tmem_cols = 128 * t.m_tiles;
  int step = *g.step;
  if (step >= run.n_t) step = run.n_t - 1;
  const double hdt = 0.5 * g.dt;
  const double* pco = g.coef + ((size_t)CF_P * g.n_m + m) * n_l;

  if (threadIdx.x == 0) {
    for (int s = 0; s < t.stages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&acc_bar, 1);
    mbar_init(&xb_bar, AT_THREADS / 32 - AT_EPI_WARP0);
    mbar_init(&drain_bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(&tmem_slot, tmem_cols);

  // per-point potentials (FP64)
  if (threadIdx.x < AT_NP) {
    const int p = threadIdx.x, r = r0 + p;
    const bool rv = r < g.n_r;
    const int rc = rv ? r : 0;
    const double rr = rv ? g.r[r] : 1.0, E = run.E[step];
    double v1 = 0.0, v2 = 0.0, v3 = 0.0, sb = 0.0;
    if (g.hartree_on) {
      v1 = run.v[1 * g.n_r + rc];
      v2 = run.v[2 * g.n_r + rc];
      v3 = run.v[3 * g.n_r + rc];
      sb = run.v[rc] - run.v0[rc] + run.vexc[rc] - run.vexc0[rc];
    }
    pbase[0][p] = (float)rr;
    pbase[1][p] = (float)((g.p_hartree ? (rr * E + v1) : (rr * E)) * hdt);
    pbase[2][p] = (float)(v2 * hdt);
    pbase[3][p] = (float)(v3 * hdt);
    pbase[4][p] = (float)(sb * hdt);
  }
  __syncthreads();

  // operand: x tile (all l, 64 points), [second half: l-diagonal S phase], split into BF16 planes
  const int lk = t.k_atoms * AT_KATOM;
  {
    // eight independent loads in flight per thread, then split and store
    constexpr int U = 8;
    for (int base = threadIdx.x; base < lk * AT_NP; base += U * AT_THREADS) {
      float2 v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int idx = base + u * AT_THREADS;
        const int l = idx / AT_NP, p = idx - l * AT_NP, r = r0 + p;
        v[u] = (idx < lk * AT_NP && l < n_l && r < g.n_r) ? __ldcg(xin + ((size_t)l * g.n_cols + col) * g.n_r + r)
                                                        : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int idx = base + u * AT_THREADS;
        if (idx < lk * AT_NP) {
          const int l = idx / AT_NP, p = idx - l * AT_NP;
          float2 w = v[u];
          if (SECOND_HALF && ch.pre_s && l < n_l) w = rot(w, pbase[4][p] + (float)pco[l] * pbase[2][p]);
          split_put(xb, t.k_atoms, p, l, w);
        }
      }
    }
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  volatile int* abort_p = &abort_flag;

  if (warp == 0) {
    // ---------------- producer: S^T tiles of every product, in consumption order
    if (lane == 0) {
      int it = 0;
      bool ok = true;
      for (int o = 0; o < n_ops && ok; ++o) {
        const int mat = ch.ops[o].mat;
        for (int mt = 0; mt < t.m_tiles && ok; ++mt)
          for (int ka = 0; ka < t.k_atoms && ok; ++ka)
            for (int pl = 0; pl < AT_S_PLANES; ++pl, ++it) {
              const int s = it % t.stages;
              if (it >= t.stages && !mbar_wait(&empty_bar[s], ((it / t.stages) & 1) ^ 1, abort_p)) {
                ok = false;
                break;
              }
              mbar_expect_tx(&full_bar[s], AT_A_TILE);
              tma_load_5d(sst + (size_t)s * AT_A_TILE, &tmS, ka * AT_KATOM, mt * 128, pl, m, mat, &full_bar[s]);
            }
      }
      if (!ok) {
        // drain: every stage issued but not consumed must land before the CTA exits
        for (int q = (it > t.stages ? it - t.stages : 0); q < it; ++q) mbar_drain(&full_bar[q % t.stages], (q / t.stages) & 1);
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16_mn(128, AT_NB, false);
      const uint32_t xplane = (uint32_t)t.k_atoms * AT_B_TILE;
      const uint32_t sxb = smem_u32(xb);
      int it = 0;
      for (int o = 0; o < n_ops; ++o) {
        if (o > 0 && !mbar_wait(&xb_bar, (o - 1) & 1, abort_p)) break;
        tc_fence_after();
        bool ok = true;
        for (int mt = 0; mt < t.m_tiles && ok; ++mt) {
          const uint32_t d = tmem + 128 * mt;      // columns [0,64) Re, [64,128) Im
          for (int ka = 0; ka < t.k_atoms && ok; ++ka)
            for (int pl = 0; pl < AT_S_PLANES; ++pl, ++it) {
              const int s = it % t.stages;
              if (!mbar_wait(&full_bar[s], (it / t.stages) & 1, abort_p)) {
                ok = false;
                break;
              }
              tc_fence_after();
              const uint32_t sa = smem_u32(sst + (size_t)s * AT_A_TILE);
#pragma unroll
              for (int kk = 0; kk < 4; ++kk) {
                const int slice = ka * 4 + kk;
                if (slice >= t.k_slices) break;
                const uint32_t ko = kk * 32;
                const uint64_t a = sdesc_kmajor(sa + ko, 128, 2);
                const uint32_t bx = sxb + ka * AT_B_TILE + ko;
                const uint64_t bh = sdesc_kmajor(bx, 128, 2), bl = sdesc_kmajor(bx + xplane, 128, 2);
                // S_h X_h + S_h X_l + S_m X_h + S_m X_l + S_l X_h
                tc_mma(d, a, bh, idesc, (slice > 0 || pl > 0) ? 1u : 0u);
                if (pl < 2) tc_mma(d, a, bl, idesc, 1u);
              }
              tc_commit(&empty_bar[s]);
            }
        }
        tc_commit(&acc_bar);   // completes when every MMA of this product is done
        if (!ok) break;
      }
    }
  } else {
    // ---------------- epilogue warps 2..9
    const int ew = warp - AT_EPI_WARP0;         // 0..7
    const int q = warp & 3;                     // TMEM lane quarter this warp may access
    const int grp = ew >> 2;                    // 0 or 1
    // [N_l][64] FP32 staging of the last product: the operand and stage buffers are free once its
    // MMAs have completed
    float2* stage_out = reinterpret_cast<float2*>(smem);
    for (int o = 0; o < n_ops; ++o) {
      const bool ok = mbar_wait(&acc_bar, o & 1, abort_p);
      tc_fence_after();
      if (!ok) break;
      const ChainOp op = ch.ops[o];
      const bool last = (o == n_ops - 1);
      const double* Dv = g.dph + ((size_t)op.coupling * g.n_m + m) * g.ldS;
      // this thread's eigen-channel and points
      const int mt = (t.m_tiles == 2) ? grp : 0;
      const int j = 128 * mt + 32 * q + lane;
      const int p_begin = (t.m_tiles == 2) ? 0 : 32 * grp;
      const int p_end = (t.m_tiles == 2) ? AT_NP : 32 * grp + 32;
      const float dj = (op.phase != PH_NONE && j >= m && j < n_l) ? (float)Dv[j] : 0.f;
      const int pb = op.phase == PH_P ? 1 : op.phase == PH_D ? 2 : 3;
      const bool post_s = last && !SECOND_HALF && ch.post_s && j < n_l;
      const float pj = post_s ? (float)pco[j] : 0.f;
      const uint32_t lane_base = (uint32_t)(32 * q) << 16;
      for (int p0 = p_begin; p0 < p_end; p0 += 16) {
        uint32_t re[16], im[16];
        tmem_ld16(tmem + lane_base + 128 * mt + p0, re);
        tmem_ld16(tmem + lane_base + 128 * mt + AT_NP + p0, im);
        tmem_ld_wait();
        tmem_regs_ready(re);
        tmem_regs_ready(im);
#pragma unroll
        for (int u = 0; u < 16; ++u) {
          const int p = p0 + u;
          float2 v = make_float2(__uint_as_float(re[u]), __uint_as_float(im[u]));
          if (dj != 0.f) v = rot(v, pbase[pb][p] * dj);
          if (post_s) v = rot(v, pbase[4][p] + pj * pbase[2][p]);
          if (!last) {
            if (j < lk) split_put(xb, t.k_atoms, p, j, v);
          } else if (j < n_l) {
            stage_out[(size_t)j * AT_NP + p] = v;
          }
        }
      }
      tc_fence_before();
      if (!last) {
        fence_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(&xb_bar);
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (abort_flag) {
    if (threadIdx.x == 0) atomicOr(g.status, ST_TC_TIMEOUT);
  } else {
    // ---------------- outputs of the last product, coalesced along r
    const float2* xs = reinterpret_cast<const float2*>(smem);
    if (!SECOND_HALF) {
      const size_t plane = (size_t)t.cols_pad * t.k_pad;
      for (int idx = threadIdx.x; idx < n_l * AT_NP; idx += AT_THREADS) {
        const int l = idx / AT_NP, p = idx - l * AT_NP, r = r0 + p;
        if (r < g.n_r) {
          const float2 v = xs[idx];
          const __nv_bfloat16 rh = __float2bfloat16_rn(v.x), ih = __float2bfloat16_rn(v.y);
          __nv_bfloat16* b = t.xsp + (size_t)l * 4 * plane + (size_t)col * t.k_pad + r;
          b[0] = rh;
          b[plane] = __float2bfloat16_rn(v.x - __bfloat162float(rh));
          b[2 * plane] = ih;
          b[3 * plane] = __float2bfloat16_rn(v.y - __bfloat162float(ih));
        }
      }
    } else {
      for (int idx = threadIdx.x; idx < n_l * AT_NP; idx += AT_THREADS) {
        const int l = idx / AT_NP, p = idx - l * AT_NP, r = r0 + p;
        if (r < g.n_r) xout[((size_t)l * g.n_cols + col) * g.n_r + r] = xs[idx];
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    if (abort_flag && lane == 0) {
      // every MMA this thread issued must be complete before TMEM is released
      tc_commit(&drain_bar);
      mbar_drain(&drain_bar, 0);
    }
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, tmem_cols);
  }
}

// ---------------------------------------------------------------------------------------------

static size_t angular_tc_smem(int k_atoms, int stages) {
  return (size_t)2 * k_atoms * AT_B_TILE + (size_t)stages * AT_A_TILE + 1024;
}

int angular_tc_config(int n_l, int& k_atoms, int& m_tiles, int& stages, size_t& smem) {
  k_atoms = (n_l + AT_KATOM - 1) / AT_KATOM;
  m_tiles = (n_l + 127) / 128;
  if (m_tiles > 2) return -1;
  const int optin_budget = 227 * 1024 - 4096;
  // two CTAs per SM when they fit (one CTA's epilogue overlaps the other's MMAs), else deep pipelining
  const int pair_budget = 113 * 1024 - 4096;
  stages = 2;
  while (stages < 4 && angular_tc_smem(k_atoms, stages + 1) <= (size_t)pair_budget) ++stages;
  if (angular_tc_smem(k_atoms, stages) > (size_t)pair_budget) {
    stages = 4;
    while (stages > 2 && angular_tc_smem(k_atoms, stages) > (size_t)optin_budget) --stages;
  }
  // the FP32 staging of the last product reuses the operand and stage buffers: N_l x 64 x 8 bytes
  if ((size_t)n_l * AT_NP * 8 > angular_tc_smem(k_atoms, stages) - 1024) return -1;
  smem = angular_tc_smem(k_atoms, stages);
  if (smem > (size_t)optin_budget) return -1;
  return 0;
}

cudaError_t angular_tc_configure() {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaError_t e = set_max_dynamic_smem((const void*)k_angular_tc<false>, optin);
  if (e != cudaSuccess) return e;
  return set_max_dynamic_smem((const void*)k_angular_tc<true>, optin);
}

void launch_angular_tc(const MixedGroup& mg, const GroupArgs& a, int half, const float2* xin, float2* xout,
                       cudaStream_t s) {
  AngTcArgs t;
  t.k_atoms = mg.at_k_atoms;
  t.m_tiles = mg.at_m_tiles;
  t.k_slices = (a.n_l + 15) / 16;
  t.stages = mg.at_stages;
  t.k_pad = mg.k_pad;
  t.cols_pad = mg.cols_pad;
  t.xsp = mg.Xsp;
  const dim3 grid(a.n_cols * ((a.n_r + AT_NP - 1) / AT_NP));
  if (half == 0) k_angular_tc<false><<<grid, AT_THREADS, mg.at_smem, s>>>(mg.tmS, a, t, xin, xout);
  else k_angular_tc<true><<<grid, AT_THREADS, mg.at_smem, s>>>(mg.tmS, a, t, xin, xout);
}

}  // namespace ggb
