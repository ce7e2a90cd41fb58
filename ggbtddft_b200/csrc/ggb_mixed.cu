// Split-precision form of the step.
//
//  k_split_w        one-time: W[l][k][i] (complex128) -> A(i,k) = W[l][k][i] as six BF16 planes
//                   (Wr hi, mid, lo, Wi hi, mid, lo: three terms, residual 2^-25 of |W|), K-major,
//                   zero padded, for TMA.  Three terms, because W is applied every step: a 2^-17
//                   representation error of a constant unitary operator is a fixed non-unitarity that
//                   compounds over tens of thousands of steps, while the rounding of the (changing)
//                   orbitals only random-walks.
//  k_angular_f32    the angular half-step chain of k_angular_fp64 in FP32 on complex64 orbitals;
//                   the first half writes the radial B operand directly as BF16 hi/lo planes, the
//                   second half keeps the FP64 density/dipole partial sums of the FP64 form.
//  k_radial_tc      x_l <- A_l x_l on tcgen05: TMA-staged tiles (128 radii x 32 k per plane),
//                   split products W_h x_h + W_h x_l + W_m x_h + W_m x_l + W_l x_h (only W_l x_l,
//                   ~2^-24, dropped) for each of the four real products of the complex GEMM, the
//                   -Wi Xi term through the A-negate bit of the instruction descriptor, FP32
//                   accumulators Re/Im in tensor memory.
//  The potentials/observables kernel (k_finalize) is shared with the FP64 form.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include "../../include/ggbtddft.h"
#include "ggb_angular.cuh"
#include "ggb_mixed.cuh"
#include "ggb_tc_common.cuh"

namespace ggb {

// ---------------------------------------------------------------------------------------------
// conversions
// ---------------------------------------------------------------------------------------------

__device__ __forceinline__ void split_bf16(double v, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __double2bfloat16(v);
  lo = __double2bfloat16(v - (double)__bfloat162float(hi));
}
__device__ __forceinline__ void split3_bf16(double v, __nv_bfloat16& hi, __nv_bfloat16& mid, __nv_bfloat16& lo) {
  hi = __double2bfloat16(v);
  const double r1 = v - (double)__bfloat162float(hi);
  mid = __double2bfloat16(r1);
  lo = __double2bfloat16(r1 - (double)__bfloat162float(mid));
}
__device__ __forceinline__ void split_bf16f(float v, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(v);
  lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

constexpr int W_PLANES = 6;   // Wr hi, mid, lo, Wi hi, mid, lo
constexpr int S_PLANES = 3;   // S^T hi, mid, lo

// 32x32 tiles through shared memory: read W[l][k][i] along i, write A(i,k) along k.
__global__ void k_split_w(const double2* __restrict__ W, __nv_bfloat16* __restrict__ Wsp, int n_r, int rows_pad,
                          int k_pad) {
  __shared__ double2 t[32][33];
  const int l = blockIdx.z;
  const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int q = ty; q < 32; q += 8) {
    const int k = k0 + q, i = i0 + tx;
    t[q][tx] = (k < n_r && i < n_r) ? W[((size_t)l * n_r + k) * n_r + i] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  const size_t plane = (size_t)rows_pad * k_pad;
  __nv_bfloat16* base = Wsp + (size_t)l * W_PLANES * plane;
  for (int q = ty; q < 32; q += 8) {
    const int i = i0 + q, k = k0 + tx;
    if (i < rows_pad && k < k_pad) {
      const double2 w = t[tx][q];
      __nv_bfloat16 rh, rm, rl, ih, im, il;
      split3_bf16(w.x, rh, rm, rl);
      split3_bf16(w.y, ih, im, il);
      const size_t o = (size_t)i * k_pad + k;
      base[o] = rh;
      base[plane + o] = rm;
      base[2 * plane + o] = rl;
      base[3 * plane + o] = ih;
      base[4 * plane + o] = im;
      base[5 * plane + o] = il;
    }
  }
}

// S^T planes for the tensor-core angular chain: St[mat][m][plane][j][l] = 3-term split of S[mat][m][l][j],
// zero for j >= N_l or l >= N_l.
__global__ void k_build_st(const double* __restrict__ mats, __nv_bfloat16* __restrict__ St, int n_mats, int n_m,
                           int n_l, int ldS, int rows, int lk) {
  const size_t total = (size_t)n_mats * n_m * rows * lk;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int l = (int)(i % lk);
    const int j = (int)((i / lk) % rows);
    const size_t mm = i / ((size_t)lk * rows);      // mat * n_m + m
    double v = 0.0;
    if (j < n_l && l < n_l) v = mats[(mm * n_l + l) * ldS + j];
    __nv_bfloat16 hi, mid, lo;
    split3_bf16(v, hi, mid, lo);
    const size_t plane = (size_t)rows * lk;
    St[mm * S_PLANES * plane + (size_t)j * lk + l] = hi;
    St[mm * S_PLANES * plane + plane + (size_t)j * lk + l] = mid;
    St[mm * S_PLANES * plane + 2 * plane + (size_t)j * lk + l] = lo;
  }
}

__global__ void k_d2f(const double2* __restrict__ a, float2* __restrict__ b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = make_float2((float)a[i].x, (float)a[i].y);
}
__global__ void k_f2d(const float2* __restrict__ a, double2* __restrict__ b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = make_double2((double)a[i].x, (double)a[i].y);
}
__global__ void k_d2f_real(const double* __restrict__ a, float* __restrict__ b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// ---------------------------------------------------------------------------------------------
// angular chain, FP32
// ---------------------------------------------------------------------------------------------

__device__ __forceinline__ float2 phase_f(float2 x, float eta) {
  float s, c;
  sincosf(eta, &s, &c);
  return make_float2(c * x.x + s * x.y, c * x.y - s * x.x);
}

struct MixArgs {
  const float* mats_f;
  int k_pad;
  int cols_pad;
  __nv_bfloat16* xsp;   // radial B operand (first half output)
};

constexpr int ANGF_JB = 8;

// OUT_SPLIT = true: write the radial B operand planes; false: write complex64 orbitals.
template <bool OUT_SPLIT>
__global__ void __launch_bounds__(ANG_WARPS * 32)
k_angular_f32(GroupArgs g, MixArgs mx, int half, const float2* __restrict__ xin, float2* __restrict__ xout,
              int do_obs) {
  extern __shared__ float2 smf[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int tiles32 = (g.n_r + TR - 1) / TR;     // this kernel's CTAs cover 32 radii each
  const int col = blockIdx.x / tiles32;
  const int tile = blockIdx.x - col * tiles32;
  const int r = tile * TR + lane;
  const bool rv = r < g.n_r;
  const int n_l = g.n_l;
  float2* xs = smf;
  float2* ys = smf + (size_t)n_l * TR;
  const int m = g.col_m[col];
  const RunDev run = g.runs[g.col_run[col]];
  int step = *g.step;
  if (step >= run.n_t) step = run.n_t - 1;

  for (int l = warp; l < n_l; l += ANG_WARPS)
    xs[l * TR + lane] = rv ? xin[((size_t)l * g.n_cols + col) * g.n_r + r] : make_float2(0.f, 0.f);

  const double rr = rv ? g.r[r] : 1.0;
  const int rc = rv ? r : 0;
  const double E = run.E[step];
  double v1 = 0.0, v2 = 0.0, v3 = 0.0, sbase = 0.0;
  if (g.hartree_on) {
    v1 = run.v[1 * g.n_r + rc];
    v2 = run.v[2 * g.n_r + rc];
    v3 = run.v[3 * g.n_r + rc];
    sbase = run.v[rc] - run.v0[rc] + run.vexc[rc] - run.vexc0[rc];
  }
  const double hdt = 0.5 * g.dt;
  const double* pco = g.coef + ((size_t)CF_P * g.n_m + m) * n_l;
  __syncthreads();

  const Chain& ch = g.chain[half];
  if (ch.pre_s) {
    for (int l = warp; l < n_l; l += ANG_WARPS)
      xs[l * TR + lane] = phase_f(xs[l * TR + lane], (float)((sbase + pco[l] * v2) * hdt));
    __syncthreads();
  }
  for (int o = 0; o < ch.n_ops; ++o) {
    const ChainOp op = ch.ops[o];
    const float* S = mx.mats_f + ((size_t)op.mat * g.n_m + m) * (size_t)n_l * g.ldS;
    const bool last = (o == ch.n_ops - 1);
    double base = 0.0;
    if (op.phase == PH_P) base = g.p_hartree ? (rr * E + v1) : (rr * E);
    else if (op.phase == PH_D) base = v2;
    else if (op.phase != PH_NONE) base = v3;
    const double* Dv = g.dph + ((size_t)op.coupling * g.n_m + m) * g.ldS;
    for (int j0 = warp * ANGF_JB; j0 < n_l; j0 += ANG_WARPS * ANGF_JB) {
      float2 acc[ANGF_JB];
#pragma unroll
      for (int q = 0; q < ANGF_JB; ++q) acc[q] = make_float2(0.f, 0.f);
      const float* Sc = S + j0;
      for (int l = m; l < n_l; ++l) {
        const float2 xv = xs[l * TR + lane];
        const float4* Srow = reinterpret_cast<const float4*>(Sc + (size_t)l * g.ldS);
#pragma unroll
        for (int h = 0; h < ANGF_JB / 4; ++h) {
          const float4 sv = __ldg(Srow + h);
          acc[4 * h].x += sv.x * xv.x;     acc[4 * h].y += sv.x * xv.y;
          acc[4 * h + 1].x += sv.y * xv.x; acc[4 * h + 1].y += sv.y * xv.y;
          acc[4 * h + 2].x += sv.z * xv.x; acc[4 * h + 2].y += sv.z * xv.y;
          acc[4 * h + 3].x += sv.w * xv.x; acc[4 * h + 3].y += sv.w * xv.y;
        }
      }
#pragma unroll
      for (int q = 0; q < ANGF_JB; ++q) {
        const int j = j0 + q;
        if (j < n_l) {
          float2 y = acc[q];
          if (op.phase != PH_NONE && j >= m) y = phase_f(y, (float)(base * (hdt * Dv[j])));
          if (last && ch.post_s) y = phase_f(y, (float)((sbase + pco[j] * v2) * hdt));
          ys[j * TR + lane] = y;
        }
      }
    }
    __syncthreads();
    float2* t = xs; xs = ys; ys = t;
  }

  if (OUT_SPLIT) {
    // radial B operand: planes [l][p][col][k_pad] (re hi, re lo, im hi, im lo)
    if (rv) {
      const size_t plane = (size_t)mx.cols_pad * mx.k_pad;
      for (int l = warp; l < n_l; l += ANG_WARPS) {
        const float2 v = xs[l * TR + lane];
        __nv_bfloat16 rh, rl, ih, il;
        split_bf16f(v.x, rh, rl);
        split_bf16f(v.y, ih, il);
        __nv_bfloat16* b = mx.xsp + (size_t)l * 4 * plane + (size_t)col * mx.k_pad + r;
        b[0] = rh;
        b[plane] = rl;
        b[2 * plane] = ih;
        b[3 * plane] = il;
      }
    }
  } else if (rv && xout) {
    for (int l = warp; l < n_l; l += ANG_WARPS) xout[((size_t)l * g.n_cols + col) * g.n_r + r] = xs[l * TR + lane];
  }

  if (do_obs) {
    const double fr2 = rv ? pow(rr, -2.0) : 0.0;
    observables_tile(g, xs, col, m, tile * TR, lane, warp, ANG_WARPS, rr, fr2);
    const int n_den = g.n_den > 0 ? g.n_den : 1;
    for (int L = warp; L < n_den; L += ANG_WARPS) {
      const double d = density_multipole(L, m, n_l, xs, lane, g.coef, g.n_m);
      if (rv) g.dens[((size_t)col * N_DEN + L) * g.n_r + r] = d;
    }
  }
}

static size_t angular_smem_f32(int n_l) { return 2 * (size_t)n_l * TR * sizeof(float2); }

// ---------------------------------------------------------------------------------------------
// radial propagator on tcgen05
// ---------------------------------------------------------------------------------------------

constexpr int RT_BM = 128;         // radii per tile (MMA M)
constexpr int RT_BK = 32;          // k per stage (64 bytes of BF16 per row: 64-byte swizzle)
constexpr int RT_THREADS = 192;    // warp 0 TMA, warp 1 MMA + TMEM, warps 2-5 epilogue
// Instruction descriptor of the radial product: M = 128 radii, N = n columns.
__host__ __device__ constexpr uint32_t idesc_bf16(int n, bool negate_a) { return idesc_bf16_mn(RT_BM, n, negate_a); }
// Shared-memory descriptor of the radial tiles: K-major, 64-byte swizzle, 64-byte rows.
__device__ __forceinline__ uint64_t sdesc_sw64(uint32_t saddr) { return sdesc_kmajor(saddr, 64, 4); }

template <int BN>
struct RadialTile {
  static constexpr int A_PLANE = RT_BM * RT_BK * 2;       // bytes of one plane tile of W
  static constexpr int B_PLANE = BN * RT_BK * 2;          // bytes of one plane tile of x
  static constexpr int A_STAGE = W_PLANES * A_PLANE;
  static constexpr int STAGE = A_STAGE + 4 * B_PLANE;
  static constexpr int TMEM_COLS = (2 * BN <= 32) ? 32 : (2 * BN <= 64) ? 64 : (2 * BN <= 128) ? 128 : (2 * BN <= 256) ? 256 : 512;
};

// The MMAs of one 32-wide k block of the radial product into D_re / D_im:
//   Re += Wr Xr - Wi Xi,  Im += Wr Xi + Wi Xr,  each real product W X as
//   W_h X_h + W_h X_l + W_m X_h + W_m X_l + W_l X_h  (W in three BF16 terms, X in two).
template <int BN>
__device__ __forceinline__ void radial_mma_kblock(uint32_t sa, uint32_t sb, uint32_t d_re, uint32_t d_im,
                                                  bool first, uint32_t a_plane, uint32_t b_plane) {
  const uint32_t id_pos = idesc_bf16(BN, false), id_neg = idesc_bf16(BN, true);
#pragma unroll
  for (int kk = 0; kk < RT_BK / 16; ++kk) {
    const uint32_t ko = kk * 32;  // 16 BF16 = 32 bytes along k
    uint64_t w[W_PLANES], x[4];
#pragma unroll
    for (int p = 0; p < W_PLANES; ++p) w[p] = sdesc_sw64(sa + p * a_plane + ko);
#pragma unroll
    for (int p = 0; p < 4; ++p) x[p] = sdesc_sw64(sb + p * b_plane + ko);
    const uint32_t acc0 = (!first || kk > 0) ? 1u : 0u;
    // w: 0-2 Wr (h, m, l), 3-5 Wi (h, m, l);  x: 0 Xr h, 1 Xr l, 2 Xi h, 3 Xi l
    tc_mma(d_re, w[0], x[0], id_pos, acc0);
    tc_mma(d_re, w[0], x[1], id_pos, 1u);
    tc_mma(d_re, w[1], x[0], id_pos, 1u);
    tc_mma(d_re, w[1], x[1], id_pos, 1u);
    tc_mma(d_re, w[2], x[0], id_pos, 1u);
    tc_mma(d_re, w[3], x[2], id_neg, 1u);
    tc_mma(d_re, w[3], x[3], id_neg, 1u);
    tc_mma(d_re, w[4], x[2], id_neg, 1u);
    tc_mma(d_re, w[4], x[3], id_neg, 1u);
    tc_mma(d_re, w[5], x[2], id_neg, 1u);
    tc_mma(d_im, w[0], x[2], id_pos, acc0);
    tc_mma(d_im, w[0], x[3], id_pos, 1u);
    tc_mma(d_im, w[1], x[2], id_pos, 1u);
    tc_mma(d_im, w[1], x[3], id_pos, 1u);
    tc_mma(d_im, w[2], x[2], id_pos, 1u);
    tc_mma(d_im, w[3], x[0], id_pos, 1u);
    tc_mma(d_im, w[3], x[1], id_pos, 1u);
    tc_mma(d_im, w[4], x[0], id_pos, 1u);
    tc_mma(d_im, w[4], x[1], id_pos, 1u);
    tc_mma(d_im, w[5], x[0], id_pos, 1u);
  }
}

template <int BN>
__global__ void __launch_bounds__(RT_THREADS, 1)
k_radial_tc(const __grid_constant__ CUtensorMap tmW, const __grid_constant__ CUtensorMap tmX, int n_r, int n_cols,
            int n_k_blocks, int stages, float2* __restrict__ Y, unsigned* status) {
  using T = RadialTile<BN>;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ uint64_t full_bar[8], empty_bar[8], acc_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  // aligned by an offset from the __shared__ array itself, so that the compiler keeps the shared
  // address space (shared loads and stores, not generic ones) for every access through it
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * RT_BM;
  const int c0 = blockIdx.y * BN;
  const int l = blockIdx.z;

  if (threadIdx.x == 0) {
    for (int s = 0; s < stages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&acc_bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(T::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  volatile int* abort_p = &abort_flag;

  if (warp == 0) {
    if (lane == 0) {
      // producer: 4 W planes (128 x 32) and 4 x planes (BN x 32) per stage
      int issued = 0;
      for (int kb = 0; kb < n_k_blocks; ++kb) {
        const int s = kb % stages;
        if (kb >= stages && !mbar_wait(&empty_bar[s], ((kb / stages) & 1) ^ 1, abort_p)) break;
        uint8_t* st = smem + (size_t)s * T::STAGE;
        mbar_expect_tx(&full_bar[s], T::STAGE);
        tma_load_4d(st, &tmW, kb * RT_BK, m0, 0, l, &full_bar[s]);
        tma_load_4d(st + T::A_STAGE, &tmX, kb * RT_BK, c0, 0, l, &full_bar[s]);
        issued = kb + 1;
      }
      // never leave copies in flight: on abort, wait (bounded) for every issued stage to land
      if (*abort_p) {
        for (int kb = (issued > stages ? issued - stages : 0); kb < issued; ++kb) {
          const uint64_t t0 = gtimer();
          while (!mbar_try(&full_bar[kb % stages], (kb / stages) & 1) && gtimer() - t0 < WAIT_LIMIT_NS) {
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t d_re = tmem, d_im = tmem + BN;
      int done = 0;
      for (int kb = 0; kb < n_k_blocks; ++kb) {
        const int s = kb % stages;
        if (!mbar_wait(&full_bar[s], (kb / stages) & 1, abort_p)) break;
        tc_fence_after();
        const uint32_t sa = smem_u32(smem + (size_t)s * T::STAGE);
        radial_mma_kblock<BN>(sa, sa + T::A_STAGE, d_re, d_im, kb == 0, T::A_PLANE, T::B_PLANE);
        tc_commit(&empty_bar[s]);   // frees the stage once these MMAs have read it
        done = kb + 1;
      }
      // the accumulator barrier also tracks completion of every MMA issued above
      tc_commit(&acc_bar);
      (void)done;
    }
  } else {
    // epilogue: TMEM -> registers -> Y[l][c][i] (complex64)
    const int q = warp & 3;
    const int i = m0 + 32 * q + lane;
    const bool ok = mbar_wait(&acc_bar, 0, abort_p);
    tc_fence_after();
    if (ok && !*abort_p) {
      const uint32_t lane_base = (uint32_t)(32 * q) << 16;
#pragma unroll 1
      for (int cc = 0; cc < BN; cc += 16) {
        uint32_t re[16], im[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(re[0]), "=r"(re[1]), "=r"(re[2]), "=r"(re[3]), "=r"(re[4]), "=r"(re[5]), "=r"(re[6]), "=r"(re[7]),
              "=r"(re[8]), "=r"(re[9]), "=r"(re[10]), "=r"(re[11]), "=r"(re[12]), "=r"(re[13]), "=r"(re[14]),
              "=r"(re[15])
            : "r"(tmem + lane_base + cc));
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(im[0]), "=r"(im[1]), "=r"(im[2]), "=r"(im[3]), "=r"(im[4]), "=r"(im[5]), "=r"(im[6]), "=r"(im[7]),
              "=r"(im[8]), "=r"(im[9]), "=r"(im[10]), "=r"(im[11]), "=r"(im[12]), "=r"(im[13]), "=r"(im[14]),
              "=r"(im[15])
            : "r"(tmem + lane_base + BN + cc));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (i < n_r) {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int c = c0 + cc + j;
            if (c < n_cols)
              Y[((size_t)l * n_cols + c) * n_r + i] = make_float2(__uint_as_float(re[j]), __uint_as_float(im[j]));
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (abort_flag && threadIdx.x == 0) atomicOr(status, ST_TC_TIMEOUT);
  if (warp == 1) {
    if (abort_flag && lane == 0) {
      // the accumulator barrier is committed after every issued MMA: wait (bounded) before freeing TMEM
      const uint64_t t0 = gtimer();
      while (!mbar_try(&acc_bar, 0) && gtimer() - t0 < WAIT_LIMIT_NS) {
      }
    }
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(T::TMEM_COLS));
  }
}

// Persistent form: one CTA per SM walks the (M tile, N tile, l) tiles with stride gridDim.x.  The
// stage ring (TMA -> MMA) runs across tile boundaries without draining, and the accumulators are
// double-buffered in tensor memory so the epilogue of one tile overlaps the MMAs of the next.
template <int BN>
__global__ void __launch_bounds__(RT_THREADS, 1)
k_radial_tc_persistent(const __grid_constant__ CUtensorMap tmW, const __grid_constant__ CUtensorMap tmX, int n_r,
                       int n_cols, int n_l, int n_k_blocks, int stages, float2* __restrict__ Y, unsigned* status) {
  using T = RadialTile<BN>;
  constexpr int TMEM_COLS = 2 * T::TMEM_COLS;   // two accumulator buffers
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ uint64_t full_bar[8], empty_bar[8], accf_bar[2], acce_bar[2], drain_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  // aligned by an offset from the __shared__ array itself, so that the compiler keeps the shared
  // address space (shared loads and stores, not generic ones) for every access through it
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m_tiles = (n_r + RT_BM - 1) / RT_BM, n_tiles = (n_cols + BN - 1) / BN;
  const int total = m_tiles * n_tiles * n_l;
  if (threadIdx.x == 0) {
    for (int s = 0; s < stages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf_bar[b], 1);
      mbar_init(&acce_bar[b], 4);   // the four epilogue warps release a buffer
    }
    mbar_init(&drain_bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(&tmem_slot, TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  volatile int* abort_p = &abort_flag;

  if (warp == 0) {
    if (lane == 0) {
      int it = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < total && ok; tile += gridDim.x) {
        const int mt = tile % m_tiles, rest = tile / m_tiles, nt = rest % n_tiles, l = rest / n_tiles;
        for (int kb = 0; kb < n_k_blocks; ++kb, ++it) {
          const int s = it % stages;
          if (it >= stages && !mbar_wait(&empty_bar[s], ((it / stages) & 1) ^ 1, abort_p)) {
            ok = false;
            break;
          }
          uint8_t* st = smem + (size_t)s * T::STAGE;
          mbar_expect_tx(&full_bar[s], T::STAGE);
          tma_load_4d(st, &tmW, kb * RT_BK, mt * RT_BM, 0, l, &full_bar[s]);
          tma_load_4d(st + T::A_STAGE, &tmX, kb * RT_BK, nt * BN, 0, l, &full_bar[s]);
        }
      }
      if (!ok)
        for (int q = (it > stages ? it - stages : 0); q < it; ++q) mbar_drain(&full_bar[q % stages], (q / stages) & 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int it = 0, local = 0;
      for (int tile = blockIdx.x; tile < total; tile += gridDim.x, ++local) {
        const int buf = local & 1;
        // the epilogue must have drained this buffer (its use two tiles back)
        if (local >= 2 && !mbar_wait(&acce_bar[buf], ((local >> 1) - 1) & 1, abort_p)) break;
        tc_fence_after();
        const uint32_t d_re = tmem + buf * T::TMEM_COLS, d_im = d_re + BN;
        bool ok = true;
        for (int kb = 0; kb < n_k_blocks; ++kb, ++it) {
          const int s = it % stages;
          if (!mbar_wait(&full_bar[s], (it / stages) & 1, abort_p)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = smem_u32(smem + (size_t)s * T::STAGE);
          radial_mma_kblock<BN>(sa, sa + T::A_STAGE, d_re, d_im, kb == 0, T::A_PLANE, T::B_PLANE);
          tc_commit(&empty_bar[s]);
        }
        tc_commit(&accf_bar[buf]);
        if (!ok) break;
      }
    }
  } else {
    const int q = warp & 3;
    const uint32_t lane_base = (uint32_t)(32 * q) << 16;
    int local = 0;
    for (int tile = blockIdx.x; tile < total; tile += gridDim.x, ++local) {
      const int buf = local & 1;
      const int mt = tile % m_tiles, rest = tile / m_tiles, nt = rest % n_tiles, l = rest / n_tiles;
      const bool ok = mbar_wait(&accf_bar[buf], (local >> 1) & 1, abort_p);
      tc_fence_after();
      if (!ok) break;
      const int i = mt * RT_BM + 32 * q + lane, c0 = nt * BN;
      const uint32_t d_re = tmem + buf * T::TMEM_COLS, d_im = d_re + BN;
#pragma unroll 1
      for (int cc = 0; cc < BN; cc += 16) {
        uint32_t re[16], im[16];
        tmem_ld16(d_re + lane_base + cc, re);
        tmem_ld16(d_im + lane_base + cc, im);
        tmem_ld_wait();
        tmem_regs_ready(re);
        tmem_regs_ready(im);
        if (i < n_r) {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int c = c0 + cc + j;
            if (c < n_cols)
              Y[((size_t)l * n_cols + c) * n_r + i] = make_float2(__uint_as_float(re[j]), __uint_as_float(im[j]));
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acce_bar[buf]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (abort_flag && threadIdx.x == 0) atomicOr(status, ST_TC_TIMEOUT);
  if (warp == 1) {
    if (abort_flag && lane == 0) {
      // the drain barrier completes once every MMA this thread issued is done
      tc_commit(&drain_bar);
      mbar_drain(&drain_bar, 0);
    }
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, TMEM_COLS);
  }
}

template <int BN>
static size_t radial_smem(int stages) {
  return (size_t)stages * RadialTile<BN>::STAGE + 1024;
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------

EncodeTiledFn tensor_map_encoder() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// 4-D BF16 tensor (k, rows, plane, l) with a (32, box_rows, planes, 1) box and 64-byte swizzle.
static bool make_map(CUtensorMap* map, void* base, int k_pad, int rows, int planes, int n_l, int box_rows) {
  EncodeTiledFn enc = tensor_map_encoder();
  if (!enc) return false;
  cuuint64_t dims[4] = {(cuuint64_t)k_pad, (cuuint64_t)rows, (cuuint64_t)planes, (cuuint64_t)n_l};
  cuuint64_t strides[3] = {(cuuint64_t)k_pad * 2, (cuuint64_t)rows * k_pad * 2,
                           (cuuint64_t)planes * rows * k_pad * 2};
  cuuint32_t box[4] = {RT_BK, (cuuint32_t)box_rows, (cuuint32_t)planes, 1};
  cuuint32_t es[4] = {1, 1, 1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

#define MX_CK(call)                                                       \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) {                                              \
      err = std::string(#call) + ": " + cudaGetErrorString(e_);           \
      return GGB_ERR_CUDA;                                                \
    }                                                                     \
  } while (0)

static int pick_bn(int n_cols) {
  if (n_cols <= 16) return 16;
  if (n_cols <= 32) return 32;
  if (n_cols <= 64) return 64;
  return 128;
}

template <int BN>
static cudaError_t configure_radial(int stages) {
  cudaError_t e = cudaFuncSetAttribute(k_radial_tc<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)radial_smem<BN>(stages));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_radial_tc_persistent<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)radial_smem<BN>(stages));
}

static int stages_for(int bn) {
  const int stage = W_PLANES * RT_BM * RT_BK * 2 + 4 * bn * RT_BK * 2;
  int s = (200 * 1024) / stage;
  if (s > 8) s = 8;
  if (s < 2) s = 2;
  return s;
}

int mixed_prepare(MixedGroup& m, GroupArgs& a, const double2* W_fp64, double2* x_fp64, double2* y_fp64,
                  int precision, std::string& err) {
  if (precision != GGB_SPLIT_BF16 && precision != GGB_SPLIT_INT8) {
    err = "split_tf32 is not available in this build; use split_int8 or split_bf16";
    return GGB_ERR_ARG;
  }
  m.precision = precision;
  const int n_r = a.n_r, n_l = a.n_l, nc = a.n_cols;
  m.k_pad = ((n_r + RT_BK - 1) / RT_BK) * RT_BK;
  m.rows_pad = ((n_r + RT_BM - 1) / RT_BM) * RT_BM;
  m.bn = pick_bn(nc);
  m.cols_pad = ((nc + m.bn - 1) / m.bn) * m.bn;
  m.stages = stages_for(m.bn);
  int n_mats = 0;
  for (int h = 0; h < 2; ++h)
    for (int o = 0; o < a.chain[h].n_ops; ++o) n_mats = std::max(n_mats, a.chain[h].ops[o].mat + 1);
  if (precision == GGB_SPLIT_INT8) {
    // the orbitals stay in the context's FP64 buffers; the observables pass is the FP64 one
    m.Xd = x_fp64;
    m.Yd = y_fp64;
    const int rc = int8_prepare(m, a, W_fp64, n_mats, err);
    if (rc) return rc;
    m.ready = true;
    return GGB_OK;
  }
  const size_t nx = (size_t)n_l * nc * n_r;
  MX_CK(cudaMalloc(&m.X, nx * sizeof(float2)));
  MX_CK(cudaMalloc(&m.Y, nx * sizeof(float2)));
  MX_CK(cudaMemset(m.Y, 0, nx * sizeof(float2)));
  int dev = 0, optin = 0;
  MX_CK(cudaGetDevice(&dev));
  MX_CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (angular_smem_f32(n_l) > (size_t)optin) {
    err = "N_l too large for the FP32 angular kernel";
    return GGB_ERR_ARG;
  }
  MX_CK(set_max_dynamic_smem((const void*)k_angular_f32<true>, optin));
  MX_CK(set_max_dynamic_smem((const void*)k_angular_f32<false>, optin));
  const size_t nxs = (size_t)n_l * 4 * m.cols_pad * m.k_pad;
  MX_CK(cudaMalloc(&m.Xsp, nxs * sizeof(__nv_bfloat16)));
  MX_CK(cudaMemset(m.Xsp, 0, nxs * sizeof(__nv_bfloat16)));
  const size_t nws = (size_t)n_l * W_PLANES * m.rows_pad * m.k_pad;
  MX_CK(cudaMalloc(&m.Wsp, nws * sizeof(__nv_bfloat16)));
  const dim3 tb(32, 8), tg((m.rows_pad + 31) / 32, (m.k_pad + 31) / 32, n_l);
  k_split_w<<<tg, tb>>>(W_fp64, m.Wsp, n_r, m.rows_pad, m.k_pad);
  MX_CK(cudaGetLastError());
  const size_t n_mat_el = (size_t)n_mats * a.n_m * n_l * a.ldS;
  MX_CK(cudaMalloc(&m.mats_f, n_mat_el * sizeof(float)));
  k_d2f_real<<<256, 256>>>(a.mats, m.mats_f, n_mat_el);
  MX_CK(cudaGetLastError());
  if (!make_map(&m.tmW, m.Wsp, m.k_pad, m.rows_pad, W_PLANES, n_l, RT_BM) ||
      !make_map(&m.tmX, m.Xsp, m.k_pad, m.cols_pad, 4, n_l, m.bn)) {
    err = "cuTensorMapEncodeTiled failed";
    return GGB_ERR_CUDA;
  }
  // tensor-core angular chain (falls back to the FP32 chain when N_l does not fit its tiles)
  if (angular_tc_config(n_l, m.at_k_atoms, m.at_m_tiles, m.at_stages, m.at_smem) == 0) {
    const int rows = 128 * m.at_m_tiles, lk = 64 * m.at_k_atoms;
    const size_t nst = (size_t)n_mats * a.n_m * S_PLANES * rows * lk;
    MX_CK(cudaMalloc(&m.St, nst * sizeof(__nv_bfloat16)));
    k_build_st<<<512, 256>>>(a.mats, m.St, n_mats, a.n_m, n_l, a.ldS, rows, lk);
    MX_CK(cudaGetLastError());
    EncodeTiledFn enc = tensor_map_encoder();
    cuuint64_t dims[5] = {(cuuint64_t)lk, (cuuint64_t)rows, S_PLANES, (cuuint64_t)a.n_m, (cuuint64_t)n_mats};
    cuuint64_t strides[4] = {(cuuint64_t)lk * 2, (cuuint64_t)rows * lk * 2, (cuuint64_t)S_PLANES * rows * lk * 2,
                             (cuuint64_t)a.n_m * S_PLANES * rows * lk * 2};
    cuuint32_t box[5] = {64, 128, 1, 1, 1};
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    if (!enc || enc(&m.tmS, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, m.St, dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
      err = "cuTensorMapEncodeTiled (angular S^T) failed";
      return GGB_ERR_CUDA;
    }
    MX_CK(angular_tc_configure());
    m.angular_tc = true;
  }
  switch (m.bn) {
    case 16: MX_CK(configure_radial<16>(m.stages)); m.smem = radial_smem<16>(m.stages); break;
    case 32: MX_CK(configure_radial<32>(m.stages)); m.smem = radial_smem<32>(m.stages); break;
    case 64: MX_CK(configure_radial<64>(m.stages)); m.smem = radial_smem<64>(m.stages); break;
    default: MX_CK(configure_radial<128>(m.stages)); m.smem = radial_smem<128>(m.stages); break;
  }
  MX_CK(cudaDeviceGetAttribute(&m.persistent_ctas, cudaDevAttrMultiProcessorCount, dev));
  MX_CK(cudaDeviceSynchronize());
  m.ready = true;
  return GGB_OK;
}

int mixed_load_orbitals(MixedGroup& m, const GroupArgs& a, const double2* x_fp64) {
  if (!m.ready) return GGB_ERR_STATE;
  if (m.precision == GGB_SPLIT_INT8) {
    // the state is the FP64 buffer itself; node-basis vectors kept for basis reuse no longer match it
    if (!m.i8.yth_step) return GGB_OK;
    if (cudaMemset(m.i8.yth_step, 0xFF, sizeof(int)) != cudaSuccess) return GGB_ERR_CUDA;
    return cudaDeviceSynchronize() == cudaSuccess ? GGB_OK : GGB_ERR_CUDA;
  }
  const size_t n = (size_t)a.n_l * a.n_cols * a.n_r;
  k_d2f<<<512, 256>>>(x_fp64, m.X, n);
  return cudaDeviceSynchronize() == cudaSuccess ? GGB_OK : GGB_ERR_CUDA;
}

int mixed_store_orbitals(MixedGroup& m, const GroupArgs& a, double2* x_fp64) {
  if (!m.ready) return GGB_ERR_STATE;
  if (m.precision == GGB_SPLIT_INT8) return GGB_OK;
  const size_t n = (size_t)a.n_l * a.n_cols * a.n_r;
  k_f2d<<<512, 256>>>(m.X, x_fp64, n);
  return cudaDeviceSynchronize() == cudaSuccess ? GGB_OK : GGB_ERR_CUDA;
}

static void launch_radial_tc(MixedGroup& m, const GroupArgs& a, cudaStream_t s) {
  const int nkb = m.k_pad / RT_BK;
  if (m.persistent_ctas > 0) {
    const int tiles = ((a.n_r + RT_BM - 1) / RT_BM) * ((a.n_cols + m.bn - 1) / m.bn) * a.n_l;
    const dim3 g(tiles < m.persistent_ctas ? tiles : m.persistent_ctas);
    switch (m.bn) {
      case 16: k_radial_tc_persistent<16><<<g, RT_THREADS, m.smem, s>>>(m.tmW, m.tmX, a.n_r, a.n_cols, a.n_l, nkb, m.stages, m.Y, a.status); break;
      case 32: k_radial_tc_persistent<32><<<g, RT_THREADS, m.smem, s>>>(m.tmW, m.tmX, a.n_r, a.n_cols, a.n_l, nkb, m.stages, m.Y, a.status); break;
      case 64: k_radial_tc_persistent<64><<<g, RT_THREADS, m.smem, s>>>(m.tmW, m.tmX, a.n_r, a.n_cols, a.n_l, nkb, m.stages, m.Y, a.status); break;
      default: k_radial_tc_persistent<128><<<g, RT_THREADS, m.smem, s>>>(m.tmW, m.tmX, a.n_r, a.n_cols, a.n_l, nkb, m.stages, m.Y, a.status); break;
    }
    return;
  }
  const dim3 grid((a.n_r + RT_BM - 1) / RT_BM, (a.n_cols + m.bn - 1) / m.bn, a.n_l);
  switch (m.bn) {
    case 16: k_radial_tc<16><<<grid, RT_THREADS, m.smem, s>>>(m.tmW, m.tmX, a.n_r, a.n_cols, nkb, m.stages, m.Y, a.status); break;
    case 32: k_radial_tc<32><<<grid, RT_THREADS, m.smem, s>>>(m.tmW, m.tmX, a.n_r, a.n_cols, nkb, m.stages, m.Y, a.status); break;
    case 64: k_radial_tc<64><<<grid, RT_THREADS, m.smem, s>>>(m.tmW, m.tmX, a.n_r, a.n_cols, nkb, m.stages, m.Y, a.status); break;
    default: k_radial_tc<128><<<grid, RT_THREADS, m.smem, s>>>(m.tmW, m.tmX, a.n_r, a.n_cols, nkb, m.stages, m.Y, a.status); break;
  }
}

static void launch_angular_mixed(MixedGroup& m, const GroupArgs& a, int half, const float2* xin, float2* xout,
                                 bool split_out, int do_obs, cudaStream_t s) {
  MixArgs mx{m.mats_f, m.k_pad, m.cols_pad, m.Xsp};
  const dim3 grid(a.n_cols * ((a.n_r + TR - 1) / TR)), block(ANG_WARPS * 32);
  const size_t smem = angular_smem_f32(a.n_l);
  if (split_out) k_angular_f32<true><<<grid, block, smem, s>>>(a, mx, half, xin, xout, do_obs);
  else k_angular_f32<false><<<grid, block, smem, s>>>(a, mx, half, xin, xout, do_obs);
}

void mixed_init(MixedGroup& m, const GroupArgs& a, const double2*, cudaStream_t s) {
  if (m.precision == GGB_SPLIT_INT8) launch_angular_fp64(a, 2, m.Xd, nullptr, 1, s);
  else launch_angular_mixed(m, a, 2, m.X, m.X, false, 1, s);
}

static void angular_half(MixedGroup& m, const GroupArgs& a, int half, cudaStream_t s) {
  if (m.precision == GGB_SPLIT_INT8) {
    if (half == 0) {
      if (m.angular_fp64) launch_angular_fp64(a, 0, m.Xd, m.Xd, 0, s);
      else int8_angular(m, a, 0, m.Xd, m.Xd, s);
      int8_slice_x(m, a, m.Xd, s);
    } else {
      // also the density and dipole partial sums
      if (m.angular_fp64) launch_angular_fp64(a, 1, m.Yd, m.Xd, 1, s);
      else int8_angular(m, a, 1, m.Yd, m.Xd, s);
    }
    return;
  }
  if (m.angular_tc) {
    if (half == 0) {
      launch_angular_tc(m, a, 0, m.X, nullptr, s);
    } else {
      launch_angular_tc(m, a, 1, m.Y, m.X, s);
      // FP64 density and dipole partial sums of the new orbitals (empty chain, no write-back)
      launch_angular_mixed(m, a, 2, m.X, nullptr, false, 1, s);
    }
  } else {
    if (half == 0) launch_angular_mixed(m, a, 0, m.X, nullptr, true, 0, s);
    else launch_angular_mixed(m, a, 1, m.Y, m.X, false, 1, s);
  }
}

static void radial(MixedGroup& m, const GroupArgs& a, cudaStream_t s) {
  if (m.precision == GGB_SPLIT_INT8) int8_radial(m, a, s);
  else launch_radial_tc(m, a, s);
}

void mixed_step(MixedGroup& m, const GroupArgs& a, cudaStream_t s) {
  angular_half(m, a, 0, s);
  radial(m, a, s);
  angular_half(m, a, 1, s);
}

void mixed_phase(MixedGroup& m, const GroupArgs& a, int phase, cudaStream_t s) {
  if (phase == 0) angular_half(m, a, 0, s);
  if (phase == 1) radial(m, a, s);
  if (phase == 2) angular_half(m, a, 1, s);
}

void mixed_release(MixedGroup& m) {
  cudaFree(m.X);
  cudaFree(m.Y);
  cudaFree(m.Xsp);
  cudaFree(m.Wsp);
  cudaFree(m.mats_f);
  cudaFree(m.St);
  int8_release(m.i8);
  m = MixedGroup();
}

}  // namespace ggb
