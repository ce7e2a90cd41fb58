// Integer-split form of the step (GGB_SPLIT_INT8): exact accumulation on tcgen05.
//
// Why: the tensor cores' FP32 accumulators do not round to nearest.  Every accumulator update
// shrinks |acc| by a fraction of an ulp, always in the same direction, and a time step makes a few
// hundred updates per orbital value: the norm then decays geometrically (measured: ~1.4e-8 per
// update, 2.4 % over the 8,826 steps of the hydrogen pulse).  Integer products accumulate exactly.
//
// Representation (Ozaki-style split, base 256):
//   every operand row (a row of W_l, of a chain matrix S^T, of orbital values) is scaled by a power
//   of two 2^e that puts its largest |value| in [63, 126), rounded once to an integer T ~ v 2^e 2^24
//   (to nearest for orbital values; dithered for the constant operators, below)
//   (|T| < 2^31) and cut into its four balanced base-256 digits, the bytes of T + 0x80808080 each
//   less 128 (an int8 in [-128, 127]):
//       v 2^e = a1 + a2 2^-8 + a3 2^-16 + a4 2^-24 (+ at most 2^-25)
//   A row is resolved to ~2^-31 of its own maximum.  The constant operators (W_l, the chain
//   matrices) are applied every step, so a fixed rounding error of theirs compounds linearly over
//   the pulse (measured: W rounded to nearest alone moves the helium harmonics by 6e-4).  They are
//   therefore held as several dithered variants, rounded with offsets that cycle through
//   (j + 1/2) / n_var, and the step counter picks variant (step mod n_var): over n_var steps the
//   variants average to the exact operator to within 2^-24 / (2 n_var) of the row scale, and what
//   is left of the rounding is a zero-mean oscillation.  The orbital values are rounded to nearest
//   afresh at every product, which is already zero-mean.
//   product: the ten slice pairs (j, m) with j + m <= 3 (0-based; the rest weigh < 2^-32 of the
//   row maxima and are zero-mean), accumulated exactly in int32 tensor memory, one accumulator per
//   weight 2^-8(j+m); the epilogue combines the four accumulators exactly (int64 shifts), undoes the
//   two row scales exactly and rounds once to FP64.  The orbitals stay complex128 between products.
//   int32 range: |a b| <= 2^14, at most 8 products per k and accumulator, K <= 8192: <= 2^30.
//
//  k_slice_w_i8      W[l][k][i] -> A(i,k) planes [variant][l][8][rows][k] (Wr a1..a4, Wi a1..a4) + exponents
//  k_build_st_i8     chain matrices -> S^T planes [variant n_mats + mat][m][4][rows][lk] + exponents
//  k_slice_x         orbitals (complex128) -> radial B operand planes (Xr, Xi, -Xi) + exponents
//  k_radial_i8       persistent radial product, kind::i8, 32-byte swizzle, 16 MMAs per 32-wide k block
//                    (each covers all x slices m of one W slice j):
//                      Re_s += Wr_j Xr_m + Wi_j (-Xi)_m,  Im_s += Wr_j Xi_m + Wi_j Xr_m   (j + m = s)
//  k_angular_i8      the angular chain with int8 operands, exact accumulation and per-point scales
#include <cuda.h>

#include <algorithm>
#include <cstdio>

#include "../../include/ggbtddft.h"
#include "ggb_angular.cuh"
#include "ggb_mixed.cuh"
#include "ggb_tc_common.cuh"

namespace ggb {

constexpr int I8_SLICES = 4;

// ---------------------------------------------------------------------------------------------
// slicing
// ---------------------------------------------------------------------------------------------


// exponent e with max 2^e in [63, 126) (0 for an all-zero row): with max = f 2^E, f in [0.5, 1),
// f 2^7 lies in [64, 126) unless f >= 126 / 128, and then f 2^6 lies in [63, 64).  Below 126 the
// top slice never exceeds 126 (see slice_int).  Clamped to e <= 1000 (rows below 1e-290 are
// resolved less finely; 2^e stays a normal double).
__device__ __forceinline__ int row_exponent(double mx) {
  if (!(mx > 0.0) || !(mx < 1e300)) return 0;
  int ex;
  const double f = frexp(mx, &ex);
  return min(1000, 7 - ex - (f >= 126.0 / 128.0 ? 1 : 0));
}

// The four balanced base-256 digits of T = rint(t3), t3 = t 2^24 with |t| < 126 (|T| < 2^31): the
// bytes of (T + 0x80808080) xor 0x80808080, each an int8 in [-128, 127], T = sum_k a_k 2^(8(3-k)).
__device__ __forceinline__ uint32_t slice_word(double t3) {
  return ((uint32_t)__double2int_rn(t3) + 0x80808080u) ^ 0x80808080u;
}
// the four slices of t3 stored one byte at dst + k * PLANE, most significant first
template <uint32_t PLANE>
__device__ __forceinline__ void store_slices(uint8_t* dst, double t3) {
  const uint32_t v = slice_word(t3);
  dst[0] = (uint8_t)(v >> 24);
  dst[PLANE] = (uint8_t)(v >> 16);
  dst[2 * PLANE] = (uint8_t)(v >> 8);
  dst[3 * PLANE] = (uint8_t)v;
}
// Dithered variants of the constant operators: variant v of element (a, b, c) rounds t 2^24 down
// after adding ((v + h(a, b, c)) mod n_var + 1/2) / n_var.  Over the n_var variants the offsets
// take every value once, so their mean is t 2^24 to within 1 / (2 n_var); the hash h staggers the
// cycle from element to element, so that one step's errors are as uncorrelated as rounding to
// nearest.  n_var is a power of two.
constexpr int I8_W_VARIANTS = 8;
constexpr int I8_S_VARIANTS = 16;

__device__ __forceinline__ uint32_t dither_hash(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t h = a * 0x9E3779B1u ^ b * 0x85EBCA77u ^ c * 0xC2B2AE3Du;
  h ^= h >> 15;
  h *= 0x2C1B3C6Du;
  h ^= h >> 13;
  return h;
}
__device__ __forceinline__ double dither_offset(int v, int n_var, uint32_t h) {
  return ((double)((v + (int)(h >> 8)) & (n_var - 1)) + 0.5) / (double)n_var;
}
// the four slices of floor(t 2^24 + d) (|t| < 126, 0 < d < 1) as int8 values, most significant first
__device__ __forceinline__ void slice4_dithered(double t, double d, int8_t* s) {
  const uint32_t v = ((uint32_t)__double2int_rd(fma(t, 16777216.0, d)) + 0x80808080u) ^ 0x80808080u;
#pragma unroll
  for (int q = 0; q < I8_SLICES; ++q) s[q] = (int8_t)(uint8_t)(v >> (24 - 8 * q));
}

// row maxima of A(i,k) = W[l][k][i] over k (re and im)
__global__ void k_w_rowmax(const double2* __restrict__ W, int* __restrict__ wexp, int n_r, int rows_pad) {
  const int l = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows_pad) return;
  double mx = 0.0;
  if (i < n_r)
    for (int k = 0; k < n_r; ++k) {
      const double2 w = W[((size_t)l * n_r + k) * n_r + i];
      mx = fmax(mx, fmax(fabs(w.x), fabs(w.y)));
    }
  wexp[(size_t)l * rows_pad + i] = row_exponent(mx);
}

// A(i,k) planes, transposed through shared memory (read along i, write along k)
__global__ void k_slice_w_i8(const double2* __restrict__ W, const int* __restrict__ wexp, int8_t* __restrict__ Wi8,
                             int n_r, int rows_pad, int k_pad, int variant, int n_var) {
  __shared__ double2 t[32][33];
  const int l = blockIdx.z;
  const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int q = ty; q < 32; q += 8) {
    const int k = k0 + q, i = i0 + tx;
    t[q][tx] = (k < n_r && i < n_r) ? W[((size_t)l * n_r + k) * n_r + i] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  const size_t plane = (size_t)rows_pad * k_pad;
  int8_t* base = Wi8 + (size_t)l * 8 * plane;
  for (int q = ty; q < 32; q += 8) {
    const int i = i0 + q, k = k0 + tx;
    if (i < rows_pad && k < k_pad) {
      const double sc = ldexp(1.0, wexp[(size_t)l * rows_pad + i]);
      const double2 w = t[tx][q];
      const uint32_t h = dither_hash((uint32_t)l, (uint32_t)i, (uint32_t)k);
      int8_t sr[I8_SLICES], si[I8_SLICES];
      slice4_dithered(w.x * sc, dither_offset(variant, n_var, h), sr);
      slice4_dithered(w.y * sc, dither_offset(variant, n_var, h * 0x165667B1u), si);
      const size_t o = (size_t)i * k_pad + k;
#pragma unroll
      for (int p = 0; p < I8_SLICES; ++p) {
        base[p * plane + o] = sr[p];
        base[(I8_SLICES + p) * plane + o] = si[p];
      }
    }
  }
}

// S^T planes of the chain matrices: St[mat][m][slice][j][l] with the row (j) exponents
__global__ void k_build_st_i8(const double* __restrict__ mats, int8_t* __restrict__ St, int* __restrict__ sexp,
                              int n_mm, int n_m, int n_l, int ldS, int rows, int lk, int variant, int n_var) {
  const int row = blockIdx.x;                 // (mat * n_m + m) * rows + j
  const int mm = row / rows, j = row - mm * rows;
  if (mm >= n_mm) return;
  __shared__ double red[256];
  double mx = 0.0;
  for (int l = threadIdx.x; l < n_l; l += blockDim.x)
    if (j < n_l) mx = fmax(mx, fabs(mats[((size_t)mm * n_l + l) * ldS + j]));
  red[threadIdx.x] = mx;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  const int e = row_exponent(red[0]);
  if (threadIdx.x == 0 && variant == 0) sexp[row] = e;
  const double sc = ldexp(1.0, e);
  const size_t plane = (size_t)rows * lk;
  for (int l = threadIdx.x; l < lk; l += blockDim.x) {
    const double v = (j < n_l && l < n_l) ? mats[((size_t)mm * n_l + l) * ldS + j] * sc : 0.0;
    int8_t s[I8_SLICES];
    // the hash leaves out m, so that a matrix gets the same variants in any group of runs
    slice4_dithered(v, dither_offset(variant, n_var, dither_hash((uint32_t)(mm / n_m), (uint32_t)j, (uint32_t)l)), s);
#pragma unroll
    for (int p = 0; p < I8_SLICES; ++p) St[(size_t)mm * I8_SLICES * plane + p * plane + (size_t)j * lk + l] = s[p];
  }
}

// ---------------------------------------------------------------------------------------------
// radial product, kind::i8
// ---------------------------------------------------------------------------------------------

constexpr int R8_BM = 128, R8_BK = 32, R8_THREADS = 192;
constexpr int R8_W_PLANES = 8;      // Wr a1..a4, Wi a1..a4
constexpr int R8_X_PLANES = 12;     // Xr b1..b4, Xi b1..b4, -Xi b1..b4

__host__ __device__ constexpr uint32_t idesc_i8(int m, int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
__device__ __forceinline__ void tc_mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&v)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr));
}

// 2^k as a double (0 below the normal range)
__device__ __forceinline__ double pow2i(int k) {
  return k < -1022 ? 0.0 : __longlong_as_double((long long)(k + 1023) << 52);
}
// sum_s D_s 2^(8(3-s)) of the four int32 accumulators of column u, exactly (|D_s| <= 2^30: < 2^55)
template <int W>
__device__ __forceinline__ long long combine_int(const uint32_t (&d)[4][W], int u) {
  return (long long)(int)d[0][u] * 16777216LL + (long long)(int)d[1][u] * 65536LL + (long long)(int)d[2][u] * 256LL +
         (long long)(int)d[3][u];
}
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&v)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
               : "r"(taddr));
}

template <int BN>
struct R8Tile {
  static constexpr int A_PLANE = R8_BM * R8_BK;     // 4 KB
  static constexpr int B_PLANE = BN * R8_BK;
  static constexpr int A_STAGE = R8_W_PLANES * A_PLANE;
  static constexpr int STAGE = A_STAGE + R8_X_PLANES * B_PLANE;
  static constexpr int ACC_COLS = 8 * BN;           // Re s=2..5, Im s=2..5
  static constexpr int NBUF = (2 * ACC_COLS <= 512) ? 2 : 1;
  static constexpr int TMEM_COLS = NBUF * ACC_COLS <= 32 ? 32 : NBUF * ACC_COLS <= 64 ? 64
                                 : NBUF * ACC_COLS <= 128 ? 128 : NBUF * ACC_COLS <= 256 ? 256 : 512;
};

template <int BN>
__global__ void __launch_bounds__(R8_THREADS, 1)
k_radial_i8(const __grid_constant__ CUtensorMap tmW, const __grid_constant__ CUtensorMap tmX,
            const int* __restrict__ wexp, const int* __restrict__ xexp, int n_r, int rows_pad, int n_cols,
            int cols_pad, int n_l, int n_k_blocks, int stages, const int* __restrict__ step, int n_var,
            double2* __restrict__ Y, unsigned* status) {
  using T = R8Tile<BN>;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ uint64_t full_bar[8], empty_bar[8], accf_bar[2], acce_bar[2], drain_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  // aligned by an offset from the __shared__ array itself, so that the compiler keeps the shared
  // address space (shared loads and stores, not generic ones) for every access through it
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m_tiles = (n_r + R8_BM - 1) / R8_BM, n_tiles = (n_cols + BN - 1) / BN;
  const int total = m_tiles * n_tiles * n_l;
  if (threadIdx.x == 0) {
    for (int s = 0; s < stages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf_bar[b], 1);
      mbar_init(&acce_bar[b], 4);
    }
    mbar_init(&drain_bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(&tmem_slot, T::TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  volatile int* abort_p = &abort_flag;
  // tile order: N tile fastest, so CTAs that share a W tile run side by side (one HBM read)
  auto decode = [&](int tile, int& mt, int& nt, int& l) {
    nt = tile % n_tiles;
    const int rest = tile / n_tiles;
    mt = rest % m_tiles;
    l = rest / m_tiles;
  };

  if (warp == 0) {
    if (lane == 0) {
      const int var = *step & (n_var - 1);     // this step's variant of W
      int it = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < total && ok; tile += gridDim.x) {
        int mt, nt, l;
        decode(tile, mt, nt, l);
        for (int kb = 0; kb < n_k_blocks; ++kb, ++it) {
          const int s = it % stages;
          if (it >= stages && !mbar_wait(&empty_bar[s], ((it / stages) & 1) ^ 1, abort_p)) {
            ok = false;
            break;
          }
          uint8_t* st = smem + (size_t)s * T::STAGE;
          mbar_expect_tx(&full_bar[s], T::STAGE);
          tma_load_5d(st, &tmW, kb * R8_BK, mt * R8_BM, 0, l, var, &full_bar[s]);
          tma_load_4d(st + T::A_STAGE, &tmX, kb * R8_BK, nt * BN, 0, l, &full_bar[s]);
        }
      }
      if (!ok)
        for (int q = (it > stages ? it - stages : 0); q < it; ++q) mbar_drain(&full_bar[q % stages], (q / stages) & 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc[I8_SLICES] = {idesc_i8(R8_BM, 4 * BN), idesc_i8(R8_BM, 3 * BN), idesc_i8(R8_BM, 2 * BN),
                                          idesc_i8(R8_BM, BN)};
      // descriptors: those of stage 0 plus the byte offset / 16 in the start-address field (this
      // thread's issue rate paces the products)
      const uint64_t desc0 = sdesc_kmajor(smem_u32(smem), 32, 6);
      int local = 0, s = 0, ph = 0;
      for (int tile = blockIdx.x; tile < total; tile += gridDim.x, ++local) {
        const int buf = (T::NBUF == 2) ? (local & 1) : 0;
        const int use = (T::NBUF == 2) ? (local >> 1) : local;
        if (use >= 1 && !mbar_wait(&acce_bar[buf], (use - 1) & 1, abort_p)) break;
        tc_fence_after();
        const uint32_t d0 = tmem + buf * T::ACC_COLS;
        bool ok = true;
        for (int kb = 0; kb < n_k_blocks; ++kb) {
          if (!mbar_wait(&full_bar[s], ph, abort_p)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t da = desc0 + (uint64_t)(((uint32_t)s * T::STAGE) >> 4);
          // one 32-wide k block: for each W slice j, one MMA per real product covers the x slices
          // m = 0 .. 3 - j at once (the x planes of each kind are contiguous rows), N = (4 - j) BN,
          // written from accumulator group j on, so that column group m lands on weight 2^-8(j+m)
          const uint64_t xr = da + (T::A_STAGE >> 4);
          const uint64_t xi = xr + ((I8_SLICES * T::B_PLANE) >> 4);
          const uint64_t xn = xr + ((2 * I8_SLICES * T::B_PLANE) >> 4);
#pragma unroll
          for (int j = 0; j < I8_SLICES; ++j) {
            const uint64_t wr = da + ((j * T::A_PLANE) >> 4);
            const uint64_t wi = da + (((I8_SLICES + j) * T::A_PLANE) >> 4);
            const uint32_t dre = d0 + j * BN, dim = d0 + (4 + j) * BN;
            const uint32_t first = (kb == 0 && j == 0) ? 0u : 1u;
            tc_mma_i8(dre, wr, xr, idesc[j], first);
            tc_mma_i8(dre, wi, xn, idesc[j], 1u);
            tc_mma_i8(dim, wr, xi, idesc[j], first);
            tc_mma_i8(dim, wi, xr, idesc[j], 1u);
          }
          tc_commit(&empty_bar[s]);
          if (++s == stages) {
            s = 0;
            ph ^= 1;
          }
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
      const int buf = (T::NBUF == 2) ? (local & 1) : 0;
      const int use = (T::NBUF == 2) ? (local >> 1) : local;
      int mt, nt, l;
      decode(tile, mt, nt, l);
      const bool ok = __all_sync(0xffffffffu, mbar_wait(&accf_bar[buf], use & 1, abort_p));
      tc_fence_after();
      if (!ok) break;
      const int i = mt * R8_BM + 32 * q + lane, c0 = nt * BN;
      const int ew = (i < n_r) ? wexp[(size_t)l * rows_pad + i] : 0;
      const uint32_t d0 = tmem + buf * T::ACC_COLS + lane_base;
#pragma unroll 1
      for (int cc = 0; cc < BN; cc += 8) {
        uint32_t re[4][8], im[4][8];
#pragma unroll
        for (int sidx = 0; sidx < 4; ++sidx) {
          tmem_ld8(d0 + sidx * BN + cc, re[sidx]);
          tmem_ld8(d0 + (4 + sidx) * BN + cc, im[sidx]);
        }
        tmem_ld_wait();
#pragma unroll
        for (int sidx = 0; sidx < 4; ++sidx) {
          tmem_regs_ready(re[sidx]);
          tmem_regs_ready(im[sidx]);
        }
        if (i < n_r) {
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int c = c0 + cc + u;
            if (c < n_cols) {
              const double sc = pow2i(-ew - xexp[(size_t)l * cols_pad + c] - 24);
              Y[((size_t)l * n_cols + c) * n_r + i] =
                  make_double2((double)combine_int(re, u) * sc, (double)combine_int(im, u) * sc);
            }
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
      tc_commit(&drain_bar);
      mbar_drain(&drain_bar, 0);
    }
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, T::TMEM_COLS);
  }
}

// ---------------------------------------------------------------------------------------------
// angular chain, kind::i8
// ---------------------------------------------------------------------------------------------

constexpr int A8_THREADS = 320;
constexpr int A8_EPI_WARP0 = 2;
constexpr int A8_KATOM = 128;            // int8 per 128-byte swizzled row
constexpr int A8_A_TILE = 128 * 128;     // one S^T slice plane: 128 rows (j) x 128 k (l), one stage
constexpr int A8_PTS = 16;               // points per epilogue thread and product
constexpr int A8_TMEM_COLS = 256;        // 4 accumulators x 2 NP columns x m_tiles: two CTAs per SM

struct Ang8Args {
  int k_atoms;            // ceil(N_l / 128)
  int m_tiles;            // ceil(N_l / 128)
  int k_steps;            // ceil(N_l / 32): 32-wide K steps that carry data
  int stages;
  const int* sexp;        // S^T row exponents [mat][m][rows]
  int rows;               // m_tiles * 128
  int ld_stage;           // row length of the FP64 staging tiles [NP][ld_stage] (odd when it fits)
  int n_mats;             // chain matrices per variant
  int n_var;              // dithered variants of the chain matrices (a power of two)
  // theta form: the node-basis vectors of the second half after its phase, [N_l][n_cols][N_r]
  // (nullptr: not kept), and the step whose first half may start from them (-1: none)
  double2* yth;
  int* yth_step;
};

// Byte offset of (row n, k) of slice plane 0 in the B operand: per 128-wide k atom, the four slice
// planes of nrows K-major 128-byte-swizzled rows each, one after the other (plane q at + q nrows 128),
// so that for one k atom the planes form one operand of 4 nrows rows.
__device__ __forceinline__ uint32_t a8_off(int nrows, int n, int k) {
  const int chunk = ((k & 127) >> 4) ^ (n & 7);
  return (uint32_t)((k >> 7) * I8_SLICES * nrows * 128 + n * 128 + chunk * 16 + (k & 15));
}

// sin and cos of e in FP64: for |e| <= 1/2 the Maclaurin series through e^11 (sine) and e^12
// (cosine), evaluated by Estrin's scheme (short dependency chains); truncation below 2e-14 at
// |e| = 1/2 and far less for the small angles of most phases.  The length-gauge phase r E dt/2 of a
// step stays below 1/2 for the configurations here (r_max E_0 dt/2 <= 0.4); larger angles take the
// library sincos.
__device__ __forceinline__ void sincos_series(double e, double* s, double* c) {
  if (fabs(e) <= 0.5) {
    const double z = e * e, z2 = z * z, z4 = z2 * z2;
    const double s01 = fma(z, -1.0 / 6, 1.0), s23 = fma(z, -1.0 / 5040, 1.0 / 120);
    const double s45 = fma(z, -1.0 / 39916800, 1.0 / 362880);
    *s = e * fma(z4, s45, fma(z2, s23, s01));
    const double c01 = fma(z, -1.0 / 2, 1.0), c23 = fma(z, -1.0 / 720, 1.0 / 24);
    const double c45 = fma(z, -1.0 / 3628800, 1.0 / 40320);
    *c = fma(z4 * z2, 1.0 / 479001600.0, fma(z4, c45, fma(z2, c23, c01)));
  } else {
    sincos(e, s, c);
  }
}
// x exp(-i e), FP64
__device__ __forceinline__ double2 rotd(double2 x, double e) {
  double s, c;
  sincos_series(e, &s, &c);
  return make_double2(c * x.x + s * x.y, c * x.y - s * x.x);
}

// x_k(p) into the four slice planes: Re in row p, Im in row NP + p (the same swizzle chunk, NP being
// a multiple of 8); sc3 = 2^e(p) 2^24
template <int NP, uint32_t PLANE>
__device__ __forceinline__ void slice_put(uint8_t* xb, int p, int k, double2 v, double sc3) {
  const uint32_t o = a8_off(2 * NP, p, k);
  store_slices<PLANE>(xb + o, v.x * sc3);
  store_slices<PLANE>(xb + o + NP * 128, v.y * sc3);
}

// One CTA per (orbital column, NP radii): NP = 32 for N_l <= 128 (one M tile of 128 channels),
// NP = 16 for N_l <= 256 (two M tiles), so that every CTA holds 256 TMEM columns and two CTAs share
// an SM (one CTA's epilogue overlaps the other's products and loads).
//
// The B operand (the l-vectors of the CTA's points, Re rows then Im rows) stays in shared memory
// as four int8 slice planes.  Every point carries one power-of-two scale for its Re and Im rows,
// chosen from the 2-norm of its l-vector: each product of the chain is an orthogonal matrix and
// each phase unitary, so that norm bounds every entry of every intermediate vector and one
// exponent serves the whole chain.  The chain matrices S^T stream through a TMA pipeline, one
// slice plane per stage.  Orbitals in and out are complex128 (xout may alias xin: each CTA reads
// its whole tile before it writes).
//
// Basis reuse (theta form, t.yth set): a half-step is x <- V diag(phase) V^T x with V orthogonal,
// and nothing acts on the orbitals between the second half of one step and the first half of the
// next (the potentials only change the phase).  So V^T x at the start of the next first half is
// the second half's node-basis vector after its phase, which the second half keeps (t.yth, one
// FP64 copy); the next first half loads it, applies its own phase in the prologue and runs only
// its last product, one product instead of two.  The skipped pair V^T V is the identity up to the
// int8 operands' rounding (~2^-31 of each row), which is then not applied.  t.yth_step names the
// step that may start from the kept vectors; setting orbitals invalidates it.
template <int NP, bool SECOND_HALF, bool THETA>
__global__ void __launch_bounds__(A8_THREADS, 2)
k_angular_i8(const __grid_constant__ CUtensorMap tmS, GroupArgs g, Ang8Args t, const double2* xin, double2* xout) {
  constexpr int NB = 2 * NP;                 // B rows: Re of NP points, then Im
  constexpr int B_TILE = NB * 128;           // one slice plane, one k atom
  constexpr int K_ATOMS = NP == 32 ? 1 : 2;  // = M tiles = ceil(N_l / 128)
  constexpr uint32_t XPLANE = K_ATOMS * B_TILE;  // one slice plane over all k atoms
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ uint64_t full_bar[4], empty_bar[4], acc_bar, xb_bar, drain_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  __shared__ double pbase[5][NP];
  __shared__ double pnorm2[NP];
  __shared__ double pscale3[NP], pinv[NP];    // 2^e(p) 2^24 and 2^-e(p) of each point's B rows
  // aligned by an offset from the __shared__ array itself, so that the compiler keeps the shared
  // address space (shared loads and stores, not generic ones) for every access through it
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint8_t* xb = smem;                                              // 4 planes x k_atoms x B_TILE
  uint8_t* sst = smem + (size_t)I8_SLICES * XPLANE;                 // stages x 16 KB
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_l = g.n_l;
  const int tilesN = (g.n_r + NP - 1) / NP;
  const int col = blockIdx.x / tilesN;
  const int r0 = (blockIdx.x - col * tilesN) * NP;
  const int m = g.col_m[col];
  const RunDev run = g.runs[g.col_run[col]];
  const Chain& ch = g.chain[SECOND_HALF ? 1 : 0];
  const int n_ops = ch.n_ops;
  const int acc_cols = 4 * NB;                // per M tile: weights 2^0 .. 2^-24
  const int step_raw = *g.step;
  const int step = step_raw < run.n_t ? step_raw : run.n_t - 1;
  const double hdt = 0.5 * g.dt;
  const double* pco = g.coef + ((size_t)CF_P * g.n_m + m) * n_l;
  // basis reuse: the second half keeps its node-basis vectors, the first half of the step they
  // were kept for starts from them at its last product (o0 = 1, the theta chain having two)
  const bool keep_theta = THETA && SECOND_HALF && t.yth != nullptr;
  const bool from_theta = THETA && !SECOND_HALF && t.yth != nullptr && *t.yth_step == step_raw;
  const int o0 = from_theta ? 1 : 0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < t.stages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&acc_bar, 1);
    mbar_init(&xb_bar, A8_THREADS / 32 - A8_EPI_WARP0);
    mbar_init(&drain_bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(&tmem_slot, A8_TMEM_COLS);
  if (threadIdx.x < NP) {
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
    pbase[0][p] = rr;
    pbase[1][p] = ((g.p_hartree || g.theta) ? (rr * E + v1) : (rr * E)) * hdt;
    pbase[2][p] = v2 * hdt;
    pbase[3][p] = v3 * hdt;
    pbase[4][p] = sb * hdt;
    pnorm2[p] = 0.0;
  }
  __syncthreads();

  // operand: the x tile (all l, NP points) [second half: l-diagonal S phase], staged in the stage
  // buffers (free until the producer starts) as [NP][ldf], the per-point norms, then the slices
  const int lk = t.k_atoms * A8_KATOM;
  const int ldf = t.ld_stage;
  double2* stg = reinterpret_cast<double2*>(sst);
  {
    constexpr int U = 4;
    double part = 0.0;          // this thread's points are fixed: p = threadIdx.x % NP (A8_THREADS % NP == 0)
    const double2* src = from_theta ? t.yth : xin;
    // the reuse path applies the first product's phase here, as its epilogue would (same angle)
    const double* Dv0 = g.dph + ((size_t)ch.ops[0].coupling * g.n_m + m) * g.ldS;
    for (int base = threadIdx.x; base < n_l * NP; base += U * A8_THREADS) {
      double2 v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int idx = base + u * A8_THREADS;
        const int l = idx / NP, p = idx - l * NP, r = r0 + p;
        v[u] = (idx < n_l * NP && r < g.n_r) ? src[((size_t)l * g.n_cols + col) * g.n_r + r] : make_double2(0.0, 0.0);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int idx = base + u * A8_THREADS;
        if (idx < n_l * NP) {
          const int l = idx / NP, p = idx - l * NP;
          double2 w = v[u];
          if (SECOND_HALF && ch.pre_s) w = rotd(w, pbase[4][p] + pco[l] * pbase[2][p]);
          if (!SECOND_HALF && THETA && from_theta && l >= m) {
            const double dj = Dv0[l], p2j = legendre_p2(dj), p3j = legendre_p3(dj);
            double ang = pbase[1][p] * dj + pbase[2][p] * p2j + pbase[3][p] * p3j + pbase[4][p];
            if (g.theta_tab && r0 + p < g.n_r) ang += run.htab[((size_t)m * n_l + l) * g.n_r + r0 + p] * hdt;
            w = rotd(w, ang);
          }
          stg[p * ldf + l] = w;
          part += w.x * w.x + w.y * w.y;
        }
      }
    }
    atomicAdd(&pnorm2[threadIdx.x % NP], part);
  }
  __syncthreads();
  if (threadIdx.x < NP) {
    // |Re y_j|, |Im y_j| <= |y| = |x| for every vector of the chain; the margin covers the chain's
    // rounding and the non-orthogonality of the sliced matrices (both ~2^-31)
    const int e = row_exponent(sqrt(pnorm2[threadIdx.x]) * (1.0 + 0x1p-20));
    pscale3[threadIdx.x] = pow2i(e + 24);
    pinv[threadIdx.x] = pow2i(-e);
  }
  __syncthreads();
  // lanes along l: each warp writes consecutive bytes of one B row
  for (int idx = threadIdx.x; idx < lk * NP; idx += A8_THREADS) {
    const int p = idx / lk, l = idx - p * lk;
    const double2 w = l < n_l ? stg[p * ldf + l] : make_double2(0.0, 0.0);
    slice_put<NP, B_TILE>(xb, p, l, w, pscale3[p]);
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  volatile int* abort_p = &abort_flag;

  if (warp == 0) {
    if (lane == 0) {
      int it = 0;
      bool ok = true;
      for (int o = o0; o < n_ops && ok; ++o) {
        const int mat = ch.ops[o].mat + (step_raw & (t.n_var - 1)) * t.n_mats;   // this step's variant
        // stage pa takes slice plane pa; the ring turns once per (tile, atom)
        for (int mt = 0; mt < t.m_tiles && ok; ++mt)
          for (int ka = 0; ka < t.k_atoms && ok; ++ka) {
            const int round = it / I8_SLICES;
#pragma unroll
            for (int pa = 0; pa < I8_SLICES; ++pa, ++it) {
              if (round > 0 && !mbar_wait(&empty_bar[pa], (round & 1) ^ 1, abort_p)) {
                ok = false;
                break;
              }
              mbar_expect_tx(&full_bar[pa], A8_A_TILE);
              tma_load_5d(sst + pa * A8_A_TILE, &tmS, ka * A8_KATOM, mt * 128, pa, m, mat, &full_bar[pa]);
            }
          }
      }
      if (!ok)
        for (int q = (it > t.stages ? it - t.stages : 0); q < it; ++q) mbar_drain(&full_bar[q % t.stages], (q / t.stages) & 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // one MMA per (S^T slice pa, 32-wide k step): N = (4 - pa) NB rows of the stacked x slice planes
      // 0 .. 3 - pa, written at TMEM column pa NB, so that its column group pb lands on the
      // accumulator of weight 2^-8(pa + pb)
      const uint32_t idesc[I8_SLICES] = {idesc_i8(128, 4 * NB), idesc_i8(128, 3 * NB), idesc_i8(128, 2 * NB),
                                          idesc_i8(128, NB)};
      // The loads come four per (M tile, k atom), one per slice plane pa, into a ring of four
      // stages, so stage pa always holds plane pa and the ring turns once per (tile, atom).  The
      // descriptors of stage pa and k step kk are those of stage 0 (or of the B operand's atom) plus
      // the byte offset / 16 in the start-address field, which keeps this thread's loop short: it
      // shares its SM sub-partition with busy epilogue warps, and its issue rate paces the products.
      const uint64_t adesc = sdesc_kmajor(smem_u32(sst), 128, 2);
      const uint64_t bdesc = sdesc_kmajor(smem_u32(xb), 128, 2);
      int round = 0;
      for (int o = o0; o < n_ops; ++o) {
        if (o > o0 && !mbar_wait(&xb_bar, (o - o0 - 1) & 1, abort_p)) break;
        tc_fence_after();
        bool ok = true;
        for (int mt = 0; mt < t.m_tiles && ok; ++mt) {
          const uint32_t d0 = tmem + acc_cols * mt;
          for (int ka = 0; ka < t.k_atoms && ok; ++ka, ++round) {
            const uint64_t bk = bdesc + (uint64_t)((ka * I8_SLICES * B_TILE) >> 4);
            const int nk = min(A8_KATOM / 32, t.k_steps - ka * (A8_KATOM / 32));
#pragma unroll
            for (int pa = 0; pa < I8_SLICES; ++pa) {
              if (!mbar_wait(&full_bar[pa], round & 1, abort_p)) {
                ok = false;
                break;
              }
              tc_fence_after();
              const uint64_t ak = adesc + (uint64_t)((pa * A8_A_TILE) >> 4);
#pragma unroll
              for (int kk = 0; kk < A8_KATOM / 32; ++kk)
                if (kk < nk) tc_mma_i8(d0 + pa * NB, ak + 2 * kk, bk + 2 * kk, idesc[pa], (ka | kk | pa) ? 1u : 0u);
              tc_commit(&empty_bar[pa]);
            }
          }
        }
        // one commit for all M tiles: every tile's products read the whole operand, which the
        // epilogue overwrites with the next product's
        tc_commit(&acc_bar);
        if (!ok) break;
      }
    }
  } else {
    const int ew = warp - A8_EPI_WARP0;
    const int q = warp & 3;                     // TMEM lane quarter of this warp
    const int grp = ew >> 2;
    const int mt = (t.m_tiles == 2) ? grp : 0;
    const int j = 128 * mt + 32 * q + lane;     // eigen-channel (M row) of this thread
    const int p_begin = (t.m_tiles == 2) ? 0 : A8_PTS * grp;
    // staging of the last product, [N_l][NP + 1] (the odd row length keeps both this write, lanes
    // along l, and the reads below, lanes along the points, free of bank conflicts)
    double2* stage_out = reinterpret_cast<double2*>(smem);
    const uint32_t d0 = tmem + ((uint32_t)(32 * q) << 16) + acc_cols * mt;
    // a warp whose 32 channels are all padding (j >= N_l) does no work: its rows of the next
    // operand stay as the fill left them (zero), and the next product's S^T columns there are zero
    const bool live = 128 * mt + 32 * q < n_l;
    for (int o = o0; o < n_ops; ++o) {
      const bool ok = __all_sync(0xffffffffu, mbar_wait(&acc_bar, (o - o0) & 1, abort_p));
      tc_fence_after();
      if (!ok) break;
      const ChainOp op = ch.ops[o];
      const bool last = (o == n_ops - 1);
      // basis reuse: the second half keeps the first product's result after its phase (row j of
      // this column, from radius r0)
      double2* const ykeep = (keep_theta && o == 0 && j < n_l) ? t.yth + ((size_t)j * g.n_cols + col) * g.n_r + r0 : nullptr;
      if (!live) {
        if (!last) {
          __syncwarp();
          if (lane == 0) mbar_arrive(&xb_bar);
        }
        continue;
      }
      const double* Dv = g.dph + ((size_t)op.coupling * g.n_m + m) * g.ldS;
      const double dj = (op.phase != PH_NONE && j >= m && j < n_l) ? Dv[j] : 0.0;
      const int pb = op.phase == PH_P ? 1 : op.phase == PH_D ? 2 : 3;
      // the theta form: angle = pbase1 x_j + pbase2 P_2(x_j) + pbase3 P_3(x_j) + pbase4 (all x dt/2)
      const bool th = THETA && op.phase == PH_THETA && j >= m && j < n_l;
      const double p2j = th ? legendre_p2(dj) : 0.0, p3j = th ? legendre_p3(dj) : 0.0;
      const bool post_s = last && !SECOND_HALF && ch.post_s && j < n_l;
      const double pj = post_s ? pco[j] : 0.0;
      const double sj = pow2i(-t.sexp[((size_t)op.mat * g.n_m + m) * t.rows + j]);   // S^T row scale
      // software pipeline over chunks of 4 points: the next chunk's accumulators are requested
      // from tensor memory before this chunk is rotated and sliced
      uint32_t re[4][4], im[4][4];
      auto tload = [&](int p0) {
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          tmem_ld4(d0 + s * NB + p0, re[s]);
          tmem_ld4(d0 + s * NB + NP + p0, im[s]);
        }
      };
      auto tready = [&]() {
        tmem_ld_wait();
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          tmem_regs_ready(re[s]);
          tmem_regs_ready(im[s]);
        }
      };
      tload(p_begin);
      tready();
#pragma unroll 1
      for (int c4 = 0; c4 < A8_PTS / 4; ++c4) {
        const int p0 = p_begin + 4 * c4;
        // the accumulators hold y 2^(e_j + e_p) 2^24; rotations commute with the scale, and the
        // next product's slices want y 2^e_p 2^24: one exact power of two in between
        double2 v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          v[u] = make_double2((double)combine_int(re, u) * sj, (double)combine_int(im, u) * sj);
        if (c4 + 1 < A8_PTS / 4) tload(p0 + 4);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int p = p0 + u;
          if constexpr (THETA) {
            if (th) {
              double ang = pbase[1][p] * dj + pbase[2][p] * p2j + pbase[3][p] * p3j + pbase[4][p];
              // n_har > 4: the multipoles L >= 1 at this node come from the exact-quadrature table
              if (g.theta_tab && r0 + p < g.n_r) ang += run.htab[((size_t)m * n_l + j) * g.n_r + r0 + p] * hdt;
              v[u] = rotd(v[u], ang);
            }
          } else {
            if (dj != 0.0) v[u] = rotd(v[u], pbase[pb][p] * dj);
          }
          if (post_s) v[u] = rotd(v[u], pbase[4][p] + pj * pbase[2][p]);
          if (ykeep && r0 + p < g.n_r) {
            const double sc = pinv[p] * 0x1p-24;
            ykeep[p] = make_double2(v[u].x * sc, v[u].y * sc);
          }
          if (!last) {
            if (j < lk) {
              const uint32_t o = a8_off(2 * NP, p, j);
              store_slices<B_TILE>(xb + o, v[u].x);
              store_slices<B_TILE>(xb + o + NP * 128, v[u].y);
            }
          } else if (j < n_l) {
            const double sc = pinv[p] * 0x1p-24;
            stage_out[j * (NP + 1) + p] = make_double2(v[u].x * sc, v[u].y * sc);
          }
        }
        if (c4 + 1 < A8_PTS / 4) tready();
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
    // the kept vectors serve the first half of the next step (the step counter advances once
    // per step, after this kernel)
    if (keep_theta && blockIdx.x == 0 && threadIdx.x == 0) *t.yth_step = step_raw + 1;
    const double2* xs = reinterpret_cast<const double2*>(smem);
    for (int idx = threadIdx.x; idx < n_l * NP; idx += A8_THREADS) {
      const int l = idx / NP, p = idx - l * NP, r = r0 + p;
      if (r < g.n_r) xout[((size_t)l * g.n_cols + col) * g.n_r + r] = xs[l * (NP + 1) + p];
    }
    if (SECOND_HALF) {
      // FP64 dipole and acceleration partial sums and density multipoles of the new orbitals, from
      // the staged tile, with the coefficient rows of this m staged after it.
      constexpr int NW = A8_THREADS / 32;
      constexpr int LG = 32 / NP;        // lane groups per warp: lane = (point, l-loop group)
      constexpr int NG = NW * LG;        // groups that stride the density's l loops
      double* rows = reinterpret_cast<double*>(smem + (((size_t)n_l * (NP + 1) * 16 + 255) & ~(size_t)255));
      double* red = rows + COEF_N * n_l;                    // [NG][N_DEN][NP]
      double* prr = red + NG * N_DEN * NP;                  // [2][NP]: r and r^-2 of each point (0 past N_r)
      for (int i = threadIdx.x; i < COEF_N * n_l; i += A8_THREADS) {
        const int c = i / n_l, l = i - c * n_l;
        rows[i] = g.coef[((size_t)c * g.n_m + m) * n_l + l];
      }
      if (threadIdx.x < NP) {
        const int r = r0 + threadIdx.x;
        const double rr = r < g.n_r ? g.r[r] : 0.0;
        prr[threadIdx.x] = rr;
        prr[NP + threadIdx.x] = r < g.n_r ? pow(rr, -2.0) : 0.0;
      }
      __syncthreads();
      // dipole and acceleration: one thread per l, summing this CTA's NP radii in order (the same
      // terms as observables_tile; one partial per (l, NP radii))
      for (int l = threadIdx.x; l < n_l; l += A8_THREADS) {
        double sx = 0.0, sy = 0.0, sz = 0.0, sw = 0.0;
        if (l >= m) {
          const double c_u = rows[CF_CU * n_l + l], c_d = rows[CF_CD * n_l + l];
          const bool has_u = l + 1 < n_l, has_d = l >= 1;
          for (int p = 0; p < NP; ++p) {
            const double rr = prr[p], fr2 = prr[NP + p];
            const double2 xl = xs[l * (NP + 1) + p];
            const double2 xu = has_u ? xs[(l + 1) * (NP + 1) + p] : make_double2(0.0, 0.0);
            const double2 xd = has_d ? xs[(l - 1) * (NP + 1) + p] : make_double2(0.0, 0.0);
            double2 z1, z2;
            if (l == m) {
              z1 = make_double2(rr * c_u * xu.x, rr * c_u * xu.y);
              z2 = make_double2(fr2 * c_u * xu.x, fr2 * c_u * xu.y);
            } else if (l == n_l - 1) {
              z1 = make_double2(rr * c_d * xd.x, rr * c_d * xd.y);
              z2 = make_double2(fr2 * c_d * xd.x, fr2 * c_d * xd.y);
            } else {
              z1 = make_double2(rr * c_u * xu.x + rr * c_d * xd.x, rr * c_u * xu.y + rr * c_d * xd.y);
              z2 = make_double2(fr2 * (c_u * xu.x + c_d * xd.x), fr2 * (c_u * xu.y + c_d * xd.y));
            }
            sx += xl.x * z1.x + xl.y * z1.y;
            sy += xl.x * z1.y - xl.y * z1.x;
            sz += xl.x * z2.x + xl.y * z2.y;
            sw += xl.x * z2.y - xl.y * z2.x;
          }
        }
        double4* o = g.obs + 2 * (((size_t)col * n_l + l) * g.n_tiles + r0 / NP);
        o[0] = make_double4(sx, sy, sz, sw);
        o[1] = make_double4(0.0, 0.0, 0.0, 0.0);
      }
      // density multipoles: every lane works (point lane % NP), the literal l loops strided over the
      // NG lane groups, then the groups summed in order
      const int n_den = g.n_den > 0 ? g.n_den : 1;   // L = 0 is always needed for the norm
      const int pt = lane % NP, gi = warp * LG + lane / NP;
      double d[N_DEN] = {0.0, 0.0, 0.0, 0.0};
      density_partials<double2, NP + 1>(n_den, m, n_l, xs, pt, rows, gi, NG, d);
#pragma unroll
      for (int L = 0; L < N_DEN; ++L) red[(gi * N_DEN + L) * NP + pt] = d[L];
      __syncthreads();
      if (threadIdx.x < n_den * NP) {
        const int L = threadIdx.x / NP, pp = threadIdx.x - L * NP, rl = r0 + pp;
        double sum = 0.0;
        for (int w = 0; w < NG; ++w) sum += red[(w * N_DEN + L) * NP + pp];
        if (rl < g.n_r) g.dens[((size_t)col * N_DEN + L) * g.n_r + rl] = sum;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    if (abort_flag && lane == 0) {
      tc_commit(&drain_bar);
      mbar_drain(&drain_bar, 0);
    }
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, A8_TMEM_COLS);
  }
}

// Radial B operand of one (l, orbital column) row: exponent f with max(|Re|, |Im|) 2^f in
// [63.75, 127.5) over the row, then Xr, Xi, -Xi as four slices each ([l][12][cols_pad][k_pad]).
constexpr int SX_THREADS = 128;
__global__ void __launch_bounds__(SX_THREADS)
k_slice_x(const double2* __restrict__ x, int n_r, int n_cols, int cols_pad, int k_pad, int8_t* __restrict__ X,
          int* __restrict__ xexp) {
  const int row = blockIdx.x;                  // l * n_cols + col
  const int l = row / n_cols, col = row - l * n_cols;
  const double2* xr = x + (size_t)row * n_r;
  double mx = 0.0;
  for (int r = threadIdx.x; r < n_r; r += SX_THREADS) {
    const double2 v = xr[r];
    mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  __shared__ double wm[SX_THREADS / 32];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = mx;
  __syncthreads();
  mx = wm[0];
#pragma unroll
  for (int w = 1; w < SX_THREADS / 32; ++w) mx = fmax(mx, wm[w]);
  const int f = row_exponent(mx);
  if (threadIdx.x == 0) xexp[(size_t)l * cols_pad + col] = f;
  const double sc = pow2i(f);
  const size_t plane = (size_t)cols_pad * k_pad;
  int8_t* b = X + (size_t)l * 12 * plane + (size_t)col * k_pad;
  // four radii per thread and plane: one 32-bit store each
  for (int r4 = 4 * threadIdx.x; r4 < n_r; r4 += 4 * SX_THREADS) {
    uint32_t pr[I8_SLICES] = {0, 0, 0, 0}, pi[I8_SLICES] = {0, 0, 0, 0}, pn[I8_SLICES] = {0, 0, 0, 0};
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int r = r4 + u;
      const double2 v = r < n_r ? xr[r] : make_double2(0.0, 0.0);
      // -Xi is sliced from -x itself: negating a digit -128 would not fit an int8
      const uint32_t wr = slice_word(v.x * sc * 16777216.0), wi = slice_word(v.y * sc * 16777216.0),
                     wn = slice_word(-v.y * sc * 16777216.0);
#pragma unroll
      for (int qq = 0; qq < I8_SLICES; ++qq) {
        pr[qq] |= ((wr >> (24 - 8 * qq)) & 0xffu) << (8 * u);
        pi[qq] |= ((wi >> (24 - 8 * qq)) & 0xffu) << (8 * u);
        pn[qq] |= ((wn >> (24 - 8 * qq)) & 0xffu) << (8 * u);
      }
    }
#pragma unroll
    for (int qq = 0; qq < I8_SLICES; ++qq) {
      reinterpret_cast<uint32_t*>(b + qq * plane + r4)[0] = pr[qq];
      reinterpret_cast<uint32_t*>(b + (I8_SLICES + qq) * plane + r4)[0] = pi[qq];
      reinterpret_cast<uint32_t*>(b + (2 * I8_SLICES + qq) * plane + r4)[0] = pn[qq];
    }
  }
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------

template <int BN>
static size_t r8_smem(int stages) { return (size_t)stages * R8Tile<BN>::STAGE + 1024; }

static int r8_bn(int n_cols) { return n_cols <= 16 ? 16 : n_cols <= 32 ? 32 : 64; }

static int r8_stages(int bn) {
  const int stage = R8_W_PLANES * R8_BM * R8_BK + R8_X_PLANES * bn * R8_BK;
  int s = (200 * 1024) / stage;
  return s > 8 ? 8 : (s < 2 ? 2 : s);
}

template <int NP>
static size_t a8_smem(int k_atoms, int stages) {
  return (size_t)I8_SLICES * k_atoms * (2 * NP * 128) + (size_t)stages * A8_A_TILE + 1024;
}

#define I8_CK(call)                                                      \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) {                                             \
      err = std::string(#call) + ": " + cudaGetErrorString(e_);          \
      return GGB_ERR_CUDA;                                               \
    }                                                                    \
  } while (0)

int int8_prepare(MixedGroup& mg, GroupArgs& a, const double2* W_fp64, int n_mats, std::string& err) {
  const int n_r = a.n_r, n_l = a.n_l;
  I8Group& q = mg.i8;
  q.bn = q.tune_bn > 0 ? q.tune_bn : r8_bn(a.n_cols);
  q.cols_pad = ((a.n_cols + q.bn - 1) / q.bn) * q.bn;
  q.stages = r8_stages(q.bn);
  if (q.tune_stages > 0) q.stages = std::min(q.tune_stages, q.stages);
  // W planes and row exponents
  const size_t nw = (size_t)n_l * R8_W_PLANES * mg.rows_pad * mg.k_pad;    // one variant
  I8_CK(cudaMalloc(&q.W, nw * I8_W_VARIANTS));
  I8_CK(cudaMalloc(&q.wexp, (size_t)n_l * mg.rows_pad * sizeof(int)));
  k_w_rowmax<<<dim3((mg.rows_pad + 127) / 128, n_l), 128>>>(W_fp64, q.wexp, n_r, mg.rows_pad);
  const dim3 tb(32, 8), tg((mg.rows_pad + 31) / 32, (mg.k_pad + 31) / 32, n_l);
  for (int v = 0; v < I8_W_VARIANTS; ++v)
    k_slice_w_i8<<<tg, tb>>>(W_fp64, q.wexp, q.W + nw * v, n_r, mg.rows_pad, mg.k_pad, v, I8_W_VARIANTS);
  I8_CK(cudaGetLastError());
  // radial B operand planes
  const size_t nx = (size_t)n_l * R8_X_PLANES * q.cols_pad * mg.k_pad;
  I8_CK(cudaMalloc(&q.X, nx));
  I8_CK(cudaMemset(q.X, 0, nx));
  I8_CK(cudaMalloc(&q.xexp, (size_t)n_l * q.cols_pad * sizeof(int)));
  I8_CK(cudaMemset(q.xexp, 0, (size_t)n_l * q.cols_pad * sizeof(int)));
  EncodeTiledFn enc = tensor_map_encoder();
  if (!enc) {
    err = "cuTensorMapEncodeTiled unavailable";
    return GGB_ERR_CUDA;
  }
  {
    cuuint64_t dims[5] = {(cuuint64_t)mg.k_pad, (cuuint64_t)mg.rows_pad, R8_W_PLANES, (cuuint64_t)n_l,
                          (cuuint64_t)I8_W_VARIANTS};
    cuuint64_t strides[4] = {(cuuint64_t)mg.k_pad, (cuuint64_t)mg.rows_pad * mg.k_pad,
                             (cuuint64_t)R8_W_PLANES * mg.rows_pad * mg.k_pad, (cuuint64_t)nw};
    cuuint32_t box[5] = {R8_BK, R8_BM, R8_W_PLANES, 1, 1};
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    if (enc(&q.tmW, CU_TENSOR_MAP_DATA_TYPE_UINT8, 5, q.W, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
        CUDA_SUCCESS) {
      err = "tensor map (int8 W) failed";
      return GGB_ERR_CUDA;
    }
  }
  {
    cuuint64_t dims[4] = {(cuuint64_t)mg.k_pad, (cuuint64_t)q.cols_pad, R8_X_PLANES, (cuuint64_t)n_l};
    cuuint64_t strides[3] = {(cuuint64_t)mg.k_pad, (cuuint64_t)q.cols_pad * mg.k_pad,
                             (cuuint64_t)R8_X_PLANES * q.cols_pad * mg.k_pad};
    cuuint32_t box[4] = {R8_BK, (cuuint32_t)q.bn, R8_X_PLANES, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    if (enc(&q.tmX, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, q.X, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
        CUDA_SUCCESS) {
      err = "tensor map (int8 x) failed";
      return GGB_ERR_CUDA;
    }
  }
  // angular chain: S^T slices
  q.a_m_tiles = (n_l + 127) / 128;
  q.a_k_atoms = (n_l + A8_KATOM - 1) / A8_KATOM;
  if (q.a_m_tiles > 2) {
    err = "N_l > 256 is not supported by the int8 angular chain";
    return GGB_ERR_ARG;
  }
  // two CTAs per SM: 256 TMEM columns each (NP points x {Re, Im} x 4 accumulators x M tiles) and
  // at most ~110 KB of shared memory each
  q.np = q.a_m_tiles == 1 ? 32 : 16;     // the kernel takes k_atoms = m_tiles = (NP == 32 ? 1 : 2)
  q.a_stages = I8_SLICES;   // the MMA issue loop relies on stage = slice plane
  q.a_smem = q.np == 32 ? a8_smem<32>(q.a_k_atoms, q.a_stages) : a8_smem<16>(q.a_k_atoms, q.a_stages);
  // FP64 staging: the input tile [NP][ld] in the stage buffers (an odd ld when it fits), the last
  // product [N_l][NP + 1] over the operand planes and stage buffers
  q.a_ld = ((size_t)q.np * (n_l | 1) * 16 <= (size_t)q.a_stages * A8_A_TILE) ? (n_l | 1) : n_l;
  // the second half's tail: output tile, coefficient rows and the multipoles' warp partials
  const size_t tail = (((size_t)n_l * (q.np + 1) * 16 + 255) & ~(size_t)255) + (size_t)COEF_N * n_l * 8 +
                      (size_t)(A8_THREADS / 32) * N_DEN * 32 * 8 + 2 * (size_t)q.np * 8;
  if ((size_t)q.np * q.a_ld * 16 > (size_t)q.a_stages * A8_A_TILE || tail > q.a_smem - 1024 ||
      q.a_smem > 110 * 1024) {
    err = "int8 angular chain: shared memory";
    return GGB_ERR_ARG;
  }
  if (a.obs_seg != q.np) {
    // the second half writes one observables partial per CTA, so the group's partials are NP radii
    err = "int8 angular chain: observables partials do not match its tile";
    return GGB_ERR_STATE;
  }
  const int rows = 128 * q.a_m_tiles, lk = A8_KATOM * q.a_k_atoms;
  q.a_rows = rows;
  const int n_mm = n_mats * a.n_m;
  const size_t nst = (size_t)n_mm * I8_SLICES * rows * lk;    // one variant
  q.n_mats = n_mats;
  I8_CK(cudaMalloc(&q.St, nst * I8_S_VARIANTS));
  I8_CK(cudaMalloc(&q.sexp, (size_t)n_mm * rows * sizeof(int)));
  for (int v = 0; v < I8_S_VARIANTS; ++v)
    k_build_st_i8<<<n_mm * rows, 256>>>(a.mats, q.St + nst * v, q.sexp, n_mm, a.n_m, n_l, a.ldS, rows, lk, v,
                                        I8_S_VARIANTS);
  I8_CK(cudaGetLastError());
  // basis reuse of the theta form (one phase op and one closing product per half); the angular
  // products on the FP64 kernel keep the full chain
  if (q.theta_reuse && a.theta && !mg.angular_fp64 && a.chain[0].n_ops == 2 && a.chain[1].n_ops == 2) {
    I8_CK(cudaMalloc(&q.yth, (size_t)n_l * a.n_cols * n_r * sizeof(double2)));
    I8_CK(cudaMalloc(&q.yth_step, sizeof(int)));
    I8_CK(cudaMemset(q.yth_step, 0xFF, sizeof(int)));   // -1: nothing kept yet
  }
  {
    // the variants follow one another along the matrix index: matrix mat of variant v is mat + v n_mats
    cuuint64_t dims[5] = {(cuuint64_t)lk, (cuuint64_t)rows, I8_SLICES, (cuuint64_t)a.n_m,
                          (cuuint64_t)n_mats * I8_S_VARIANTS};
    cuuint64_t strides[4] = {(cuuint64_t)lk, (cuuint64_t)rows * lk, (cuuint64_t)I8_SLICES * rows * lk,
                             (cuuint64_t)a.n_m * I8_SLICES * rows * lk};
    cuuint32_t box[5] = {A8_KATOM, 128, 1, 1, 1};
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    if (enc(&q.tmS, CU_TENSOR_MAP_DATA_TYPE_UINT8, 5, q.St, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
        CUDA_SUCCESS) {
      err = "tensor map (int8 S^T) failed";
      return GGB_ERR_CUDA;
    }
  }
  int dev = 0, optin = 0, sms = 0;
  I8_CK(cudaGetDevice(&dev));
  I8_CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  I8_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  q.ctas = sms;
  switch (q.bn) {
    case 16: I8_CK(set_max_dynamic_smem((const void*)k_radial_i8<16>, optin)); q.smem = r8_smem<16>(q.stages); break;
    case 32: I8_CK(set_max_dynamic_smem((const void*)k_radial_i8<32>, optin)); q.smem = r8_smem<32>(q.stages); break;
    default: I8_CK(set_max_dynamic_smem((const void*)k_radial_i8<64>, optin)); q.smem = r8_smem<64>(q.stages); break;
  }
  I8_CK(set_max_dynamic_smem((const void*)k_angular_i8<32, false, false>, optin));
  I8_CK(set_max_dynamic_smem((const void*)k_angular_i8<32, true, false>, optin));
  I8_CK(set_max_dynamic_smem((const void*)k_angular_i8<16, false, false>, optin));
  I8_CK(set_max_dynamic_smem((const void*)k_angular_i8<16, true, false>, optin));
  I8_CK(set_max_dynamic_smem((const void*)k_angular_i8<32, false, true>, optin));
  I8_CK(set_max_dynamic_smem((const void*)k_angular_i8<32, true, true>, optin));
  I8_CK(set_max_dynamic_smem((const void*)k_angular_i8<16, false, true>, optin));
  I8_CK(set_max_dynamic_smem((const void*)k_angular_i8<16, true, true>, optin));
  I8_CK(cudaDeviceSynchronize());
  return GGB_OK;
}

void int8_radial(MixedGroup& mg, const GroupArgs& a, cudaStream_t s) {
  const I8Group& q = mg.i8;
  const int tiles = ((a.n_r + R8_BM - 1) / R8_BM) * ((a.n_cols + q.bn - 1) / q.bn) * a.n_l;
  const dim3 g(tiles < q.ctas ? tiles : q.ctas);
  const int nkb = mg.k_pad / R8_BK;
  switch (q.bn) {
    case 16: k_radial_i8<16><<<g, R8_THREADS, q.smem, s>>>(q.tmW, q.tmX, q.wexp, q.xexp, a.n_r, mg.rows_pad, a.n_cols, q.cols_pad, a.n_l, nkb, q.stages, a.step, I8_W_VARIANTS, mg.Yd, a.status); break;
    case 32: k_radial_i8<32><<<g, R8_THREADS, q.smem, s>>>(q.tmW, q.tmX, q.wexp, q.xexp, a.n_r, mg.rows_pad, a.n_cols, q.cols_pad, a.n_l, nkb, q.stages, a.step, I8_W_VARIANTS, mg.Yd, a.status); break;
    default: k_radial_i8<64><<<g, R8_THREADS, q.smem, s>>>(q.tmW, q.tmX, q.wexp, q.xexp, a.n_r, mg.rows_pad, a.n_cols, q.cols_pad, a.n_l, nkb, q.stages, a.step, I8_W_VARIANTS, mg.Yd, a.status); break;
  }
}

void int8_angular(MixedGroup& mg, const GroupArgs& a, int half, const double2* xin, double2* xout, cudaStream_t s) {
  const I8Group& q = mg.i8;
  Ang8Args t;
  t.k_atoms = q.a_k_atoms;
  t.m_tiles = q.a_m_tiles;
  t.k_steps = (a.n_l + 31) / 32;
  t.stages = q.a_stages;
  t.sexp = q.sexp;
  t.rows = q.a_rows;
  t.ld_stage = q.a_ld;
  t.n_mats = q.n_mats;
  t.n_var = I8_S_VARIANTS;
  t.yth = q.yth;
  t.yth_step = q.yth_step;
  const dim3 grid(a.n_cols * ((a.n_r + q.np - 1) / q.np));
#define GGB_A8(NP, SH, TH) k_angular_i8<NP, SH, TH><<<grid, A8_THREADS, q.a_smem, s>>>(q.tmS, a, t, xin, xout)
  if (q.np == 32) {
    if (half == 0) { if (a.theta) GGB_A8(32, false, true); else GGB_A8(32, false, false); }
    else { if (a.theta) GGB_A8(32, true, true); else GGB_A8(32, true, false); }
  } else {
    if (half == 0) { if (a.theta) GGB_A8(16, false, true); else GGB_A8(16, false, false); }
    else { if (a.theta) GGB_A8(16, true, true); else GGB_A8(16, true, false); }
  }
#undef GGB_A8
}

void int8_slice_x(MixedGroup& mg, const GroupArgs& a, const double2* x, cudaStream_t s) {
  const I8Group& q = mg.i8;
  k_slice_x<<<a.n_l * a.n_cols, SX_THREADS, 0, s>>>(x, a.n_r, a.n_cols, q.cols_pad, mg.k_pad, q.X, q.xexp);
}

void int8_release(I8Group& q) {
  cudaFree(q.W);
  cudaFree(q.wexp);
  cudaFree(q.X);
  cudaFree(q.xexp);
  cudaFree(q.St);
  cudaFree(q.sexp);
  cudaFree(q.yth);
  cudaFree(q.yth_step);
  q = I8Group();
}

}  // namespace ggb
