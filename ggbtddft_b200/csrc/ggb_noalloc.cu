// ggb_observables_noalloc: dipole, acceleration and norm of a set of orbitals without any device
// allocation.
//
// Some callers cannot call cudaMalloc: code that runs inside another framework's memory pool or
// allocator (which must own every device allocation), code on a path that is being captured into a
// CUDA graph after its set-up, or a process that has reserved all device memory up front.  This
// entry point computes the same per-(l, orbital) dipole and acceleration sums and per-orbital norm
// that the time step records (dipoleMoment.cuh / dipoleAcceleration.cuh plus the norm), from
// caller-provided device-accessible buffers only.  The partial sums over radius tiles, which the
// context keeps in buffers it allocates, live here in a file-scope __device__ array of fixed size.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/ggbtddft.h"
#include "ggb_angular.cuh"

namespace ggb {

// Capacity of the shared scratch: n_orb * N_l * ceil(N_r / 32) partial sums (each two double4,
// 64 bytes: 4 MiB in all) and n_orb * ceil(N_r / 32) norm partials (dd, 16 bytes: 256 KiB).
constexpr int NA_MAX_PARTIALS = 65536;
constexpr int NA_MAX_NORM = 16384;
constexpr int NA_MAX_NL = 256;

static __device__ __align__(256) double4 g_obs_scratch[2 * NA_MAX_PARTIALS];
static __device__ __align__(256) double2 g_norm_scratch[NA_MAX_NORM];

constexpr int NA_WARPS = 8;

// One CTA per (orbital, 32-radius tile): the tile of every l in shared memory, then the same
// per-l dipole/acceleration partials as the time step (observables_tile) and a compensated norm
// partial.
__global__ void __launch_bounds__(NA_WARPS * 32)
k_obs_partials(const double2* __restrict__ x, const double* __restrict__ r, const double* __restrict__ coef,
               const int* __restrict__ m_of, int n_l, int n_orb, int n_r, int n_tiles, double4* __restrict__ obs,
               double2* __restrict__ norm_part) {
  extern __shared__ double2 xs[];  // [N_l][32]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int k = blockIdx.x / n_tiles, tile = blockIdx.x - k * n_tiles;
  const int rr_i = tile * TR + lane;
  const bool rv = rr_i < n_r;
  for (int l = warp; l < n_l; l += NA_WARPS)
    xs[l * TR + lane] = rv ? x[((size_t)l * n_orb + k) * n_r + rr_i] : make_double2(0.0, 0.0);
  __syncthreads();
  GroupArgs g{};
  g.n_l = n_l;
  g.n_m = NA_MAX_NL;      // the coefficient rows are laid out for m = 0 .. NA_MAX_NL-1
  g.n_tiles = n_tiles;
  g.obs_seg = TR;
  g.coef = coef;
  g.obs = obs;
  int m = m_of[k];
  if (m < 0 || m > n_l) m = n_l;   // an invalid m contributes nothing (no l satisfies l >= m)
  const double rr = rv ? r[rr_i] : 1.0;
  const double fr2 = rv ? pow(rr, -2.0) : 0.0;
  // the coefficient rows of this m, NA_MAX_NL long whatever the call's N_l
  const int mr = m < NA_MAX_NL ? m : NA_MAX_NL - 1;
  const double* cu_row = coef + ((size_t)CF_CU * NA_MAX_NL + mr) * NA_MAX_NL;
  const double* cd_row = coef + ((size_t)CF_CD * NA_MAX_NL + mr) * NA_MAX_NL;
  observables_tile(g, xs, k, m, tile * TR, lane, warp, NA_WARPS, rr, fr2, TR, cu_row, cd_row);
  if (warp == 0) {
    dd s{0.0, 0.0};
    for (int l = m; l < n_l; ++l) {
      const double2 v = xs[l * TR + lane];
      s = dd_add(s, dd{v.x * v.x + v.y * v.y, 0.0});
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s = dd_add(s, dd{__shfl_xor_sync(0xffffffffu, s.hi, o),
                                                       __shfl_xor_sync(0xffffffffu, s.lo, o)});
    if (lane == 0) norm_part[(size_t)k * n_tiles + tile] = make_double2(s.hi, s.lo);
  }
}

// One thread per (l, orbital) sums the tiles; one thread per orbital sums the norm partials.
__global__ void k_obs_reduce(const double4* __restrict__ obs, const double2* __restrict__ norm_part, int n_l,
                             int n_orb, int n_tiles, double2* __restrict__ dip, double2* __restrict__ acc,
                             double* __restrict__ norm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_l * n_orb) {
    const int l = i / n_orb, k = i - l * n_orb;
    const double4* p = obs + 2 * (((size_t)k * n_l + l) * n_tiles);
    dd sx{0.0, 0.0}, sy{0.0, 0.0}, sz{0.0, 0.0}, sw{0.0, 0.0};
    for (int t = 0; t < n_tiles; ++t) {
      const double4 h = p[2 * t], lo = p[2 * t + 1];
      sx = dd_add(sx, dd{h.x, lo.x}); sy = dd_add(sy, dd{h.y, lo.y});
      sz = dd_add(sz, dd{h.z, lo.z}); sw = dd_add(sw, dd{h.w, lo.w});
    }
    dip[(size_t)l * n_orb + k] = make_double2(sx.hi + sx.lo, sy.hi + sy.lo);
    acc[(size_t)l * n_orb + k] = make_double2(sz.hi + sz.lo, sw.hi + sw.lo);
  }
  if (i < n_orb) {
    dd s{0.0, 0.0};
    for (int t = 0; t < n_tiles; ++t) {
      const double2 v = norm_part[(size_t)i * n_tiles + t];
      s = dd_add(s, dd{v.x, v.y});
    }
    norm[i] = s.hi + s.lo;
  }
}

// Angular coefficient rows c_u, c_d (l, m < NA_MAX_NL) of the observables, [coef][m][l] with rows
// NA_MAX_NL long (independent of a call's N_l, so filled once per device): the same closed forms
// as the context's tables (angularCoefficients.cuh:57-111).
static __device__ __align__(256) double g_coef[2 * NA_MAX_NL * NA_MAX_NL];

__global__ void k_fill_coef(double* coef) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NA_MAX_NL * NA_MAX_NL) return;
  const int n_l = NA_MAX_NL;
  const int m = i / n_l, l = i - m * n_l;
  const double dl = l, dm = m;
  const double cu = (l >= m) ? sqrt((pow(dl + 1.0, 2.0) - pow(dm, 2.0)) / ((2.0 * dl + 1.0) * (2.0 * dl + 3.0))) : 0.0;
  const double cd = (l >= 1 && l - 1 >= m) ? sqrt((pow(dl, 2.0) - pow(dm, 2.0)) / ((2.0 * dl + 1.0) * (2.0 * dl - 1.0)))
                                           : 0.0;
  coef[((size_t)CF_CU * NA_MAX_NL + m) * n_l + l] = cu;
  coef[((size_t)CF_CD * NA_MAX_NL + m) * n_l + l] = cd;
}

// Per-device addresses of the file-scope arrays, resolved on a device's first call.
struct NoallocDevice {
  bool ready = false;
  double4* obs = nullptr;
  double2* norm = nullptr;
  double* coef = nullptr;
};
static NoallocDevice g_dev[64];
static std::mutex g_setup_mutex;

// Resolves the arrays' device addresses with `dev` current and fills the coefficient table, once
// per device (synchronously); serialised across host threads.
static int noalloc_setup(int dev) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  NoallocDevice& d = g_dev[dev];
  if (d.ready) return GGB_OK;
  if (cudaGetSymbolAddress((void**)&d.obs, g_obs_scratch) != cudaSuccess) return GGB_ERR_CUDA;
  if (cudaGetSymbolAddress((void**)&d.norm, g_norm_scratch) != cudaSuccess) return GGB_ERR_CUDA;
  if (cudaGetSymbolAddress((void**)&d.coef, g_coef) != cudaSuccess) return GGB_ERR_CUDA;
  if (cudaFuncSetAttribute(k_obs_partials, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           NA_MAX_NL * TR * (int)sizeof(double2)) != cudaSuccess)
    return GGB_ERR_CUDA;
  k_fill_coef<<<(NA_MAX_NL * NA_MAX_NL + 255) / 256, 256>>>(d.coef);
  if (cudaStreamSynchronize(0) != cudaSuccess) return GGB_ERR_CUDA;
  d.ready = true;
  return GGB_OK;
}

}  // namespace ggb

extern "C" int ggb_observables_noalloc(const double* x, const double* r, const int* m, int n_l, int n_orb, int n_r,
                                       double* dip, double* acc, double* norm, void* stream) {
  using namespace ggb;
  if (!x || !r || !m || !dip || !acc || !norm) return GGB_ERR_ARG;
  if (n_l < 2 || n_l > NA_MAX_NL || n_orb < 1 || n_r < 1) return GGB_ERR_ARG;
  const int n_tiles = (n_r + TR - 1) / TR;
  if ((long long)n_orb * n_l * n_tiles > NA_MAX_PARTIALS || (long long)n_orb * n_tiles > NA_MAX_NORM)
    return GGB_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return GGB_ERR_CUDA;
  const int rc = noalloc_setup(dev);
  if (rc) return rc;
  const NoallocDevice& d = g_dev[dev];
  cudaStream_t s = (cudaStream_t)stream;
  k_obs_partials<<<n_orb * n_tiles, NA_WARPS * 32, (size_t)n_l * TR * sizeof(double2), s>>>(
      reinterpret_cast<const double2*>(x), r, d.coef, m, n_l, n_orb, n_r, n_tiles, d.obs, d.norm);
  const int nt = n_l * n_orb > n_orb ? n_l * n_orb : n_orb;
  k_obs_reduce<<<(nt + 127) / 128, 128, 0, s>>>(d.obs, d.norm, n_l, n_orb, n_tiles, reinterpret_cast<double2*>(dip),
                                                 reinterpret_cast<double2*>(acc), norm);
  return cudaGetLastError() == cudaSuccess ? GGB_OK : GGB_ERR_CUDA;
}
