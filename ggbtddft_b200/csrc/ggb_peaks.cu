// Peak-throughput microbenchmarks of the GPU the library runs on, with kernels of its own: the
// denominators of the roofline fractions of the FP64 form (FP64 FMA on the CUDA cores) and of the
// int8 form (tcgen05.mma kind::i8 with int32 accumulation in tensor memory).
//
//  k_peak_fp64  eight independent FMA chains per thread, every SM filled with 8 x 256 threads:
//               2 flops per DFMA, nothing else issued in the loop.
//  k_peak_dmma  eight independent mma.sync m8n8k4 f64 accumulators per warp, the same grid as
//               k_peak_fp64: 2 * 8 * 8 * 4 flops per MMA.
//  k_peak_i8    one CTA per SM (its shared-memory request leaves no room for a second); one
//               thread issues back-to-back M = 128, N = 256, K = 32 int8 MMAs from two tiles (K-major, 32-byte swizzle, pseudo-random bytes) into
//               one tensor-memory accumulator, then commits once: 2 * 128 * 256 * 32 ops per MMA.
//               The commit wait is bounded (2 s); on a timeout the kernel raises ST_TC_TIMEOUT in
//               its status word, drains (bounded) and still frees its tensor memory.
// No device memory is allocated: status and sink are file-scope __device__ variables.
#include <cuda_runtime.h>

#include "../../include/ggbtddft.h"
#include "ggb_internal.cuh"
#include "ggb_mixed.cuh"
#include "ggb_tc_common.cuh"

namespace ggb {
namespace {

constexpr int PK_FMA_CHAINS = 8;
constexpr int PK_FMA_THREADS = 256;
constexpr int PK_FMA_BLOCKS_PER_SM = 8;
constexpr int PK_MMA_M = 128, PK_MMA_N = 256, PK_MMA_K = 32;

__device__ unsigned g_peak_status;
__device__ double g_peak_sink;

__host__ __device__ constexpr uint32_t pk_idesc_i8(int m, int n) {
  // kind::i8: signed A and B (bits 7, 10), int32 D (bits 4-5 = 2), N >> 3 at bit 17, M >> 4 at bit 24
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__global__ void __launch_bounds__(PK_FMA_THREADS) k_peak_fp64(int iters, double seed) {
  double a[PK_FMA_CHAINS];
#pragma unroll
  for (int k = 0; k < PK_FMA_CHAINS; ++k) a[k] = seed + 1e-9 * (threadIdx.x + blockIdx.x) + k;
  const double b = 1.0 - 1e-13, c = 1e-14;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < PK_FMA_CHAINS; ++k) a[k] = fma(a[k], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < PK_FMA_CHAINS; ++k) s += a[k];
  if (s == -1.0) g_peak_sink = s;   // never true; keeps the chains live
}

__global__ void __launch_bounds__(PK_FMA_THREADS) k_peak_dmma(int iters, double seed) {
  double c[PK_FMA_CHAINS][2];
#pragma unroll
  for (int k = 0; k < PK_FMA_CHAINS; ++k) {
    c[k][0] = seed + k;
    c[k][1] = seed - k;
  }
  const double a = 1.0 - 1e-13 * (threadIdx.x & 7), b = 1e-3;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < PK_FMA_CHAINS; ++k)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                   : "+d"(c[k][0]), "+d"(c[k][1])
                   : "d"(a), "d"(b));
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < PK_FMA_CHAINS; ++k) s += c[k][0] + c[k][1];
  if (s == -1.0) g_peak_sink = s;   // never true; keeps the chains live
}

__global__ void __launch_bounds__(128, 1) k_peak_i8(int n_mma) {
  extern __shared__ __align__(1024) uint8_t raw[];
  __shared__ uint64_t done_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  uint8_t* sm = raw + ((1024u - (smem_u32(raw) & 1023u)) & 1023u);
  uint32_t* w = reinterpret_cast<uint32_t*>(sm);
  for (int i = threadIdx.x; i < (PK_MMA_M + PK_MMA_N) * PK_MMA_K / 4; i += blockDim.x) {
    uint32_t h = (uint32_t)i * 2654435761u + blockIdx.x * 40503u;
    h ^= h >> 15;
    w[i] = h * 2246822519u;
  }
  fence_async_smem();
  if (threadIdx.x == 0) {
    mbar_init(&done_bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x < 32) tmem_alloc(&tmem_slot, PK_MMA_N);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  if (threadIdx.x == 0) {
    const uint64_t adesc = sdesc_kmajor(smem_u32(sm), PK_MMA_K, 6);
    const uint64_t bdesc = sdesc_kmajor(smem_u32(sm + PK_MMA_M * PK_MMA_K), PK_MMA_K, 6);
    const uint32_t idesc = pk_idesc_i8(PK_MMA_M, PK_MMA_N);
    for (int i = 0; i < n_mma; ++i)
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "setp.ne.b32 p, %4, 0;\n\t"
          "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
          "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)(i > 0)));
    tc_commit(&done_bar);
  }
  __syncwarp();
  volatile int* abort_p = &abort_flag;
  if (!mbar_wait(&done_bar, 0, abort_p)) {
    if (threadIdx.x == 0) atomicOr(&g_peak_status, ST_TC_TIMEOUT);
    mbar_drain(&done_bar, 0);
  }
  tc_fence_after();
  if (threadIdx.x < 32) {
    uint32_t v[4];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
                 : "r"(tmem));
    tmem_ld_wait();
    tmem_regs_ready(v);
    if ((int)(v[0] ^ v[1] ^ v[2] ^ v[3]) == 0x7f3a5c11) g_peak_sink = 1.0;   // keeps the products live
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) tmem_dealloc(tmem, PK_MMA_N);
}

}  // namespace
}  // namespace ggb

using namespace ggb;

extern "C" int ggb_measure_peaks(double* fp64_tflops, double* int8_tops, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return GGB_ERR_CUDA;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return GGB_ERR_CUDA;
  // the tiles take 12 KB; asking for 120 KB keeps one CTA per SM, so that every SM issues MMAs
  const size_t smem = 120 * 1024;
  if (cudaFuncSetAttribute((const void*)k_peak_i8, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return GGB_ERR_CUDA;
  const unsigned zero = 0;
  if (cudaMemcpyToSymbol(g_peak_status, &zero, sizeof zero) != cudaSuccess) return GGB_ERR_CUDA;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return GGB_ERR_CUDA;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return GGB_ERR_CUDA;
  }
  const int fma_iters = 1 << 16, n_mma = 1 << 16, reps = 3;
  float best_f = 1e30f, best_i = 1e30f, ms = 0.0f;
  for (int r = 0; r < reps + 1; ++r) {   // the first launch of each is a warm-up
    cudaEventRecord(e0, s);
    k_peak_fp64<<<sms * PK_FMA_BLOCKS_PER_SM, PK_FMA_THREADS, 0, s>>>(fma_iters, 1.0);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && ms < best_f) best_f = ms;
    cudaEventRecord(e0, s);
    k_peak_i8<<<sms, 128, smem, s>>>(n_mma);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && ms < best_i) best_i = ms;
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) return GGB_ERR_CUDA;
  unsigned st = 0;
  if (cudaMemcpyFromSymbol(&st, g_peak_status, sizeof st) != cudaSuccess) return GGB_ERR_CUDA;
  if (st) return GGB_ERR_DEVICE;
  const double fma_flops = 2.0 * PK_FMA_CHAINS * (double)fma_iters * PK_FMA_THREADS * PK_FMA_BLOCKS_PER_SM * sms;
  const double mma_ops = 2.0 * PK_MMA_M * PK_MMA_N * PK_MMA_K * (double)n_mma * sms;
  if (fp64_tflops) *fp64_tflops = fma_flops / (best_f * 1e-3) / 1e12;
  if (int8_tops) *int8_tops = mma_ops / (best_i * 1e-3) / 1e12;
  return GGB_OK;
}

extern "C" int ggb_measure_peak_fp64_mma(double* tflops, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return GGB_ERR_CUDA;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return GGB_ERR_CUDA;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return GGB_ERR_CUDA;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return GGB_ERR_CUDA;
  }
  const int iters = 1 << 13, reps = 3;
  float best = 1e30f, ms = 0.0f;
  for (int r = 0; r < reps + 1; ++r) {   // the first launch is a warm-up
    cudaEventRecord(e0, s);
    k_peak_dmma<<<sms * PK_FMA_BLOCKS_PER_SM, PK_FMA_THREADS, 0, s>>>(iters, 1.0);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && ms < best) best = ms;
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) return GGB_ERR_CUDA;
  const double warps = (double)sms * PK_FMA_BLOCKS_PER_SM * (PK_FMA_THREADS / 32);
  const double flops = 2.0 * 8 * 8 * 4 * PK_FMA_CHAINS * (double)iters * warps;
  if (tflops) *tflops = flops / (best * 1e-3) / 1e12;
  return GGB_OK;
}
