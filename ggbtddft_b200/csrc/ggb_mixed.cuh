// Split-precision forms of the step.  split_bf16: complex64 orbitals, radial propagator and angular
// chain on tcgen05 tensor cores with 3xBF16 split products and FP32 accumulation in tensor memory.
// split_int8: complex128 orbitals, radial propagator and angular chain as int8 slice products with
// exact int32 accumulation (ggb_int8.cu).  Observables and potentials in FP64 in both.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <stdint.h>

#include <string>

#include "ggb_internal.cuh"

namespace ggb {

constexpr unsigned ST_TC_TIMEOUT = 8u;   // a bounded wait in a tensor-core kernel gave up

// Integer-split form (ggb_int8.cu): int8 slice planes of W, of the chain matrices and of the radial
// B operand, with per-row power-of-two exponents of the constant operators.
struct I8Group {
  int8_t* W = nullptr;       // [variant][N_l][8][rows_pad][k_pad]: Wr slices 1-4, Wi slices 1-4; A(i,k) = W[l][k][i] 2^e(l,i)
  int* wexp = nullptr;       // [N_l][rows_pad]
  int8_t* X = nullptr;       // [N_l][12][cols_pad][k_pad]: Xr, Xi, -Xi slices 1-4 of x 2^xexp(l, col)
  int* xexp = nullptr;       // [N_l][cols_pad]
  int8_t* St = nullptr;      // [variant][mat][m][4][rows][lk]: S^T slices, rows scaled by 2^sexp
  int n_mats = 0;            // chain matrices per variant
  int* sexp = nullptr;       // [mat][m][rows]
  CUtensorMap tmW, tmX, tmS;
  int bn = 16, cols_pad = 0, stages = 2, ctas = 0;
  int tune_bn = 0, tune_stages = 0;   // ggb_set_tuning (0: built-in choice)
  size_t smem = 0;
  int np = 32, a_k_atoms = 0, a_m_tiles = 0, a_stages = 0, a_rows = 0, a_ld = 0;
  size_t a_smem = 0;
  // theta form, basis reuse (ggb_set_theta_reuse, on by default): the second half's node-basis
  // vectors after its phase [N_l][n_cols][N_r] and the step whose first half starts from them
  bool theta_reuse = true;
  double2* yth = nullptr;
  int* yth_step = nullptr;
};

struct MixedGroup {
  int precision = 0;
  bool ready = false;
  int k_pad = 0;        // N_r rounded up to the radial K block (32)
  int rows_pad = 0;     // N_r rounded up to the radial M tile (128)
  int bn = 16;          // radial N tile (orbital columns per CTA)
  int cols_pad = 0;     // n_cols rounded up to the N tile (zero columns keep every TMA box in bounds)
  int stages = 4;
  size_t smem = 0;
  int persistent_ctas = 0;  // > 0: persistent radial launch with this many CTAs (one per SM)
  float2* X = nullptr;              // state [N_l][n_cols][N_r] (BF16 form)
  double2* Xd = nullptr;            // state and radial output of the int8 form: the context's FP64
  double2* Yd = nullptr;            //   orbital buffers (not owned)
  float2* Y = nullptr;              // radial output [N_l][n_cols][N_r]
  __nv_bfloat16* Xsp = nullptr;     // radial B operand [N_l][4][cols_pad][k_pad]  (re hi, re lo, im hi, im lo)
  __nv_bfloat16* Wsp = nullptr;     // radial A operand [N_l][4][rows_pad][k_pad] (Wr hi, Wr lo, Wi hi, Wi lo), A(i,k) = W[l][k][i]
  float* mats_f = nullptr;          // chain matrices in FP32
  CUtensorMap tmW;
  CUtensorMap tmX;
  // int8 form: the angular products on the FP64 tensor cores (the FP64 form's kernel, mma.sync f64)
  // instead of int8 slices on tcgen05; the radial product stays int8
  bool angular_fp64 = false;
  // tensor-core angular chain
  bool angular_tc = false;
  __nv_bfloat16* St = nullptr;      // S^T planes [mat][m][hi,lo][m_tiles*128 (j)][k_atoms*64 (l)]
  CUtensorMap tmS;
  int at_k_atoms = 0, at_m_tiles = 0, at_stages = 0;
  size_t at_smem = 0;
  I8Group i8;
};

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn tensor_map_encoder();

int int8_prepare(MixedGroup& mg, GroupArgs& a, const double2* W_fp64, int n_mats, std::string& err);
void int8_radial(MixedGroup& mg, const GroupArgs& a, cudaStream_t s);
void int8_angular(MixedGroup& mg, const GroupArgs& a, int half, const double2* xin, double2* xout, cudaStream_t s);
void int8_slice_x(MixedGroup& mg, const GroupArgs& a, const double2* x, cudaStream_t s);
void int8_release(I8Group& q);

int angular_tc_config(int n_l, int& k_atoms, int& m_tiles, int& stages, size_t& smem);
cudaError_t angular_tc_configure();
void launch_angular_tc(const MixedGroup& mg, const GroupArgs& a, int half, const float2* xin, float2* xout,
                       cudaStream_t s);

int mixed_prepare(MixedGroup& m, GroupArgs& a, const double2* W_fp64, double2* x_fp64, double2* y_fp64,
                  int precision, std::string& err);
int mixed_load_orbitals(MixedGroup& m, const GroupArgs& a, const double2* x_fp64);
int mixed_store_orbitals(MixedGroup& m, const GroupArgs& a, double2* x_fp64);
void mixed_init(MixedGroup& m, const GroupArgs& a, const double2* x_fp64, cudaStream_t s);
void mixed_step(MixedGroup& m, const GroupArgs& a, cudaStream_t s);
void mixed_phase(MixedGroup& m, const GroupArgs& a, int phase, cudaStream_t s);
void mixed_release(MixedGroup& m);

}  // namespace ggb
