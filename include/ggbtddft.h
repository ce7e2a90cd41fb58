/*
 * ggbtddft.h -- C ABI of the B200 split-operator time step (libggbtddft.so).
 *
 * Drop-in replacement for the time loop of ggbTDDFT's main.cu: the work of
 *   h_timePropagation(ksoSetTD, hartree, propagators, mesh, observables, temp, handles, scandx)
 *   (src/subFunctions/timePropagation/h_timePropagation.cuh:32-114)
 * together with the loaders it depends on (src/main.cu:442-481).  The reference has no plugin or
 * FFI interface: its seam is that function plus its workingData files, configured by compile-time
 * macros (src/params.cuh).  Here every size is a run-time value, several independent runs
 * ("scans", src/main.cu:460) advance together, and every call returns a status code instead of
 * calling exit() or assert().
 *
 * Conventions
 *  - All pointer arguments may point to host memory (pageable or pinned) or to device memory;
 *    the library copies through unified addressing.  Inputs are copied in; the context owns all
 *    device buffers.
 *  - Complex numbers are interleaved (re, im) doubles, i.e. the layout of the reference's
 *    double2 / complex128 files.
 *  - One context per host thread.  All device work of a call is issued on the stream passed in
 *    (NULL = the legacy default stream); set-up calls are synchronous.
 *  - Return value 0 = success, < 0 = error (see ggb_status for the message).
 */
#ifndef GGBTDDFT_H
#define GGBTDDFT_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ggb_ctx ggb_ctx;

/* precision of the step (radial propagator and angular transforms) */
enum {
  GGB_FP64 = 0,        /* complex128 orbitals, FP64 arithmetic: parity form                         */
  GGB_SPLIT_BF16 = 1,  /* complex64 orbitals, 3xBF16 split products on tcgen05, FP32 accumulation    */
  GGB_SPLIT_TF32 = 2,  /* reserved: 3xTF32 split products (not built; ggb_create returns GGB_ERR_ARG) */
  GGB_SPLIT_INT8 = 3   /* complex128 orbitals; the products' operands are cut into four int8 slices
                          on tcgen05 (kind::i8) with exact int32 accumulation: the fast form         */
};

/* angular couplings (workingData/hamiltonian/propagatorsL/<dir>):  P 001/001, FP 001/003,
   D 002/002, FF 003/003 (h_initialisePropagators.cuh:26-117) */
enum { GGB_COUPLING_P = 0, GGB_COUPLING_FP = 1, GGB_COUPLING_D = 2, GGB_COUPLING_FF = 3 };

/* run flags */
enum {
  GGB_RUN_XC_PW92 = 1,  /* add PW92 correlation to the TD exchange potential (not in the reference) */
  GGB_RUN_THETA = 2,    /* theta form (not in the reference): each angular half-step is one diagonal
                           phase at the Gauss nodes x_j of the P coupling (its eigenbasis, the V/D of
                           coupling P), exp(-i dt/2 [r E x_j + sum_{L=1}^{n_har-1} v_L(r) P_L(x_j)
                           + dv_0(r) + dv_xc(r)]), instead of the reference's FF/FP/D/P/S chain: two
                           products per half-step.  n_har <= 4: the reference's l-space multipoles;
                           4 < n_har <= 2 l_max + 1: every multipole by exact Gauss-Legendre
                           quadrature of the density on 2 N_l nodes.  Runs of a group share it; the
                           split_int8 and FP64 forms only. */
  GGB_RUN_XC_FROZEN = 4 /* keep the exchange(-correlation) potential at its t = 0 value (the Hartree
                           multipoles still follow the density); not in the reference.  With the
                           adiabatic exchange following the monopole density, all-electron argon is
                           unstable in field-free propagation (a 1e-10 perturbation grows with an
                           e-folding time of ~0.5 a.u.); with it frozen it is not. */
};

/* error codes */
enum {
  GGB_OK = 0,
  GGB_ERR_ARG = -1,       /* invalid argument / size                       */
  GGB_ERR_CUDA = -2,      /* a CUDA runtime call failed                     */
  GGB_ERR_STATE = -3,     /* call out of order (e.g. step before set-up)    */
  GGB_ERR_DEVICE = -4,    /* sticky device status set (NaN, norm growth, step overflow) */
  GGB_ERR_NOMEM = -5      /* device allocation failed                      */
};

/* A grid group: runs that share the radial grid, N_l and the radial propagators W_l. */
typedef struct ggb_group_desc {
  int n_r;      /* radial points N_r (any value >= 2; no multiple-of-32 restriction)       */
  int n_l;      /* angular momenta N_l = l_max + 1 (2 .. 220 in every form: two [N_l][32]
                   complex128 tiles of the FP64 angular kernel fit in shared memory)           */
  int n_m;      /* number of azimuthal blocks N_m (m = 0 .. n_m-1)                          */
} ggb_group_desc;

/* One atom-in-field run (one "scan" of the reference). */
typedef struct ggb_run_desc {
  int group;        /* index of its grid group                                             */
  int n_orb;        /* active Kohn-Sham orbitals N_kso                                      */
  int n_har;        /* N_har: number of Hartree multipoles (params.cuh:55)                  */
  int use_hartree;  /* USE_HARTREE (params.cuh:56)                                          */
  int target_id;    /* targetID (params.cuh:36); > 0 enables the interacting couplings      */
  int flags;        /* GGB_RUN_*                                                            */
  double dt;        /* time step (a.u.)                                                     */
} ggb_run_desc;

typedef struct ggb_dims {
  int n_groups;
  int n_runs;
  int precision;    /* GGB_FP64 / GGB_SPLIT_BF16 / GGB_SPLIT_INT8                           */
  int n_t;          /* capacity of every run's field and observable time series             */
  int per_l;        /* 1: keep dipole/acceleration per (l, orbital) as the reference does   */
} ggb_dims;

/* Create a context.  Replaces the allocations of src/main.cu:228-423. */
int ggb_create(const ggb_dims* dims, const ggb_group_desc* groups, const ggb_run_desc* runs,
               ggb_ctx** out);

/* Radial grid of a group: r, drdx = dr/dx and P = P_{N_g}(x) (workingData/mesh/{r,drdx,P}.bin;
   h_initialiseMesh.cuh:1-81). */
int ggb_set_grid(ggb_ctx* ctx, int group, const double* r, const double* drdx, const double* P,
                 int n_r);

/* Radial propagators W[l][a][b], complex128, the propagatorL%03d.bin layout
   (h_initialisePropagators.cuh:12-22).  Applied as x_l <- A x_l with A(a,b) = W[l][b][a],
   i.e. the column-major reading of cublasZgemmBatched in h_propagationH0
   (h_timePropagation.cuh:1-30). */
int ggb_set_radial_propagators(ggb_ctx* ctx, int group, const double* W);

/* Eigen-system of one angular coupling for one m: V[l][j] (N_l x N_l) and D[j] (N_l), the
   V%03d.bin / D%03d.bin files (h_initialisePropagators.cuh:26-117). */
int ggb_set_angular(ggb_ctx* ctx, int group, int coupling, int m, const double* V, const double* D);

/* Initial orbitals x[l][kso][r] (complex128), and l, m, occupation per orbital, frozen density
   (h_initialiseTDKSOSet.cuh:19-107).  Resets the run's step counter and observables. */
int ggb_set_orbitals(ggb_ctx* ctx, int run, const double* x, const int* l, const int* m,
                     const int* occ, const double* rho_frozen);

/* Laser field E[t] of a run, n_t values (h_initialiseField.cuh:1-40). */
int ggb_set_field(ggb_ctx* ctx, int run, const double* E, int n_t);

/* Advance every run by n_steps steps, asynchronously on `stream` (a cudaStream_t).
   The first call after ggb_set_orbitals computes the initial potentials
   (h_timePropagation.cuh:47-57).  Every step runs from a captured CUDA graph: a 32-step graph
   replayed n_steps / 32 times, then a 1-step graph n_steps % 32 times. */
int ggb_step(ggb_ctx* ctx, int n_steps, void* stream);

/* Profiling hook: launch one phase of the step for every group on `stream`
   (0 = angular first half, 1 = radial propagator, 2 = angular second half + partial sums,
   3 = potentials/observables).  It leaves the orbitals in an intermediate state and is meant
   only for timing a kernel alone; the state must be reset with ggb_set_orbitals afterwards.
   No counterpart in the reference. */
int ggb_launch_phase(ggb_ctx* ctx, int phase, void* stream);

/* Tiles of the int8 radial product of one grid group (split_int8 form only):
   radial_bn = orbital columns per tile (16, 32 or 64; 0 = the built-in choice from the group's
   column count), radial_stages = TMA pipeline stages (2..8, capped at what fits in shared memory;
   0 = the most that fit).  Call before the first ggb_step.  The project's autotuner
   (ggbtddft_b200/autotune.py) times the candidates for a group's (N_r, l_max, columns) and caches
   the fastest.  Returns GGB_ERR_STATE for a context of another form.  No counterpart in the
   reference (its radial product is a cuBLAS call). */
int ggb_set_tuning(ggb_ctx* ctx, int group, int radial_bn, int radial_stages);

/* split_int8 form, before the first ggb_step: on = 1 runs the angular products of `group` on the FP64
   tensor cores (the FP64 form's kernel: mma.sync m8n8k4 f64, FP64 S matrices and phases) instead of as
   int8 slice products on tcgen05; the radial product stays int8.  The angular step is then exact in
   FP64 (the int8 form's angular operands carry 31 bits).  GGB_ERR_STATE for other forms or after the
   first step.  No counterpart in the reference. */
int ggb_set_angular_fp64(ggb_ctx* ctx, int group, int on);

/* split_int8 form, theta form (GGB_RUN_THETA), before the first ggb_step: basis reuse of `group`,
   on by default.  Each angular half-step is x <- V diag(phase) V^T x with V orthogonal, and nothing
   acts on the orbitals between one step's second half and the next step's first half, so the first
   half starts from the second half's node-basis vectors (kept in FP64, one more orbital-sized buffer
   per group) and runs one product instead of two: three angular products per step instead of four.
   The omitted pair V^T V is the identity up to the int8 operands' rounding.  Setting orbitals
   invalidates the kept vectors (that step runs both products).  on = 0 keeps both products of every
   half.  GGB_ERR_STATE for other forms or after the first step; no effect with ggb_set_angular_fp64
   or without the theta form.  No counterpart in the reference (its couplings run every product). */
int ggb_set_theta_reuse(ggb_ctx* ctx, int group, int on);

/* Number of steps taken since the last ggb_set_orbitals (synchronises the context's work). */
int ggb_get_step(ggb_ctx* ctx, int* step);

/* Observables of a run for steps [0, n_steps): dip/acc are complex128.
   per_l = 1: dip[l][kso][t] as h_dipoleMoment (main.cu:395); requires ggb_dims.per_l.
   per_l = 0: dip[kso][t] = sum over l.   norm[kso][t] = sum_l sum_r |x|^2 (not in the reference).
   Any output pointer may be NULL.  Synchronises the context's work. */
int ggb_get_observables(ggb_ctx* ctx, int run, double* dip, double* acc, double* norm, int per_l,
                        int n_steps);

/* Current orbitals x[l][kso][r] of a run (complex128). */
int ggb_get_orbitals(ggb_ctx* ctx, int run, double* x);

/* Current potentials of a run: v[L][r] (L < 4), v0[r], vexc[r], vexc0[r]; any may be NULL. */
int ggb_get_potentials(ggb_ctx* ctx, int run, double* v, double* v0, double* vexc, double* vexc0);

/* Sticky device status word (bit 0 NaN/Inf, bit 1 step beyond n_t, bit 2 norm growth) and the
   last error message.  Returns the status word (>= 0) or an error code. */
int ggb_status(ggb_ctx* ctx, char* msg, int len);

/* Release every device buffer of the context. */
void ggb_destroy(ggb_ctx* ctx);

/* Observables of a set of orbitals without any device allocation.  No counterpart in the
   reference.  For callers that cannot call cudaMalloc: code running inside another framework's
   memory pool, which must own every device allocation, or a process that reserved all device
   memory up front.
   From orbitals x[l][kso][r] (complex128), the grid r[N_r] and the azimuthal numbers m[N_kso]
   (int32) it writes dip[l][kso] and acc[l][kso] (complex128: the per-(l, orbital) sums that
   ggb_get_observables records for a step) and norm[kso], on `stream`.  Every pointer must be
   device-accessible (device memory or mapped host memory); nothing is copied, and no cudaMalloc,
   cudaFree or allocating library routine is called.
   Limits: N_l <= 256, N_kso * N_l * ceil(N_r / 32) <= 65536 and N_kso * ceil(N_r / 32) <= 16384;
   larger sizes return GGB_ERR_ARG.  The partial sums live in fixed arrays inside the library
   (5.25 MiB, held on every device that loads the library until the process exits) that all calls
   share: calls that overlap on the GPU (other streams or threads) race, so serialise them.  Each
   call writes every partial it reads, so nothing has to start at zero.  The first call on a device
   looks up the arrays' device addresses (cudaGetSymbolAddress) with that device current and fills
   a table of angular coefficients (synchronously): make that first call before any stream
   capture. */
int ggb_observables_noalloc(const double* x, const double* r, const int* m, int n_l, int n_orb, int n_r,
                            double* dip, double* acc, double* norm, void* stream);

/* Peak throughput of the current GPU, measured with the library's own microbenchmark kernels (no
   device allocation): FP64 FMA on the CUDA cores in TFLOP/s, and tcgen05.mma kind::i8 (M 128, N 256,
   K 32, int32 accumulation in tensor memory) in TOP/s; either pointer may be NULL.  Synchronous on
   `stream`, a few tens of milliseconds.  These are the denominators of the roofline fractions of the
   FP64 and int8 forms.  No counterpart in the reference. */
int ggb_measure_peaks(double* fp64_tflops, double* int8_tops, void* stream);

/* Peak FP64 throughput of the current GPU's tensor cores in TFLOP/s, measured with the library's own
   kernel: independent chains of mma.sync m8n8k4 f64 in every warp of a full GPU (the instruction
   the FP64 form's angular products use).  Synchronous on `stream`.  The FP64 roofline takes the
   larger of this and the FMA figure of ggb_measure_peaks.  No counterpart in the reference. */
int ggb_measure_peak_fp64_mma(double* tflops, void* stream);

/* Library version string. */
const char* ggb_version(void);

#ifdef __cplusplus
}
#endif
#endif /* GGBTDDFT_H */
