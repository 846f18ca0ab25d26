/* mpb.h -- C ABI of the mpb B200 fixed-precision linear-algebra engine.
 *
 * Plain C: int precision, size_t sizes, void pointers, an opaque stream
 * (a cudaStream_t passed as void*, NULL = the legacy default stream).  No
 * allocation, no host synchronisation: every call validates its arguments on
 * the host, enqueues its kernels on `stream` and returns.
 *
 * Precisions: prec in {64, 128, 256, 512, 1024, 2048} bits.
 * Rounding: round-to-nearest-even after every operation, bit-exact with MPFR
 * (real, MPFR_RNDN) and MPC (complex, MPC_RNDNN); zero results are +0.
 *
 * Data layout (device buffers, "SoL tiles", see mpb/layout.cuh): a real
 * vector of n elements occupies mpb_vec_bytes(prec, n) bytes, a complex one
 * mpb_cvec_bytes(prec, n); buffers must be 16-byte aligned.  Matrices are
 * row-major with a leading dimension ld that is a multiple of 32 elements.
 * Conversions to and from the mpc_cuda AoS structs (cu_fp::cu_freal<prec>,
 * cu_fp::cu_fcomplex<prec>) and from/to double are provided on the device.
 *
 * Every entry point returns MPB_OK (0) or a negative mpb_status.  n == 0 (or
 * an empty matrix) is a valid no-op.
 *
 * Each declaration names the mpc_cuda code whose behaviour it provides.
 */
#ifndef MPB_H
#define MPB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  MPB_OK = 0,
  MPB_ERR_PREC = -1,     /* precision not in the supported set */
  MPB_ERR_SIZE = -2,     /* size overflows the addressable range */
  MPB_ERR_NULL = -3,     /* a required pointer is NULL */
  MPB_ERR_ALIGN = -4,    /* a device buffer is not 16-byte aligned */
  MPB_ERR_LD = -5,       /* leading dimension not a multiple of 32 or too small */
  MPB_ERR_CUDA = -6,     /* a CUDA launch or runtime call failed */
  MPB_ERR_ARG = -7,      /* any other invalid argument */
  MPB_ERR_WORKSPACE = -8 /* workspace missing or too small */
} mpb_status;

typedef enum { MPB_OP_MUL = 0, MPB_OP_ADD = 1, MPB_OP_SUB = 2 } mpb_op;

/* ---- library information ---- */
int mpb_version(void);                         /* major*10000 + minor*100 + patch */
const char *mpb_status_string(int status);
int mpb_prec_supported(int prec);              /* 1 if prec is one of the supported values */

/* ---- opt-in phase timing (profiling aid; off by default) ----
 * mpb_profile_enable(1) clears previous records and makes multi-kernel entry
 * points (mpb_gemm_exact_r) record a CUDA event pair around each phase on the
 * caller's stream: 0 exponent statistics, 1 slicing, 2 tensor-core GEMM,
 * 3 exact rounding (first pass), 4 fallback, 5 tensor-core recomputation of
 * the low diagonals for tiles whose truncated sum did not certify.  mpb_profile_phase_ms waits for the recorded
 * events and returns the phase's total time in ms over every call since
 * enabling (-1 if none); mpb_profile_phase_count returns the number of calls
 * recorded.  mpb_profile_phases(mask) limits the events to the phases whose
 * bit is set (default all): every event recorded between two stages costs
 * the overlap of their launches (programmatic dependent launch), measured
 * 12% of a 1024^3 exact GEMM with all phases, so time one phase at a time.
 * Inside a stream capture the events become graph nodes recorded at every
 * replay.  Not thread-safe against concurrent enable.  No counterpart in the
 * reference. */
void mpb_profile_enable(int on);
void mpb_profile_phases(unsigned mask);
float mpb_profile_phase_ms(int phase);
int mpb_profile_phase_count(int phase);

/* ---- layout ---- */
size_t mpb_vec_bytes(int prec, size_t n);      /* real vector, 0 for unsupported prec */
size_t mpb_cvec_bytes(int prec, size_t n);     /* complex vector */
size_t mpb_aos_bytes(int prec);                /* sizeof(cu_fp::cu_freal<prec>) (reference cu_freal.cuh:67-77) */

/* AoS cu_freal<prec>[n] (device) <-> tiled vector (device).
 * Replaces building/reading cu_freal arrays in place (reference cu_freal.cuh:67-81,
 * tools/test_freal.cu:56-67 copies AoS structs to and from the device). */
int mpb_pack_aos(int prec, size_t n, const void *aos, void *vec, void *stream);
int mpb_unpack_aos(int prec, size_t n, const void *vec, void *aos, void *stream);
/* AoS cu_fcomplex<prec>[n] <-> complex tiled vector (reference cu_fcomplex.cuh:98-113) */
int mpb_cpack_aos(int prec, size_t n, const void *aos, void *cvec, void *stream);
int mpb_cunpack_aos(int prec, size_t n, const void *cvec, void *aos, void *stream);
/* ---- arithmetic at a runtime precision (the hook for the reference's
 * runtime-precision layer, src/mpfr_cuda/mpfr.h:582-589, 804: cu_mpfr_add /
 * sub / mul / div / sqrt / fma with RNDN at the destination's precision) ----
 * A precision prec (1 .. 2046 bits) is stored in the vector format of
 * mpb_storage_prec(prec), the smallest supported PB >= prec + 2.  r[i] =
 * op(a[i], b[i], c[i]) correctly rounded to nearest at prec bits (rounded to
 * odd at PB bits, then to nearest at prec: exact by Boldo and Melquiond's
 * theorem); operands may carry up to PB bits, results carry prec.  b is read
 * unless op is MPB_RP_SQRT, c only for MPB_RP_FMA.  a / 0 and sqrt(a < 0)
 * give 0. */
enum { MPB_RP_MUL = 0, MPB_RP_ADD = 1, MPB_RP_SUB = 2, MPB_RP_FMA = 3, MPB_RP_DIV = 4, MPB_RP_SQRT = 5 };
int mpb_storage_prec(int prec); /* PB, or MPB_ERR_PREC */
int mpb_op_rp(int op, int prec, size_t n, const void *a, const void *b, const void *c, void *r, void *stream);
/* AXPY, GEMV and GEMM at a runtime precision prec (1 .. 2046 bits), every
 * operation correctly rounded at prec bits in the order of mpb_axpy_r /
 * mpb_gemv_r / mpb_gemm_r (MPFR with prec-bit destinations; the reference's
 * runtime layer takes its precision per call, src/mpfr_cuda/mpfr.h:582-589);
 * vectors in the layout of the storage precision mpb_storage_prec(prec). */
int mpb_axpy_r_rp(int prec, size_t n, const void *a, const void *x, const void *y, void *z, void *stream);
int mpb_gemv_r_rp(int prec, size_t m, size_t n, const void *A, size_t lda, const void *x, const void *y,
                  void *y_out, void *stream);
int mpb_gemm_r_rp(int prec, size_t m, size_t n, size_t k, const void *A, size_t lda, const void *B, size_t ldb,
                  void *C, size_t ldc, void *stream);
/* an elementary function (MPB_FN_*) at a runtime precision: faithful at the
 * storage precision, then rounded to nearest at prec bits, so within 1 ULP of
 * prec bits (the faithful contract of the reference's cu_fmath functions at a
 * precision chosen per call) */
int mpb_fmath_r_rp(int fn, int prec, size_t n, const void *a, const void *b, void *r, void *stream);

/* ---- host interop with MPFR / MPC objects (host memory, no GPU, no MPFR link) ----
 * dst[i] / src[i] point to initialised mpfr_t (mpfr_ptr) or mpc_t objects; AoS
 * arrays are cu_freal<prec> / cu_fcomplex<prec> in host memory.  To MPFR: the
 * value rounded to nearest-even at the destination's own precision (exact
 * when it is >= prec), the reference's to_mpfr (tools/test_freal.cu:28-39:
 * mpz_import, mpfr_set_z RNDN, mpfr_mul_2si).  From MPFR: rounded to
 * nearest-even at prec bits; -0 becomes +0; NaN, infinities and exponents
 * outside +-2^30 return MPB_ERR_ARG.  No counterpart in the reference's
 * library (its tests carry their own converters). */
int mpb_aos_to_mpfr(int prec, size_t n, const void *aos, void *const *dst);
int mpb_aos_from_mpfr(int prec, size_t n, const void *const *src, void *aos);
int mpb_caos_to_mpc(int prec, size_t n, const void *caos, void *const *dst);
int mpb_caos_from_mpc(int prec, size_t n, const void *const *src, void *caos);

/* double[n] -> vector, exact (reference cu_freal<PB>::from_double, cu_freal.cuh:141-149) */
int mpb_from_double(int prec, size_t n, const double *d, void *vec, void *stream);
/* vector -> double[n], RNDN (reference cu_freal<PB>::to_double, cu_freal.cuh:150-165) */
int mpb_to_double(int prec, size_t n, const void *vec, double *d, void *stream);

/* ---- element-wise operators ---- */
/* r[i] = a[i] op b[i]  (reference operators * + -, cu_freal.cuh:358-364; cu_fmul/cu_fadd/cu_fsub) */
int mpb_binop_r(int prec, int op, size_t n, const void *a, const void *b, void *r, void *stream);
/* r[i] = round(a[i]*b[i] + c[i]), one rounding (mpfr_fma; no counterpart in the reference) */
int mpb_fma_r(int prec, size_t n, const void *a, const void *b, const void *c, void *r, void *stream);
/* r[i] = round(a[i] / b[i]) and r[i] = round(sqrt(a[i])), one rounding each
 * (mpfr_div / mpfr_sqrt; the drop-in cu_fdiv / cu_sqrt).  They replace the
 * reference's faithful cu_fdiv / cu_sqrt (include/mpc_cuda/cu_fmath.cuh:67-75,
 * 92-100) with correctly rounded ones.  b[i] = 0 or a[i] < 0 gives 0 (the
 * format has no infinities or NaN). */
int mpb_div_r(int prec, size_t n, const void *a, const void *b, void *r, void *stream);
int mpb_sqrt_r(int prec, size_t n, const void *a, void *r, void *stream);
/* r[i] = exp(a[i]), r[i] = log(a[i]): faithful (at most 1 ULP from the exact
 * value), the contract of the reference's cu_exp / cu_log
 * (include/mpc_cuda/cu_fmath.cuh:197-218); computed at 128 guard bits.  exp
 * of |a| >= 2^29 (result outside the exponent range) and log of a <= 0 give 0. */
int mpb_exp_r(int prec, size_t n, const void *a, void *r, void *stream);
int mpb_log_r(int prec, size_t n, const void *a, void *r, void *stream);

/* ---- elementary functions (reference include/mpc_cuda/cu_fmath.cuh:119-424,
 * cu_fcmath.cuh:13-113; the drop-in cu_<name> of the C++ surface) ----
 * Faithful (at most 1 ULP per component from the exact value; in practice
 * correctly rounded), computed at 128 guard bits like the reference's.  Each
 * function fn runs over n elements: r[i] = fn(a[i]) (pow and atan2 also read
 * b[i]).  Values with no representation in the format (no NaN or infinity)
 * give 0: exp / expm1 / sinh / cosh overflow (|a| >= 2^29), sin / cos / tan
 * of |a| >= 2^30, log of a <= 0, log1p of a <= -1, atanh of |a| >= 1, pow of
 * a negative a and a non-integer b, a complex division by zero.  asin of
 * |a| >= 1 gives +-pi/2, acos of a >= 1 gives 0 and of a <= -1 pi (the
 * reference's clamps, cu_fmath.cuh:382-399). */
enum {
  MPB_FN_EXP = 0,    /* cu_exp   cu_fmath.cuh:197 */
  MPB_FN_LOG = 1,    /* cu_log   :214 */
  MPB_FN_EXPM1 = 2,  /* cu_expm1 :234 */
  MPB_FN_LOG1P = 3,  /* cu_log1p :247 */
  MPB_FN_SIN = 4,    /* cu_sin   :293 */
  MPB_FN_COS = 5,    /* cu_cos   :299 */
  MPB_FN_TAN = 6,    /* cu_tan   :305 */
  MPB_FN_ATAN = 7,   /* cu_atan  :329 */
  MPB_FN_SINH = 8,   /* cu_sinh  :353 */
  MPB_FN_COSH = 9,   /* cu_cosh  :356 */
  MPB_FN_ATANH = 10, /* cu_atanh :373 */
  MPB_FN_ASIN = 11,  /* cu_asin  :389 */
  MPB_FN_ACOS = 12,  /* cu_acos  :401 */
  MPB_FN_CBRT = 13,  /* cu_cbrt  :119 (sign kept) */
  MPB_FN_POW = 14,   /* cu_pow(a, b) :420 */
  MPB_FN_ATAN2 = 15  /* atan2(a, b) = the angle of (b, a), cu_fcmath.cuh:20 (cu_atan2_w) */
};
int mpb_fmath_r(int fn, int prec, size_t n, const void *a, const void *b, void *r, void *stream);
/* complex (arrays of complex elements, each component faithful) */
enum {
  MPB_CFN_EXP = 0,  /* cu_cexp   cu_fcmath.cuh:47 */
  MPB_CFN_LOG = 1,  /* cu_clog   :52 */
  MPB_CFN_SQRT = 2, /* cu_csqrt  :58 (principal root) */
  MPB_CFN_SIN = 3,  /* cu_csin   :74 */
  MPB_CFN_COS = 4,  /* cu_ccos   :80 */
  MPB_CFN_TAN = 5,  /* cu_ctan   :98 */
  MPB_CFN_SINH = 6, /* cu_csinh  :86 */
  MPB_CFN_COSH = 7, /* cu_ccosh  :92 */
  MPB_CFN_DIV = 8   /* cu_cdiv(a, b) :42 */
};
int mpb_fmath_c(int fn, int prec, size_t n, const void *a, const void *b, void *r, void *stream);
/* r[i] = round(a[i] / u), one rounding (mpfr_div_ui; the reference's
 * cu_div_ui, cu_fmath.cuh:32-50, which is also correctly rounded); u = 0 gives 0 */
int mpb_div_ui_r(int prec, size_t n, const void *a, uint64_t u, void *r, void *stream);
/* r[0 .. n) = pi (which = MPB_CONST_PI) or ln 2 (MPB_CONST_LN2), correctly
 * rounded (the reference's cu_pi / cu_ln2, cu_fmath.cuh:174-175) */
enum { MPB_CONST_PI = 0, MPB_CONST_LN2 = 1 };
int mpb_const_r(int which, int prec, size_t n, void *r, void *stream);
/* complex r[i] = a[i]*b[i] + c[i], one rounding per component from exact
 * products (mpc_fma; the drop-in cu_cfma; no counterpart in the reference) */
int mpb_fma_c(int prec, size_t n, const void *a, const void *b, const void *c, void *r, void *stream);
/* complex r[i] = a[i] op b[i] (reference cu_cmul/cu_cadd/cu_csub, cu_fcomplex.cuh:115-131) */
int mpb_binop_c(int prec, int op, size_t n, const void *a, const void *b, void *r, void *stream);

/* ---- AXPY ---- */
/* z[i] = round(round(a*x[i]) + y[i]); a is element 0 of a real vector
 * (reference freal_axpy, demos/bench_3way.cu:44-50) */
int mpb_axpy_r(int prec, size_t n, const void *a, const void *x, const void *y, void *z, void *stream);
/* complex z[i] = a*x[i] + y[i], MPC_RNDNN per operation
 * (reference fcplx_axpy, demos/bench_3way.cu:51-59; axpyc, tools/axpy_fast_complex.cu:32-40) */
int mpb_axpy_c(int prec, size_t n, const void *a, const void *x, const void *y, void *z, void *stream);

/* ---- GEMV / GEMM, per-operation rounding in sequential k order ---- */
/* y_out[i] = round(dot_i + y[i]), dot_i: acc = +0; acc = round(acc + round(A[i,k]*x[k])), k = 0..n-1.
 * A is m x n (row-major, lda).  y_out may alias y.
 * (reference matvec_kernel, tools/linalg_fast.cu:37-51, which has no "+ y") */
int mpb_gemv_r(int prec, size_t m, size_t n, const void *A, size_t lda, const void *x, const void *y,
               void *y_out, void *stream);
int mpb_gemv_c(int prec, size_t m, size_t n, const void *A, size_t lda, const void *x, const void *y,
               void *y_out, void *stream);
/* C[i,j] = sequential-k dot of row i of A (m x k) and column j of B (k x n)
 * (reference matmul_kernel, tools/linalg_fast.cu:53-68; complex order of
 * cdot_ij, demos/matmul_mpc.cu:39-57) */
int mpb_gemm_r(int prec, size_t m, size_t n, size_t k, const void *A, size_t lda, const void *B, size_t ldb,
               void *C, size_t ldc, void *stream);
int mpb_gemm_c(int prec, size_t m, size_t n, size_t k, const void *A, size_t lda, const void *B, size_t ldb,
               void *C, size_t ldc, void *stream);

/* ---- thread-vs-warp split ---- */
/* Kernels with a warp-cooperative form for wide operands: one element (a
 * complex AXPY element, a GEMV row) per thread, or per group of `lanes`
 * lanes that hold its limbs between them (lanes 4 or 8 at 1024 bits, 8 or 16
 * at 2048 bits; the complex AXPY has the cooperative form at 1024 bits).
 * Results are identical either way; the split only changes the speed.  The
 * setting is process-wide, read at every launch; the defaults are the
 * fastest forms measured on B200.  No counterpart in the reference (its
 * kernels are one thread per element, demos/bench_3way.cu:44-59).
 * Returns MPB_ERR_ARG for a kind or lane count not offered at that precision. */
enum { MPB_SPLIT_AXPY_C = 0, MPB_SPLIT_GEMV_R = 1 };
int mpb_set_split(int kind, int prec, int lanes);
int mpb_get_split(int kind, int prec, int *lanes);

/* ---- plain GEMM block shape ---- */
/* The plain GEMM (mpb_gemm_r / mpb_gemm_c) runs one thread per output: a warp
 * owns one row of C and 32 columns, a block `warps` rows (4, 8 or 16).  Few
 * blocks (a small C) favour 4, wide operands whose register need caps the
 * resident blocks may favour 16; results are identical for every shape.  The
 * setting is process-wide per real/complex and precision, read at every
 * launch (default 8); mpc_cuda_b200.tune.autotune_gemm_warps times the shapes
 * on a problem and keeps the fastest.  Returns MPB_ERR_ARG for another
 * warp count. */
int mpb_set_gemm_warps(int cplx, int prec, int warps);
int mpb_get_gemm_warps(int cplx, int prec, int *warps);

/* ---- batched GEMV: thousands of independent problems, mixed sizes and precisions ---- */
/* One problem y_out = A.x + y (real, prec bits, same order as mpb_gemv_r).
 * Device pointers; lda a multiple of 32 (>= n); m or n may be 0. */
typedef struct {
  int prec;
  int m, n;
  size_t lda;
  const void *A, *x, *y;
  void *y_out;
} mpb_gemv_problem;
typedef struct mpb_batch_plan mpb_batch_plan;
/* Bytes of device workspace a plan for `count` problems needs (256-byte aligned). */
size_t mpb_batch_gemv_workspace(int count);
/* Validate the problems (host array), group them by precision, order each
 * group longest first and upload descriptors and work queues to the
 * workspace (synchronous); returns an opaque host-side plan.  The reference
 * has no batched path (its matvec is tools/linalg_fast.cu:37-51). */
int mpb_batch_gemv_plan(int count, const mpb_gemv_problem *problems, void *workspace, size_t ws_bytes,
                        mpb_batch_plan **plan);
/* Run every planned problem: one persistent kernel per precision present,
 * largest precision first, each over the whole GPU, all on `stream`; no
 * allocation, no host synchronisation (can be captured into a CUDA graph).
 * Runs of one plan must not overlap (they share the workspace queues). */
int mpb_batch_gemv_run(mpb_batch_plan *plan, void *stream);
/* Time each precision group with every candidate launch shape on the planned
 * batch (synchronous) and keep the fastest in the plan. */
int mpb_batch_gemv_autotune(mpb_batch_plan *plan, void *stream);
/* Read / install the launch shape of a precision group (threads per block, a
 * multiple of 32 up to 256; persistent blocks per SM, 0 = occupancy limit). */
int mpb_batch_gemv_get_tuning(const mpb_batch_plan *plan, int prec, int *block, int *blocks_per_sm);
int mpb_batch_gemv_set_tuning(mpb_batch_plan *plan, int prec, int block, int blocks_per_sm);
/* Read / install the thread-vs-warp split of a precision group: lanes per row
 * (1, or 4 / 8 at 1024 bits, 8 / 16 at 2048 bits; see mpb_set_split).  The
 * autotuner tries every split with every launch shape. */
int mpb_batch_gemv_get_split(const mpb_batch_plan *plan, int prec, int *lanes);
int mpb_batch_gemv_set_split(mpb_batch_plan *plan, int prec, int lanes);
/* Time of one run of the precision's problems alone on the whole GPU, as
 * measured by the last mpb_batch_gemv_autotune (-1 before any; 0 when the
 * batch has no problem of that precision). */
int mpb_batch_gemv_tuned_ms(const mpb_batch_plan *plan, int prec, float *ms);
void mpb_batch_gemv_destroy(mpb_batch_plan *plan);

/* ---- exact-accumulation GEMM on the INT8 tensor cores (no counterpart in the reference) ---- */
/* C[i,j] = RNDN(sum_k A[i,k]*B[k,j]) with ONE rounding per entry: the correctly
 * rounded dot product (MPFR mpfr_dot semantics; <= 0.5 ULP).  Each row of A and
 * column of B is aligned to its largest exponent; entries more than sp_bits
 * below it do not fit the slice budget, and such rows / columns are computed
 * by the plain per-operation-rounded kernel instead (never on the CPU).
 * workspace: device scratch of mpb_gemm_exact_workspace(...) bytes, 256-byte
 * aligned, owned by the caller; calls sharing a workspace must not overlap.
 * status: optional device int[2], written asynchronously: [0] = number of rows
 * plus columns that took the fallback, [1] = 0 or an internal kernel error code.
 * The slice budget costs S = ceil((prec + sp_bits + 2) / 8) digit slices;
 * sp_bits <= 118 is supported.  The low-order slice pairs, which only reach
 * bits far below each result's ULP, are skipped, and each rounding is
 * certified against a bound on what they could add; an entry that does not
 * certify (heavy cancellation, or a sum next to a rounding midpoint) is
 * recomputed from the full sum, so the result is always correctly rounded. */
size_t mpb_gemm_exact_workspace(int prec, size_t m, size_t n, size_t k, int sp_bits);
size_t mpb_gemm_exact_c_workspace(int prec, size_t m, size_t n, size_t k, int sp_bits);
int mpb_gemm_exact_r(int prec, size_t m, size_t n, size_t k, const void *A, size_t lda, const void *B, size_t ldb,
                     void *C, size_t ldc, int sp_bits, void *workspace, size_t ws_bytes, int *status, void *stream);
/* complex: each component rounded once (MPC mpc_dot semantics), computed in
 * the 3-multiplication form re = T0 - T1, im = T2 - T0 - T1 on exact integers
 * (T0 = Ar.Br, T1 = Ai.Bi, T2 = (Ar+Ai).(Br+Bi)); S = ceil((prec+sp_bits+3)/8).
 * Complex operands and result use complex tiles; workspace size from
 * mpb_gemm_exact_c_workspace. */
int mpb_gemm_exact_c(int prec, size_t m, size_t n, size_t k, const void *A, size_t lda, const void *B, size_t ldb,
                     void *C, size_t ldc, int sp_bits, void *workspace, size_t ws_bytes, int *status, void *stream);
/* Geometry of an exact GEMM call (cplx 0 real, 1 complex): the number of digit
 * slices S, the lowest diagonal the tensor cores compute for every tile, and
 * the slice pairs that costs per real product and multiply-add (the int8
 * tensor-core work is 2 * pairs * m * n * k per real product). */
int mpb_gemm_exact_plan_info(int prec, size_t m, size_t n, size_t k, int sp_bits, int cplx, int *slices,
                             int *first_diag, long long *pairs);
/* Test of the failure path (no counterpart in the reference): the next
 * tensor-core launch of an exact GEMM in this process runs with one
 * accumulator commit withheld in its first CTA and every barrier wait limited
 * to wait_ns nanoseconds (1e3 .. 2e9), so that CTA's wait runs out.  The
 * kernel then raises its abort flag, records an error code (1-4) in the
 * call's status[1], waits for its own MMAs and copies, frees its tensor
 * memory and returns: the results of that call are not valid, and the next
 * call on the same stream is correct again.  what: 1.  MPB_ERR_ARG otherwise. */
int mpb_gemm_exact_test_inject(int what, long long wait_ns);
/* The same exact GEMM for callers that cannot allocate device memory (a
 * latency-critical loop that must not call cudaMalloc after start-up, or a
 * framework that owns the whole memory pool): no workspace argument and no
 * allocation; the scratch is a fixed 16 MiB area inside the library, reserved
 * on every GPU that loads it.  Problems needing more scratch than that
 * (mpb_gemm_exact_workspace(...) > 16 MiB) return MPB_ERR_SIZE.  The first call
 * on a device looks the area up and should come before any stream capture.
 * All calls share the area, so calls that overlap on the GPU race.  No
 * counterpart in the reference. */
int mpb_gemm_exact_r_static(int prec, size_t m, size_t n, size_t k, const void *A, size_t lda, const void *B,
                            size_t ldb, void *C, size_t ldc, int sp_bits, int *status, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MPB_H */
