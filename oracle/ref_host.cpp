/* ref_host.cpp -- ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Builds the reference's OWN fixed-precision arithmetic for the host CPU:
 * the mpc_cuda headers include/mpc_cuda/cu_freal.cuh and cu_fcomplex.cuh are
 * host-capable by design (cu_freal.cuh:23-32 turns __host__/__device__ into
 * no-ops and uses __uint128_t, cu_freal.cuh:46-47), so this file includes them
 * straight from the reference tree (-I <reference>/include; nothing is copied)
 * and exposes the operations the CUDA engine must reproduce through a small
 * extern "C" surface over AoS arrays of cu_fp::cu_freal<PB> / cu_fcomplex<PB>.
 *
 * The result, oracle/_ref/libref_host.so, is the "reference" CPU baseline and a
 * second, independent check of the C restatement in mpb_oracle.c.  The loops
 * mirror the reference kernels: demos/bench_3way.cu:44-59 (AXPY),
 * tools/linalg_fast.cu:37-68 (sequential-k matvec/matmul),
 * demos/matmul_mpc.cu:39-57 (complex sequential-k order).
 */
#include <cstdint>
#include <cstring>
#include "mpc_cuda/cu_fcomplex.cuh"
#include "mpc_cuda/cu_fmath.cuh"
#include "mpc_cuda/cu_fcmath.cuh"

using cu_fp::cu_fcomplex;
using cu_fp::cu_freal;

namespace {

template <int PB>
void t_mul(long n, const void *A, const void *B, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto b = (const cu_freal<PB> *)B;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_fmul<PB>(a[i], b[i]);
}
/* the reference's division and square root (cu_fmath.cuh:67-75, 92-100:
 * Newton iteration at PB + CU_FGUARD bits, faithful) -- the CPU baseline of
 * the engine's correctly rounded mpb_div_r / mpb_sqrt_r */
template <int PB>
void t_div(long n, const void *A, const void *B, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto b = (const cu_freal<PB> *)B;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_fdiv<PB>(a[i], b[i]);
}
template <int PB>
void t_sqrt(long n, const void *A, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_sqrt<PB>(a[i]);
}
template <int PB>
void t_exp(long n, const void *A, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_exp<PB>(a[i]);
}
template <int PB>
void t_log(long n, const void *A, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_log<PB>(a[i]);
}
template <int PB>
void t_add(long n, const void *A, const void *B, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto b = (const cu_freal<PB> *)B;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_fadd<PB>(a[i], b[i]);
}
template <int PB>
void t_sub(long n, const void *A, const void *B, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto b = (const cu_freal<PB> *)B;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_fsub<PB>(a[i], b[i]);
}
template <int PB>
void t_cmul(long n, const void *A, const void *B, void *R) {
  auto a = (const cu_fcomplex<PB> *)A;
  auto b = (const cu_fcomplex<PB> *)B;
  auto r = (cu_fcomplex<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_cmul<PB>(a[i], b[i]);
}
template <int PB>
void t_cadd(long n, const void *A, const void *B, void *R) {
  auto a = (const cu_fcomplex<PB> *)A;
  auto b = (const cu_fcomplex<PB> *)B;
  auto r = (cu_fcomplex<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_cadd<PB>(a[i], b[i]);
}
template <int PB>
void t_csub(long n, const void *A, const void *B, void *R) {
  auto a = (const cu_fcomplex<PB> *)A;
  auto b = (const cu_fcomplex<PB> *)B;
  auto r = (cu_fcomplex<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_csub<PB>(a[i], b[i]);
}
/* freal_axpy body (demos/bench_3way.cu:47-48): t = a*x; r = t + y */
template <int PB>
void t_axpy_r(long n, const void *a, const void *X, const void *Y, void *Z) {
  const cu_freal<PB> &s = *(const cu_freal<PB> *)a;
  auto x = (const cu_freal<PB> *)X;
  auto y = (const cu_freal<PB> *)Y;
  auto z = (cu_freal<PB> *)Z;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    cu_freal<PB> t = s * x[i];
    z[i] = t + y[i];
  }
}
/* fcplx_axpy body (demos/bench_3way.cu:55-56) */
template <int PB>
void t_axpy_c(long n, const void *a, const void *X, const void *Y, void *Z) {
  const cu_fcomplex<PB> &s = *(const cu_fcomplex<PB> *)a;
  auto x = (const cu_fcomplex<PB> *)X;
  auto y = (const cu_fcomplex<PB> *)Y;
  auto z = (cu_fcomplex<PB> *)Z;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    cu_fcomplex<PB> t = s * x[i];
    z[i] = t + y[i];
  }
}
/* matvec_kernel body (tools/linalg_fast.cu:43-48) plus the engine's final +y */
template <int PB>
void t_gemv_r(long m, long n, const void *A, long lda, const void *X, const void *Yin, void *Yout) {
  auto a = (const cu_freal<PB> *)A;
  auto x = (const cu_freal<PB> *)X;
  auto yi = (const cu_freal<PB> *)Yin;
  auto yo = (cu_freal<PB> *)Yout;
#pragma omp parallel for schedule(dynamic, 4)
  for (long i = 0; i < m; i++) {
    cu_freal<PB> acc;
    acc.set_zero();
    for (long k = 0; k < n; k++) acc = cu_fp::cu_fadd<PB>(acc, cu_fp::cu_fmul<PB>(a[i * lda + k], x[k]));
    yo[i] = cu_fp::cu_fadd<PB>(acc, yi[i]);
  }
}
template <int PB>
void t_gemv_c(long m, long n, const void *A, long lda, const void *X, const void *Yin, void *Yout) {
  auto a = (const cu_fcomplex<PB> *)A;
  auto x = (const cu_fcomplex<PB> *)X;
  auto yi = (const cu_fcomplex<PB> *)Yin;
  auto yo = (cu_fcomplex<PB> *)Yout;
#pragma omp parallel for schedule(dynamic, 4)
  for (long i = 0; i < m; i++) {
    cu_fcomplex<PB> acc;
    acc.re.set_zero();
    acc.im.set_zero();
    for (long k = 0; k < n; k++) acc = acc + a[i * lda + k] * x[k];
    yo[i] = acc + yi[i];
  }
}
/* matmul_kernel body (tools/linalg_fast.cu:59-66), rows [r0, r1) */
template <int PB>
void t_gemm_r(long m, long n, long K, const void *A, long lda, const void *B, long ldb, void *C,
              long ldc, long r0, long r1) {
  auto a = (const cu_freal<PB> *)A;
  auto b = (const cu_freal<PB> *)B;
  auto c = (cu_freal<PB> *)C;
  if (r1 <= 0 || r1 > m) r1 = m;
#pragma omp parallel for collapse(2) schedule(dynamic, 16)
  for (long i = r0; i < r1; i++)
    for (long j = 0; j < n; j++) {
      cu_freal<PB> acc;
      acc.set_zero();
      for (long k = 0; k < K; k++)
        acc = cu_fp::cu_fadd<PB>(acc, cu_fp::cu_fmul<PB>(a[i * lda + k], b[k * ldb + j]));
      c[i * ldc + j] = acc;
    }
}
/* complex sequential-k order of cdot_ij (demos/matmul_mpc.cu:39-57) */
template <int PB>
void t_gemm_c(long m, long n, long K, const void *A, long lda, const void *B, long ldb, void *C,
              long ldc, long r0, long r1) {
  auto a = (const cu_fcomplex<PB> *)A;
  auto b = (const cu_fcomplex<PB> *)B;
  auto c = (cu_fcomplex<PB> *)C;
  if (r1 <= 0 || r1 > m) r1 = m;
#pragma omp parallel for collapse(2) schedule(dynamic, 16)
  for (long i = r0; i < r1; i++)
    for (long j = 0; j < n; j++) {
      cu_fcomplex<PB> acc;
      acc.re.set_zero();
      acc.im.set_zero();
      for (long k = 0; k < K; k++) acc = acc + a[i * lda + k] * b[k * ldb + j];
      c[i * ldc + j] = acc;
    }
}
template <int PB>
void t_from_double(long n, const double *d, void *R) {
  auto r = (cu_freal<PB> *)R;
  for (long i = 0; i < n; i++) r[i] = cu_freal<PB>::from_double(d[i]);
}
template <int PB>
void t_to_double(long n, const void *X, double *d) {
  auto x = (const cu_freal<PB> *)X;
  for (long i = 0; i < n; i++) d[i] = x[i].to_double();
}

/* runtime precision -> template instantiation (the reference's test set,
 * tools/test_freal.cu:92-102, plus the engine's PB list) */
/* the reference's elementary functions, numbered as the engine's MPB_FN_* /
 * MPB_CFN_* (its cu_atan2 exists only at working precision, cu_atan2_w) */
template <int PB>
void t_fn(int fn, long n, const void *A, const void *B, void *R) {
  using namespace cu_fp;
  auto a = (const cu_freal<PB> *)A;
  auto b = (const cu_freal<PB> *)B;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(dynamic, 16)
  for (long i = 0; i < n; i++) {
    const cu_freal<PB> x = a[i];
    switch (fn) {
      case 0: r[i] = cu_exp<PB>(x); break;
      case 1: r[i] = cu_log<PB>(x); break;
      case 2: r[i] = cu_expm1<PB>(x); break;
      case 3: r[i] = cu_log1p<PB>(x); break;
      case 4: r[i] = cu_sin<PB>(x); break;
      case 5: r[i] = cu_cos<PB>(x); break;
      case 6: r[i] = cu_tan<PB>(x); break;
      case 7: r[i] = cu_atan<PB>(x); break;
      case 8: r[i] = cu_sinh<PB>(x); break;
      case 9: r[i] = cu_cosh<PB>(x); break;
      case 10: r[i] = cu_atanh<PB>(x); break;
      case 11: r[i] = cu_asin<PB>(x); break;
      case 12: r[i] = cu_acos<PB>(x); break;
      case 13: r[i] = cu_cbrt<PB>(x); break;
      case 14: r[i] = cu_pow<PB>(x, b[i]); break;
      default: {
        const int W = PB + CU_FGUARD;
        r[i] = cu_convert<PB>(cu_atan2_w<W>(cu_convert<W>(x), cu_convert<W>(b[i])));
      }
    }
  }
}
template <int PB>
void t_cfn(int fn, long n, const void *A, const void *B, void *R) {
  using namespace cu_fp;
  auto a = (const cu_fcomplex<PB> *)A;
  auto b = (const cu_fcomplex<PB> *)B;
  auto r = (cu_fcomplex<PB> *)R;
#pragma omp parallel for schedule(dynamic, 16)
  for (long i = 0; i < n; i++) {
    const cu_fcomplex<PB> z = a[i];
    switch (fn) {
      case 0: r[i] = cu_cexp<PB>(z); break;
      case 1: r[i] = cu_clog<PB>(z); break;
      case 2: r[i] = cu_csqrt<PB>(z); break;
      case 3: r[i] = cu_csin<PB>(z); break;
      case 4: r[i] = cu_ccos<PB>(z); break;
      case 5: r[i] = cu_ctan<PB>(z); break;
      case 6: r[i] = cu_csinh<PB>(z); break;
      case 7: r[i] = cu_ccosh<PB>(z); break;
      default: r[i] = cu_cdiv<PB>(z, b[i]);
    }
  }
}

/* utilities over AoS arrays (test surface): op 0 cu_cmp(a, b), 1 cu_cmpmag(a, b),
 * 2 cu_lround(a) into iv; 3 cu_from_si(iv) into r */
template <int PB>
void util1(int op, long n, const void *A, const void *B, long *iv, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto b = (const cu_freal<PB> *)B;
  auto r = (cu_freal<PB> *)R;
  for (long i = 0; i < n; i++) {
    switch (op) {
      case 0: iv[i] = cu_fp::cu_cmp<PB>(a[i], b[i]); break;
      case 1: iv[i] = cu_fp::cu_cmpmag<PB>(a[i], b[i]); break;
      case 2: iv[i] = cu_fp::cu_lround<PB>(a[i]); break;
      default: r[i] = cu_fp::cu_from_si<PB>(iv[i]);
    }
  }
}
/* finalize over n rows: D row i = 4 limbs, q row i = { len, msb, Ehi, brnd, bsti, sgn } */
template <int PB>
void finalize1(long n, const unsigned long long *D, const long *q, void *R) {
  auto r = (cu_freal<PB> *)R;
  for (long i = 0; i < n; i++) {
    const long *p = q + 6 * i;
    r[i] = cu_freal<PB>::finalize(D + 4 * i, (int)p[0], (int)p[1], p[2], (unsigned long long)p[3],
                                  (unsigned long long)p[4], (int)p[5]);
  }
}
/* exact product terms (test surface): hdr row i = { sign, exp, zero } and the
 * WN limbs of cu_mk_term(a[i], b[i]); r[i] = cu_round_sum2 of that term and
 * the negated term of (c[i], d[i]) */
template <int PB>
void terms1(long n, const void *A, const void *B, const void *Cc, const void *Dd, long *hdr,
            unsigned long long *M, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto b = (const cu_freal<PB> *)B;
  auto c = (const cu_freal<PB> *)Cc;
  auto d = (const cu_freal<PB> *)Dd;
  auto r = (cu_freal<PB> *)R;
  const int WN = cu_fp::cu_wterm<PB>::WN;
  for (long i = 0; i < n; i++) {
    const cu_fp::cu_wterm<PB> t = cu_fp::cu_mk_term<PB>(a[i], b[i]);
    hdr[3 * i] = t.sign;
    hdr[3 * i + 1] = t.exp;
    hdr[3 * i + 2] = t.zero ? 1 : 0;
    for (int k = 0; k < WN; k++) M[(long)WN * i + k] = t.M[k];
    cu_fp::cu_wterm<PB> u = cu_fp::cu_mk_term<PB>(c[i], d[i]);
    u.sign = -u.sign;
    r[i] = cu_fp::cu_round_sum2<PB>(t, u);
  }
}
template <int TO, int FROM>
void convert1(long n, const void *X, void *R) {
  auto x = (const cu_freal<FROM> *)X;
  auto r = (cu_freal<TO> *)R;
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_convert<TO, FROM>(x[i]);
}
#define UTIL_SMALL_DISPATCH(P, CALL)                          \
  switch (P) {                                                \
    case 32: { constexpr int PB = 32; CALL; } break;          \
    case 96: { constexpr int PB = 96; CALL; } break;          \
    case 160: { constexpr int PB = 160; CALL; } break;        \
    case 256: { constexpr int PB = 256; CALL; } break;        \
    case 288: { constexpr int PB = 288; CALL; } break;        \
    case 1056: { constexpr int PB = 1056; CALL; } break;      \
    default: return -1;                                       \
  }
template <int TO>
int convert_to(int from, long n, const void *X, void *R) {
  UTIL_SMALL_DISPATCH(from, (convert1<TO, PB>(n, X, R)))
  return 0;
}

#define REF_DISPATCH(P, CALL)                                                                   \
  switch (P) {                                                                                  \
    case 32: { constexpr int PB = 32; CALL; } return 0;                                         \
    case 64: { constexpr int PB = 64; CALL; } return 0;                                         \
    case 96: { constexpr int PB = 96; CALL; } return 0;                                         \
    case 128: { constexpr int PB = 128; CALL; } return 0;                                       \
    case 160: { constexpr int PB = 160; CALL; } return 0;                                       \
    case 256: { constexpr int PB = 256; CALL; } return 0;                                       \
    case 288: { constexpr int PB = 288; CALL; } return 0;                                       \
    case 512: { constexpr int PB = 512; CALL; } return 0;                                       \
    case 1024: { constexpr int PB = 1024; CALL; } return 0;                                     \
    case 1056: { constexpr int PB = 1056; CALL; } return 0;                                     \
    case 2048: { constexpr int PB = 2048; CALL; } return 0;                                     \
    default: return -1;                                                                         \
  }

}  // namespace

extern "C" {
int ref_elem_bytes(int P) { REF_DISPATCH(P, return (int)sizeof(cu_freal<PB>)) }
int ref_mul(int P, long n, const void *A, const void *B, void *R) { REF_DISPATCH(P, t_mul<PB>(n, A, B, R)) }
int ref_add(int P, long n, const void *A, const void *B, void *R) { REF_DISPATCH(P, t_add<PB>(n, A, B, R)) }
int ref_div(int P, long n, const void *A, const void *B, void *R) { REF_DISPATCH(P, t_div<PB>(n, A, B, R)) }
int ref_sqrt(int P, long n, const void *A, void *R) { REF_DISPATCH(P, t_sqrt<PB>(n, A, R)) }
int ref_exp(int P, long n, const void *A, void *R) { REF_DISPATCH(P, t_exp<PB>(n, A, R)) }
int ref_log(int P, long n, const void *A, void *R) { REF_DISPATCH(P, t_log<PB>(n, A, R)) }
int ref_fn(int fn, int P, long n, const void *A, const void *B, void *R) {
  REF_DISPATCH(P, t_fn<PB>(fn, n, A, B, R))
}
int ref_cfn(int fn, int P, long n, const void *A, const void *B, void *R) {
  REF_DISPATCH(P, t_cfn<PB>(fn, n, A, B, R))
}
int ref_sub(int P, long n, const void *A, const void *B, void *R) { REF_DISPATCH(P, t_sub<PB>(n, A, B, R)) }
int ref_cmul(int P, long n, const void *A, const void *B, void *R) { REF_DISPATCH(P, t_cmul<PB>(n, A, B, R)) }
int ref_cadd(int P, long n, const void *A, const void *B, void *R) { REF_DISPATCH(P, t_cadd<PB>(n, A, B, R)) }
int ref_csub(int P, long n, const void *A, const void *B, void *R) { REF_DISPATCH(P, t_csub<PB>(n, A, B, R)) }
int ref_axpy_r(int P, long n, const void *a, const void *X, const void *Y, void *Z) {
  REF_DISPATCH(P, t_axpy_r<PB>(n, a, X, Y, Z))
}
int ref_axpy_c(int P, long n, const void *a, const void *X, const void *Y, void *Z) {
  REF_DISPATCH(P, t_axpy_c<PB>(n, a, X, Y, Z))
}
int ref_gemv_r(int P, long m, long n, const void *A, long lda, const void *X, const void *Yi, void *Yo) {
  REF_DISPATCH(P, t_gemv_r<PB>(m, n, A, lda, X, Yi, Yo))
}
int ref_gemv_c(int P, long m, long n, const void *A, long lda, const void *X, const void *Yi, void *Yo) {
  REF_DISPATCH(P, t_gemv_c<PB>(m, n, A, lda, X, Yi, Yo))
}
int ref_gemm_r(int P, long m, long n, long k, const void *A, long lda, const void *B, long ldb,
               void *C, long ldc, long r0, long r1) {
  REF_DISPATCH(P, t_gemm_r<PB>(m, n, k, A, lda, B, ldb, C, ldc, r0, r1))
}
int ref_gemm_c(int P, long m, long n, long k, const void *A, long lda, const void *B, long ldb,
               void *C, long ldc, long r0, long r1) {
  REF_DISPATCH(P, t_gemm_c<PB>(m, n, k, A, lda, B, ldb, C, ldc, r0, r1))
}
int ref_from_double(int P, long n, const double *d, void *R) { REF_DISPATCH(P, t_from_double<PB>(n, d, R)) }
int ref_to_double(int P, long n, const void *X, double *d) { REF_DISPATCH(P, t_to_double<PB>(n, X, d)) }
int ref_util(int op, int P, long n, const void *A, const void *B, long *iv, void *R) {
  if (op < 0 || op > 3) return -2;
  REF_DISPATCH(P, util1<PB>(op, n, A, B, iv, R))
}
int ref_finalize(int P, long n, const unsigned long long *D, const long *q, void *R) {
  REF_DISPATCH(P, finalize1<PB>(n, D, q, R))
}
int ref_terms(int P, long n, const void *A, const void *B, const void *Cc, const void *Dd, long *hdr,
                 unsigned long long *M, void *R) {
  REF_DISPATCH(P, terms1<PB>(n, A, B, Cc, Dd, hdr, M, R))
}
/* cu_convert<to, from> for to, from in {32, 96, 160, 256, 288, 1056} */
int ref_convert(int to, int from, long n, const void *X, void *R) {
  UTIL_SMALL_DISPATCH(to, return convert_to<PB>(from, n, X, R))
  return -1;
}
}
