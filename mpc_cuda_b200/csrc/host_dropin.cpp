/* host_dropin.cpp -- host (CPU) build of the drop-in cu_fp surface.
 *
 * The reference's fixed-precision types run on the host as well as on the GPU
 * (mpc_cuda include/mpc_cuda/cu_freal.cuh:23-32; host use in
 * demos/sample_fixed.cu:59-67 and tools/bench_cpu.cpp:31-70).  This library
 * exposes the drop-in cu_freal / cu_fcomplex operators of this engine, built
 * for the host, over AoS arrays so that host callers (and the CPU test suite)
 * get exactly the device arithmetic: the same mpb core, with each PTX
 * carry-chain instruction emulated by an explicit carry flag.
 *
 * Exported (extern "C", AoS arrays of cu_freal<prec> / cu_fcomplex<prec>):
 *   mpbh_binop(prec, op, n, a, b, r)     op 0 mul, 1 add, 2 sub
 *   mpbh_fma(prec, n, a, b, c, r)
 *   mpbh_cbinop(prec, op, n, a, b, r)    op 0 cmul, 1 cadd, 2 csub
 *   mpbh_cfma(prec, n, a, b, c, r)       cu_cfma
 *   mpbh_div(prec, n, a, b, r)           cu_fdiv
 *   mpbh_sqrt(prec, n, a, r)             cu_sqrt
 *   mpbh_exp / mpbh_log(prec, n, a, r)   cu_exp / cu_log
 *   mpbh_fmath_r(fn, prec, n, a, b, r)   real elementary function fn (mpb.h
 *                                        MPB_FN_*; b only for pow / atan2)
 *   mpbh_fmath_c(fn, prec, n, a, b, r)   complex function fn (MPB_CFN_*;
 *                                        b only for the division)
 *   mpbh_div_ui(prec, n, a, u, r)        cu_div_ui
 *   mpbh_const(which, prec, r)           cu_pi (0) / cu_ln2 (1)
 *   mpbh_op_rp(op, p, n, a, b, c, r)     op at a runtime precision p (mpb.h
 *                                        MPB_RP_*), AoS of the storage PB
 *   mpbh_axpy_r / mpbh_axpy_c(prec, n, a, x, y, z)
 *   mpbh_from_double / mpbh_to_double(prec, n, ...)
 * Return 0, or -1 for an unsupported precision.
 */
#include <cstdint>
#include <initializer_list>

#include "mpc_cuda.cuh"
#include "mpb/rprec.cuh"

using cu_fp::cu_fcomplex;
using cu_fp::cu_freal;

namespace {

template <int PB>
void binop(int op, long n, const void *A, const void *B, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto b = (const cu_freal<PB> *)B;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    if (op == 0)
      r[i] = a[i] * b[i];
    else if (op == 1)
      r[i] = a[i] + b[i];
    else
      r[i] = a[i] - b[i];
  }
}
template <int PB>
void fma3(long n, const void *A, const void *B, const void *C, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto b = (const cu_freal<PB> *)B;
  auto c = (const cu_freal<PB> *)C;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_ffma<PB>(a[i], b[i], c[i]);
}
template <int PB>
void div2(long n, const void *A, const void *B, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto b = (const cu_freal<PB> *)B;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_fdiv<PB>(a[i], b[i]);
}
template <int PB>
void sqrt1(long n, const void *A, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_sqrt<PB>(a[i]);
}
template <int PB>
void exp1(long n, const void *A, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_exp<PB>(a[i]);
}
template <int PB>
void log1(long n, const void *A, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_log<PB>(a[i]);
}
template <int PB>
cu_freal<PB> fmath1(int fn, const cu_freal<PB> &a, const cu_freal<PB> &b) {
  using namespace cu_fp;
  switch (fn) {
    case 0: return cu_exp<PB>(a);
    case 1: return cu_log<PB>(a);
    case 2: return cu_expm1<PB>(a);
    case 3: return cu_log1p<PB>(a);
    case 4: return cu_sin<PB>(a);
    case 5: return cu_cos<PB>(a);
    case 6: return cu_tan<PB>(a);
    case 7: return cu_atan<PB>(a);
    case 8: return cu_sinh<PB>(a);
    case 9: return cu_cosh<PB>(a);
    case 10: return cu_atanh<PB>(a);
    case 11: return cu_asin<PB>(a);
    case 12: return cu_acos<PB>(a);
    case 13: return cu_cbrt<PB>(a);
    case 14: return cu_pow<PB>(a, b);
    default: return cu_atan2<PB>(a, b);
  }
}
template <int PB>
void fmath_r(int fn, long n, const void *A, const void *B, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto b = (const cu_freal<PB> *)B;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(dynamic, 16)
  for (long i = 0; i < n; i++) r[i] = fmath1<PB>(fn, a[i], b ? b[i] : a[i]);
}
template <int PB>
void fmath_c(int fn, long n, const void *A, const void *B, void *R) {
  auto a = (const cu_fcomplex<PB> *)A;
  auto b = (const cu_fcomplex<PB> *)B;
  auto r = (cu_fcomplex<PB> *)R;
#pragma omp parallel for schedule(dynamic, 16)
  for (long i = 0; i < n; i++) r[i] = fn == 8 ? cu_fp::cu_cdiv<PB>(a[i], b[i]) : cu_fp::detail::cfunc<PB>(fn, a[i]);
}
template <int PB>
void div_ui1(long n, const void *A, unsigned long long u, void *R) {
  auto a = (const cu_freal<PB> *)A;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_div_ui<PB>(a[i], u);
}
template <int PB>
void const1(int which, void *R) {
  *(cu_freal<PB> *)R = which == 0 ? cu_fp::cu_pi<PB>() : cu_fp::cu_ln2<PB>();
}
template <int PB>
void op_rp1(int op, int p, long n, const void *A, const void *B, const void *Cc, void *R) {
  typedef typename cu_fp::detail::core_of<PB>::type F;
  auto a = (const cu_freal<PB> *)A;
  auto b = (const cu_freal<PB> *)B;
  auto c = (const cu_freal<PB> *)Cc;
  auto r = (cu_freal<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    F x, y, z, o;
    cu_fp::detail::to_core<PB>(x, a[i]);
    cu_fp::detail::to_core<PB>(y, op == 5 ? a[i] : b[i]);
    cu_fp::detail::to_core<PB>(z, op == 3 ? c[i] : a[i]);
    mpb::op_rp(op, p, o, x, y, z);
    r[i] = cu_fp::detail::from_core<PB>(o);
  }
}
template <int PB>
void cfma3(long n, const void *A, const void *B, const void *C, void *R) {
  auto a = (const cu_fcomplex<PB> *)A;
  auto b = (const cu_fcomplex<PB> *)B;
  auto c = (const cu_fcomplex<PB> *)C;
  auto r = (cu_fcomplex<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) r[i] = cu_fp::cu_cfma<PB>(a[i], b[i], c[i]);
}
template <int PB>
void cbinop(int op, long n, const void *A, const void *B, void *R) {
  auto a = (const cu_fcomplex<PB> *)A;
  auto b = (const cu_fcomplex<PB> *)B;
  auto r = (cu_fcomplex<PB> *)R;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    if (op == 0)
      r[i] = a[i] * b[i];
    else if (op == 1)
      r[i] = a[i] + b[i];
    else
      r[i] = a[i] - b[i];
  }
}
template <int PB>
void axpy_r(long n, const void *A, const void *X, const void *Y, void *Z) {
  const cu_freal<PB> a = *(const cu_freal<PB> *)A;
  auto x = (const cu_freal<PB> *)X;
  auto y = (const cu_freal<PB> *)Y;
  auto z = (cu_freal<PB> *)Z;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) z[i] = a * x[i] + y[i];
}
template <int PB>
void axpy_c(long n, const void *A, const void *X, const void *Y, void *Z) {
  const cu_fcomplex<PB> a = *(const cu_fcomplex<PB> *)A;
  auto x = (const cu_fcomplex<PB> *)X;
  auto y = (const cu_fcomplex<PB> *)Y;
  auto z = (cu_fcomplex<PB> *)Z;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) z[i] = a * x[i] + y[i];
}
template <int PB>
void from_double(long n, const double *d, void *R) {
  auto r = (cu_freal<PB> *)R;
  for (long i = 0; i < n; i++) r[i] = cu_freal<PB>(d[i]);
}
template <int PB>
void to_double(long n, const void *X, double *d) {
  auto x = (const cu_freal<PB> *)X;
  for (long i = 0; i < n; i++) d[i] = (double)x[i];
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

#define MPBH_DISPATCH(P, CALL)                 \
  switch (P) {                                 \
    case 32: { constexpr int PB = 32; CALL; } return 0;     \
    case 64: { constexpr int PB = 64; CALL; } return 0;     \
    case 96: { constexpr int PB = 96; CALL; } return 0;     \
    case 128: { constexpr int PB = 128; CALL; } return 0;   \
    case 160: { constexpr int PB = 160; CALL; } return 0;   \
    case 256: { constexpr int PB = 256; CALL; } return 0;   \
    case 288: { constexpr int PB = 288; CALL; } return 0;   \
    case 512: { constexpr int PB = 512; CALL; } return 0;   \
    case 1024: { constexpr int PB = 1024; CALL; } return 0; \
    case 1056: { constexpr int PB = 1056; CALL; } return 0; \
    case 2048: { constexpr int PB = 2048; CALL; } return 0; \
    default: return -1;                        \
  }

}  // namespace

extern "C" {
int mpbh_binop(int prec, int op, long n, const void *a, const void *b, void *r) {
  MPBH_DISPATCH(prec, binop<PB>(op, n, a, b, r))
}
int mpbh_fma(int prec, long n, const void *a, const void *b, const void *c, void *r) {
  MPBH_DISPATCH(prec, fma3<PB>(n, a, b, c, r))
}
int mpbh_cbinop(int prec, int op, long n, const void *a, const void *b, void *r) {
  MPBH_DISPATCH(prec, cbinop<PB>(op, n, a, b, r))
}
int mpbh_div(int prec, long n, const void *a, const void *b, void *r) {
  MPBH_DISPATCH(prec, div2<PB>(n, a, b, r))
}
int mpbh_sqrt(int prec, long n, const void *a, void *r) {
  MPBH_DISPATCH(prec, sqrt1<PB>(n, a, r))
}
int mpbh_exp(int prec, long n, const void *a, void *r) { MPBH_DISPATCH(prec, exp1<PB>(n, a, r)) }
int mpbh_log(int prec, long n, const void *a, void *r) { MPBH_DISPATCH(prec, log1<PB>(n, a, r)) }
int mpbh_fmath_r(int fn, int prec, long n, const void *a, const void *b, void *r) {
  if (fn < 0 || fn > 15 || ((fn == 14 || fn == 15) && !b)) return -2;
  MPBH_DISPATCH(prec, fmath_r<PB>(fn, n, a, b, r))
}
int mpbh_fmath_c(int fn, int prec, long n, const void *a, const void *b, void *r) {
  if (fn < 0 || fn > 8 || (fn == 8 && !b)) return -2;
  MPBH_DISPATCH(prec, fmath_c<PB>(fn, n, a, b, r))
}
int mpbh_div_ui(int prec, long n, const void *a, unsigned long long u, void *r) {
  MPBH_DISPATCH(prec, div_ui1<PB>(n, a, u, r))
}
int mpbh_const(int which, int prec, void *r) { MPBH_DISPATCH(prec, const1<PB>(which, r)) }
int mpbh_op_rp(int op, int p, long n, const void *a, const void *b, const void *c, void *r) {
  if (op < 0 || op > 5 || p < 1) return -2;
  int pb = 0;
  for (int q : {64, 128, 256, 512, 1024, 2048})
    if (!pb && q >= p + 2) pb = q;
  if (!pb) return -1;
  MPBH_DISPATCH(pb, op_rp1<PB>(op, p, n, a, b, c, r))
}
int mpbh_cfma(int prec, long n, const void *a, const void *b, const void *c, void *r) {
  MPBH_DISPATCH(prec, cfma3<PB>(n, a, b, c, r))
}
int mpbh_axpy_r(int prec, long n, const void *a, const void *x, const void *y, void *z) {
  MPBH_DISPATCH(prec, axpy_r<PB>(n, a, x, y, z))
}
int mpbh_axpy_c(int prec, long n, const void *a, const void *x, const void *y, void *z) {
  MPBH_DISPATCH(prec, axpy_c<PB>(n, a, x, y, z))
}
int mpbh_from_double(int prec, long n, const double *d, void *r) {
  MPBH_DISPATCH(prec, from_double<PB>(n, d, r))
}
int mpbh_to_double(int prec, long n, const void *x, double *d) {
  MPBH_DISPATCH(prec, to_double<PB>(n, x, d))
}
int mpbh_util(int op, int P, long n, const void *A, const void *B, long *iv, void *R) {
  if (op < 0 || op > 3) return -2;
  MPBH_DISPATCH(P, util1<PB>(op, n, A, B, iv, R))
}
int mpbh_finalize(int P, long n, const unsigned long long *D, const long *q, void *R) {
  MPBH_DISPATCH(P, finalize1<PB>(n, D, q, R))
}
int mpbh_terms(int P, long n, const void *A, const void *B, const void *Cc, const void *Dd, long *hdr,
                 unsigned long long *M, void *R) {
  MPBH_DISPATCH(P, terms1<PB>(n, A, B, Cc, Dd, hdr, M, R))
}
/* cu_convert<to, from> for to, from in {32, 96, 160, 256, 288, 1056} */
int mpbh_convert(int to, int from, long n, const void *X, void *R) {
  UTIL_SMALL_DISPATCH(to, return convert_to<PB>(from, n, X, R))
  return -1;
}
}
