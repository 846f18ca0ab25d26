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
 *   mpbh_axpy_r / mpbh_axpy_c(prec, n, a, x, y, z)
 *   mpbh_from_double / mpbh_to_double(prec, n, ...)
 * Return 0, or -1 for an unsupported precision.
 */
#include <cstdint>

#include "mpc_cuda.cuh"

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
}
