/* user_kernels.cu -- kernels written against the cu_fp surface the way the
 * reference's callers write them, for the drop-in tests and the bench.
 *
 * The callers this mirrors: the AXPY of demos/bench_3way.cu:44-59 (FP64 in and
 * out, operators on cu_freal / cu_fcomplex), the sequential-k matmul of
 * tools/linalg_fast.cu:54-68 (acc = cu_fadd(acc, cu_fmul(a, b)) per k), the
 * complex AXPY of tools/axpy_fast_complex.cu:32-40 and the element-wise
 * operator tests of tools/test_freal.cu:42-48, here over AoS arrays of
 * cu_freal<PB> / cu_fcomplex<PB> in device memory, plus cu_exp and cu_fdiv from
 * the elementary-function header.
 *
 * The same sources build against this repository's include/ (the drop-in,
 * tests/dropin/libuser_kernels.so, symbols uk_*) and, in the oracle recipe,
 * against the reference's own include/ (oracle/_ref/libref_user_kernels.so,
 * symbols refuk_*), so both run the identical kernels on the same GPU.
 *
 * Every entry point: (prec, sizes, device pointers, grid, block, stream) ->
 * 0, -1 for a precision that is not instantiated, -3 for a launch error;
 * grid <= 0 picks 4 blocks per SM.
 */
#include "user_kernels.cuh"

#ifndef UK_PREFIX
#define UK_PREFIX uk_
#endif
#define UK_CAT2(a, b) a##b
#define UK_CAT(a, b) UK_CAT2(a, b)
#define UK(name) UK_CAT(UK_PREFIX, name)

using namespace uk;

#define UK_DECL(PB) UK_LAUNCHERS(extern, PB)
#define UK_DECL_FN(PB) UK_FN_LAUNCHERS(extern, PB)
#define UK_DECL_REAL(PB) UK_REAL_LAUNCHERS(extern, PB)
namespace uk {
UK_FOR_EACH_PB(UK_DECL)
UK_FOR_EACH_FN_PB(UK_DECL_FN)
UK_FOR_EACH_REAL_ONLY_PB(UK_DECL_REAL)
}  // namespace uk

namespace {

int grid_of(int grid) {
  if (grid > 0) return grid;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return 4 * sms;
}
int launched() { return cudaGetLastError() == cudaSuccess ? 0 : -3; }

#define UK_CASE(PB_, CALL) \
  case PB_: {              \
    constexpr int PB = PB_; \
    CALL;                  \
  } break;
#define UK_DISPATCH(P, CALL)                                                              \
  switch (P) {                                                                           \
    UK_CASE(64, CALL) UK_CASE(96, CALL) UK_CASE(128, CALL) UK_CASE(160, CALL)            \
    UK_CASE(256, CALL) UK_CASE(288, CALL) UK_CASE(512, CALL) UK_CASE(1024, CALL)         \
    UK_CASE(1056, CALL) UK_CASE(2048, CALL)                                              \
    default: return -1;                                                                  \
  }                                                                                      \
  return launched();
#define UK_DISPATCH_REAL(P, CALL)                                                         \
  switch (P) {                                                                           \
    UK_CASE(64, CALL) UK_CASE(96, CALL) UK_CASE(128, CALL) UK_CASE(160, CALL)            \
    UK_CASE(256, CALL) UK_CASE(288, CALL) UK_CASE(512, CALL) UK_CASE(1024, CALL)         \
    UK_CASE(1056, CALL) UK_CASE(2048, CALL) UK_CASE(4096, CALL)                          \
    default: return -1;                                                                  \
  }                                                                                      \
  return launched();
#define UK_DISPATCH_FN(P, CALL)                                                           \
  switch (P) {                                                                           \
    UK_CASE(64, CALL) UK_CASE(96, CALL) UK_CASE(128, CALL) UK_CASE(160, CALL)            \
    UK_CASE(256, CALL) UK_CASE(288, CALL) UK_CASE(512, CALL) UK_CASE(1024, CALL)         \
    UK_CASE(1056, CALL)                                                                  \
    default: return -1;                                                                  \
  }                                                                                      \
  return launched();

}  // namespace

#define UK_LAUNCH grid_of(grid), block, (cudaStream_t)stream

extern "C" {
int UK(axpy_r)(int prec, long n, const void *a, const void *x, const void *y, void *z, int grid, int block,
               void *stream) {
  UK_DISPATCH_REAL(prec, (run_axpy_r<PB>(UK_LAUNCH, n, a, x, y, z)))
}
int UK(axpy_c)(int prec, long n, const void *a, const void *x, const void *y, void *z, int grid, int block,
               void *stream) {
  UK_DISPATCH(prec, (run_axpy_c<PB>(UK_LAUNCH, n, a, x, y, z)))
}
int UK(axpy_d)(int prec, long n, double a, const double *X, const double *Y, double *O, int grid, int block,
               void *stream) {
  UK_DISPATCH_REAL(prec, (run_axpy_d<PB>(UK_LAUNCH, n, a, X, Y, O)))
}
int UK(caxpy_d)(int prec, long n, double ar, double ai, const double *XR, const double *XI, const double *YR,
                const double *YI, double *OR, double *OI, int grid, int block, void *stream) {
  UK_DISPATCH(prec, (run_caxpy_d<PB>(UK_LAUNCH, n, ar, ai, XR, XI, YR, YI, OR, OI)))
}
int UK(matmul_r)(int prec, int m, int n, int k, const void *A, int lda, const void *B, int ldb, void *C, int ldc,
                 int grid, int block, void *stream) {
  UK_DISPATCH_REAL(prec, (run_matmul_r<PB>(UK_LAUNCH, m, n, k, A, lda, B, ldb, C, ldc)))
}
int UK(matmul_c)(int prec, int m, int n, int k, const void *A, int lda, const void *B, int ldb, void *C, int ldc,
                 int grid, int block, void *stream) {
  UK_DISPATCH(prec, (run_matmul_c<PB>(UK_LAUNCH, m, n, k, A, lda, B, ldb, C, ldc)))
}
int UK(exp)(int prec, long n, const void *x, void *r, int grid, int block, void *stream) {
  UK_DISPATCH_FN(prec, (run_exp<PB>(UK_LAUNCH, n, x, r)))
}
int UK(div)(int prec, long n, const void *x, const void *y, void *r, int grid, int block, void *stream) {
  UK_DISPATCH_FN(prec, (run_div<PB>(UK_LAUNCH, n, x, y, r)))
}
}
