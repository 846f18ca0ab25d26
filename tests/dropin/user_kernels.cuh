/* user_kernels.cuh -- the user kernels of user_kernels.cu and one launcher per
 * kernel and precision (run_*<PB>); each precision's launchers are
 * instantiated in their own translation unit (uk_pb.cu built with -DUK_PB=PB)
 * so the build runs them in parallel. */
#ifndef UK_USER_KERNELS_CUH
#define UK_USER_KERNELS_CUH
#include <cuda_runtime.h>

#include "mpc_cuda/cu_fcomplex.cuh"
#include "mpc_cuda/cu_fmath.cuh"

namespace uk {
using cu_fp::cu_fcomplex;
using cu_fp::cu_freal;

#define UK_LOOP(n) for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < (n); i += (long)gridDim.x * blockDim.x)

template <int PB>
__global__ void k_axpy_r(long n, const cu_freal<PB> *a, const cu_freal<PB> *x, const cu_freal<PB> *y,
                         cu_freal<PB> *z) {
  const cu_freal<PB> s = *a;
  UK_LOOP(n) z[i] = s * x[i] + y[i];
}
template <int PB>
__global__ void k_axpy_c(long n, const cu_fcomplex<PB> *a, const cu_fcomplex<PB> *x, const cu_fcomplex<PB> *y,
                         cu_fcomplex<PB> *z) {
  const cu_fcomplex<PB> s = *a;
  UK_LOOP(n) z[i] = s * x[i] + y[i];
}
/* the benchmark kernels of demos/bench_3way.cu:44-59: FP64 operands in, FP64 out */
template <int PB>
__global__ void k_axpy_d(long n, double a, const double *X, const double *Y, double *O) {
  UK_LOOP(n) {
    const cu_freal<PB> t = cu_freal<PB>(a) * cu_freal<PB>(X[i]);
    O[i] = (t + cu_freal<PB>(Y[i])).to_double();
  }
}
template <int PB>
__global__ void k_caxpy_d(long n, double ar, double ai, const double *XR, const double *XI, const double *YR,
                          const double *YI, double *OR, double *OI) {
  const cu_fcomplex<PB> a(ar, ai);
  UK_LOOP(n) {
    const cu_fcomplex<PB> t = a * cu_fcomplex<PB>(XR[i], XI[i]);
    const cu_fcomplex<PB> r = t + cu_fcomplex<PB>(YR[i], YI[i]);
    OR[i] = r.real_d();
    OI[i] = r.imag_d();
  }
}
/* C = A B, one thread per entry, sequential k with a rounding per operation */
template <int PB>
__global__ void k_matmul_r(int m, int n, int k, const cu_freal<PB> *A, int lda, const cu_freal<PB> *B, int ldb,
                           cu_freal<PB> *C, int ldc) {
  UK_LOOP((long)m * n) {
    const int r = (int)(i / n), c = (int)(i % n);
    cu_freal<PB> acc;
    acc.set_zero();
    for (int t = 0; t < k; t++) acc = cu_fp::cu_fadd<PB>(acc, cu_fp::cu_fmul<PB>(A[(long)r * lda + t], B[(long)t * ldb + c]));
    C[(long)r * ldc + c] = acc;
  }
}
template <int PB>
__global__ void k_matmul_c(int m, int n, int k, const cu_fcomplex<PB> *A, int lda, const cu_fcomplex<PB> *B,
                           int ldb, cu_fcomplex<PB> *C, int ldc) {
  UK_LOOP((long)m * n) {
    const int r = (int)(i / n), c = (int)(i % n);
    cu_fcomplex<PB> acc;
    acc.re.set_zero();
    acc.im.set_zero();
    for (int t = 0; t < k; t++) acc = acc + A[(long)r * lda + t] * B[(long)t * ldb + c];
    C[(long)r * ldc + c] = acc;
  }
}
template <int PB>
__global__ void k_exp(long n, const cu_freal<PB> *x, cu_freal<PB> *r) {
  UK_LOOP(n) r[i] = cu_fp::cu_exp<PB>(x[i]);
}
template <int PB>
__global__ void k_div(long n, const cu_freal<PB> *x, const cu_freal<PB> *y, cu_freal<PB> *r) {
  UK_LOOP(n) r[i] = cu_fp::cu_fdiv<PB>(x[i], y[i]);
}


template <int PB>
void run_axpy_r(int g, int b, cudaStream_t s, long n, const void *a, const void *x, const void *y, void *z) {
  k_axpy_r<PB><<<g, b, 0, s>>>(n, (const cu_freal<PB> *)a, (const cu_freal<PB> *)x, (const cu_freal<PB> *)y,
                               (cu_freal<PB> *)z);
}
template <int PB>
void run_axpy_c(int g, int b, cudaStream_t s, long n, const void *a, const void *x, const void *y, void *z) {
  k_axpy_c<PB><<<g, b, 0, s>>>(n, (const cu_fcomplex<PB> *)a, (const cu_fcomplex<PB> *)x,
                               (const cu_fcomplex<PB> *)y, (cu_fcomplex<PB> *)z);
}
template <int PB>
void run_axpy_d(int g, int b, cudaStream_t s, long n, double a, const double *X, const double *Y, double *O) {
  k_axpy_d<PB><<<g, b, 0, s>>>(n, a, X, Y, O);
}
template <int PB>
void run_caxpy_d(int g, int b, cudaStream_t s, long n, double ar, double ai, const double *XR, const double *XI,
                 const double *YR, const double *YI, double *OR, double *OI) {
  k_caxpy_d<PB><<<g, b, 0, s>>>(n, ar, ai, XR, XI, YR, YI, OR, OI);
}
template <int PB>
void run_matmul_r(int g, int b, cudaStream_t s, int m, int n, int k, const void *A, int lda, const void *B, int ldb,
                  void *C, int ldc) {
  k_matmul_r<PB><<<g, b, 0, s>>>(m, n, k, (const cu_freal<PB> *)A, lda, (const cu_freal<PB> *)B, ldb,
                                 (cu_freal<PB> *)C, ldc);
}
template <int PB>
void run_matmul_c(int g, int b, cudaStream_t s, int m, int n, int k, const void *A, int lda, const void *B, int ldb,
                  void *C, int ldc) {
  k_matmul_c<PB><<<g, b, 0, s>>>(m, n, k, (const cu_fcomplex<PB> *)A, lda, (const cu_fcomplex<PB> *)B, ldb,
                                 (cu_fcomplex<PB> *)C, ldc);
}
template <int PB>
void run_exp(int g, int b, cudaStream_t s, long n, const void *x, void *r) {
  k_exp<PB><<<g, b, 0, s>>>(n, (const cu_freal<PB> *)x, (cu_freal<PB> *)r);
}
template <int PB>
void run_div(int g, int b, cudaStream_t s, long n, const void *x, const void *y, void *r) {
  k_div<PB><<<g, b, 0, s>>>(n, (const cu_freal<PB> *)x, (const cu_freal<PB> *)y, (cu_freal<PB> *)r);
}

/* the launchers of one precision, declared (UK_EXTERN) or instantiated (UK_INST) */
/* the real kernels (every precision, 4096 bits included) */
#define UK_REAL_LAUNCHERS(KW, PB)                                                                              \
  KW template void run_axpy_r<PB>(int, int, cudaStream_t, long, const void *, const void *, const void *, void *); \
  KW template void run_axpy_d<PB>(int, int, cudaStream_t, long, double, const double *, const double *, double *); \
  KW template void run_matmul_r<PB>(int, int, cudaStream_t, int, int, int, const void *, int, const void *, int, \
                                    void *, int);
/* the complex kernels: up to 2048 bits (at 4096 their unrolled products take
 * many minutes to compile) */
#define UK_CPLX_LAUNCHERS(KW, PB)                                                                              \
  KW template void run_axpy_c<PB>(int, int, cudaStream_t, long, const void *, const void *, const void *, void *); \
  KW template void run_caxpy_d<PB>(int, int, cudaStream_t, long, double, double, const double *, const double *, \
                                   const double *, const double *, double *, double *);                       \
  KW template void run_matmul_c<PB>(int, int, cudaStream_t, int, int, int, const void *, int, const void *, int, \
                                    void *, int);
#define UK_LAUNCHERS(KW, PB) UK_REAL_LAUNCHERS(KW, PB) UK_CPLX_LAUNCHERS(KW, PB)
/* the elementary functions stop at 1056 bits: at 2048 the reference's
 * runtime-indexed guard-precision arrays take very long to compile */
#define UK_FN_LAUNCHERS(KW, PB)                                                   \
  KW template void run_exp<PB>(int, int, cudaStream_t, long, const void *, void *); \
  KW template void run_div<PB>(int, int, cudaStream_t, long, const void *, const void *, void *);

#define UK_FOR_EACH_PB(X) X(64) X(96) X(128) X(160) X(256) X(288) X(512) X(1024) X(1056) X(2048)
#define UK_FOR_EACH_REAL_ONLY_PB(X) X(4096)
#define UK_FOR_EACH_FN_PB(X) X(64) X(96) X(128) X(160) X(256) X(288) X(512) X(1024) X(1056)

}  // namespace uk
#endif
