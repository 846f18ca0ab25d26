/* rprec.cu -- element-wise arithmetic at a runtime precision (mpb/rprec.cuh):
 * round to odd at the storage format's PB bits, then to nearest at p bits. */
#include <initializer_list>

#include "common.cuh"
#include "mpb/rprec.cuh"

namespace mpb {

constexpr int kBlock = 128;

template <int N>
__global__ void __launch_bounds__(kBlock) k_op_rp(int op, int p, size_t n, const uint8_t *a, const uint8_t *b,
                                                  const uint8_t *c, uint8_t *r) {
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> x, y, z, o;
    load_elem<N, kStream>(x, a, i);
    if (op != MPB_RP_SQRT) load_elem<N, kStream>(y, b, i);
    if (op == MPB_RP_FMA) load_elem<N, kStream>(z, c, i);
    op_rp<N>(op, p, o, x, y, z);
    if (i < n) store_elem<N, kStream>(r, i, o);
  }
}

/* one operation at p bits: round to odd at the storage PB, then to nearest at p */
template <int N>
__device__ __forceinline__ void mul_p(fval<N> &r, const fval<N> &a, const fval<N> &b, int p) {
  mul<N, 1>(r, a, b);
  round_to_bits<N>(r, p);
}
template <int N>
__device__ __forceinline__ void add_p(fval<N> &r, const fval<N> &a, const fval<N> &b, int p) {
  add<N, false, 1>(r, a, b);
  round_to_bits<N>(r, p);
}

/* the linear-algebra kernels of elementwise.cu / linalg.cu with every
 * operation rounded at p bits: the same order (AXPY round(round(a x) + y);
 * GEMV acc = +0, acc = round(acc + round(A[i,k] x[k])) in k order, then + y;
 * GEMM the sequential-k dot), so each result equals MPFR's with p-bit
 * destinations */
template <int N>
__global__ void __launch_bounds__(kBlock) k_axpy_rp(int p, size_t n, const uint8_t *a, const uint8_t *x,
                                                    const uint8_t *y, uint8_t *z) {
  fval<N> av;
  load_elem<N>(av, a, 0);
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> xv, yv, t, r;
    load_elem<N, kStream>(xv, x, i);
    load_elem<N, kStream>(yv, y, i);
    mul_p<N>(t, av, xv, p);
    add_p<N>(r, t, yv, p);
    if (i < n) store_elem<N, kStream>(z, i, r);
  }
}
template <int N>
__global__ void __launch_bounds__(kBlock) k_gemv_rp(int p, size_t m, size_t n, const uint8_t *A, size_t lda,
                                                    const uint8_t *x, const uint8_t *y, uint8_t *yo) {
  const size_t mp = tiles_for(m) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < mp; i += (size_t)gridDim.x * blockDim.x) {
    const size_t ir = i < m ? i : m - 1;
    fval<N> acc, yv;
    set_zero(acc);
    for (size_t k = 0; k < n; ++k) {
      fval<N> av, xv, t;
      load_elem<N>(av, A, ir * lda + k);
      load_elem<N>(xv, x, k);
      mul_p<N>(t, av, xv, p);
      add_p<N>(acc, acc, t, p);
    }
    load_elem<N>(yv, y, ir);
    add_p<N>(acc, acc, yv, p);
    if (i < m) store_elem<N>(yo, i, acc);
  }
}
constexpr int kGemmRpWarps = 8;
template <int N>
__global__ void __launch_bounds__(kGemmRpWarps * 32) k_gemm_rp(int p, size_t m, size_t n, size_t K, const uint8_t *A,
                                                               size_t lda, const uint8_t *B, size_t ldb, uint8_t *C,
                                                               size_t ldc) {
  const size_t i = (size_t)blockIdx.y * kGemmRpWarps + (threadIdx.x >> 5);
  const size_t j = (size_t)blockIdx.x * 32u + (threadIdx.x & 31u);
  if (i >= m) return; /* warp-uniform */
  fval<N> acc;
  set_zero(acc);
  for (size_t k = 0; k < K; ++k) {
    fval<N> av, bv, t;
    load_elem<N>(av, A, i * lda + k);
    load_elem<N>(bv, B, k * ldb + j);
    mul_p<N>(t, av, bv, p);
    add_p<N>(acc, acc, t, p);
  }
  if (j < n) store_elem<N>(C, i * ldc + j, acc);
}
/* r rounded to nearest at p bits, in place */
template <int N>
__global__ void __launch_bounds__(kBlock) k_round_p(int p, size_t n, uint8_t *r) {
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> v;
    load_elem<N>(v, r, i);
    round_to_bits<N>(v, p);
    if (i < n) store_elem<N>(r, i, v);
  }
}

} /* namespace mpb */

using namespace mpb;

extern "C" int mpb_storage_prec(int prec) {
  if (prec < 1) return MPB_ERR_PREC;
  for (int pb : {64, 128, 256, 512, 1024, 2048})
    if (pb >= prec + 2) return pb;
  return MPB_ERR_PREC;
}

extern "C" int mpb_op_rp(int op, int prec, size_t n, const void *a, const void *b, const void *c, void *r,
                         void *stream) {
  if (op < MPB_RP_MUL || op > MPB_RP_SQRT) return MPB_ERR_ARG;
  const int pb = mpb_storage_prec(prec);
  if (pb < 0) return MPB_ERR_PREC;
  if (n > kMaxElems) return MPB_ERR_SIZE;
  if (n == 0) return MPB_OK;
  for (const void *q : {a, op == MPB_RP_SQRT ? a : b, op == MPB_RP_FMA ? c : a, (const void *)r}) {
    const int rc = check_buf(q);
    if (rc != MPB_OK) return rc;
  }
  MPB_DISPATCH_PREC(pb, {
    const int g = grid_for(k_op_rp<N>, kBlock, tiles_for(n) * 32u);
    k_op_rp<N><<<g, kBlock, 0, as_stream(stream)>>>(op, prec, n, (const uint8_t *)a, (const uint8_t *)b,
                                                   (const uint8_t *)c, (uint8_t *)r);
  });
  return launch_status();
}

/* ---- linear algebra and elementary functions at a runtime precision ---- */
static int rp_buffers(std::initializer_list<const void *> bufs) {
  for (const void *q : bufs) {
    const int rc = check_buf(q);
    if (rc != MPB_OK) return rc;
  }
  return MPB_OK;
}

extern "C" int mpb_axpy_r_rp(int prec, size_t n, const void *a, const void *x, const void *y, void *z,
                             void *stream) {
  const int pb = mpb_storage_prec(prec);
  if (pb < 0) return MPB_ERR_PREC;
  if (n > kMaxElems) return MPB_ERR_SIZE;
  if (n == 0) return MPB_OK;
  int rc = rp_buffers({a, x, y, z});
  if (rc != MPB_OK) return rc;
  MPB_DISPATCH_PREC(pb, {
    const int g = grid_for(k_axpy_rp<N>, kBlock, tiles_for(n) * 32u);
    k_axpy_rp<N><<<g, kBlock, 0, as_stream(stream)>>>(prec, n, (const uint8_t *)a, (const uint8_t *)x,
                                                     (const uint8_t *)y, (uint8_t *)z);
  });
  return launch_status();
}

extern "C" int mpb_gemv_r_rp(int prec, size_t m, size_t n, const void *A, size_t lda, const void *x, const void *y,
                             void *y_out, void *stream) {
  const int pb = mpb_storage_prec(prec);
  if (pb < 0) return MPB_ERR_PREC;
  if (m > kMaxElems || n > kMaxElems || lda > kMaxElems) return MPB_ERR_SIZE;
  if (m == 0) return MPB_OK;
  if (n > 0 && (lda % 32 != 0 || lda < n)) return MPB_ERR_LD;
  if (n > 0 && m > kMaxElems / lda) return MPB_ERR_SIZE;
  int rc = rp_buffers({y, y_out});
  if (rc == MPB_OK && n > 0) rc = rp_buffers({A, x});
  if (rc != MPB_OK) return rc;
  MPB_DISPATCH_PREC(pb, {
    const int g = grid_for(k_gemv_rp<N>, kBlock, tiles_for(m) * 32u);
    k_gemv_rp<N><<<g, kBlock, 0, as_stream(stream)>>>(prec, m, n, (const uint8_t *)A, lda, (const uint8_t *)x,
                                                     (const uint8_t *)y, (uint8_t *)y_out);
  });
  return launch_status();
}

extern "C" int mpb_gemm_r_rp(int prec, size_t m, size_t n, size_t k, const void *A, size_t lda, const void *B,
                             size_t ldb, void *C, size_t ldc, void *stream) {
  const int pb = mpb_storage_prec(prec);
  if (pb < 0) return MPB_ERR_PREC;
  if (m > kMaxElems || n > kMaxElems || k > kMaxElems) return MPB_ERR_SIZE;
  if (m == 0 || n == 0) return MPB_OK;
  if (ldc % 32 != 0 || ldc < n || (k > 0 && (lda % 32 != 0 || lda < k || ldb % 32 != 0 || ldb < n)))
    return MPB_ERR_LD;
  if ((m + kGemmRpWarps - 1) / kGemmRpWarps > 65535u) return MPB_ERR_SIZE;
  int rc = rp_buffers({C});
  if (rc == MPB_OK && k > 0) rc = rp_buffers({A, B});
  if (rc != MPB_OK) return rc;
  const dim3 grid((unsigned)((n + 31) / 32), (unsigned)((m + kGemmRpWarps - 1) / kGemmRpWarps));
  MPB_DISPATCH_PREC(pb, {
    k_gemm_rp<N><<<grid, kGemmRpWarps * 32, 0, as_stream(stream)>>>(prec, m, n, k, (const uint8_t *)A, lda,
                                                                   (const uint8_t *)B, ldb, (uint8_t *)C, ldc);
  });
  return launch_status();
}

extern "C" int mpb_fmath_r_rp(int fn, int prec, size_t n, const void *a, const void *b, void *r, void *stream) {
  const int pb = mpb_storage_prec(prec);
  if (pb < 0) return MPB_ERR_PREC;
  int rc = mpb_fmath_r(fn, pb, n, a, b, r, stream);
  if (rc != MPB_OK || n == 0) return rc;
  MPB_DISPATCH_PREC(pb, {
    const int g = grid_for(k_round_p<N>, kBlock, tiles_for(n) * 32u);
    k_round_p<N><<<g, kBlock, 0, as_stream(stream)>>>(prec, n, (uint8_t *)r);
  });
  return launch_status();
}
