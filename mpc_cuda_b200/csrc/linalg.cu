/* linalg.cu -- plain GEMV / GEMM: every product and every accumulation is
 * rounded (RNDN), k runs sequentially from 0, acc starts at +0: the order of
 * the reference kernels (tools/linalg_fast.cu:37-68, complex
 * demos/matmul_mpc.cu:39-57), which the MPFR/MPC oracle reproduces.
 *
 * GEMM: thread per output C[i, j].  A warp owns one row i and 32 consecutive
 * columns, i.e. one tile of each B row: B loads are whole-tile coalesced
 * 128-bit loads, A[i, k] is the same address for the warp (a broadcast), and
 * the W warps of a block (4, 8 or 16 rows, mpb_set_gemm_warps) share the B
 * tile in L1.  The work per output is ~2N^2 IMADs per k, so this kernel is
 * bound by the integer pipe, not memory; W sets how many blocks a small C
 * spreads over the SMs and, through __launch_bounds__, the register budget of
 * wide operands (measured: W = 4 is 1.3x faster than 8 on a 128 x 128 C at
 * 512 and 2048 bits, W = 16 1.25x faster on 256 x 256 at 1024 bits).
 *
 * GEMV: thread per row (the accumulation order is sequential in k per row).
 */
#include <initializer_list>

#include "common.cuh"
#include "coop_rows.cuh"

namespace mpb {

constexpr int kGemvBlock = 128;

/* W warps (rows of C) per block: mpb_set_gemm_warps */
template <int N, int W>
__global__ void __launch_bounds__(W * 32) k_gemm_r(size_t m, size_t n, size_t K, const uint8_t *A,
                                                            size_t lda, const uint8_t *B, size_t ldb, uint8_t *C,
                                                            size_t ldc) {
  const size_t i = (size_t)blockIdx.y * W + (threadIdx.x >> 5);
  const size_t j = (size_t)blockIdx.x * 32u + (threadIdx.x & 31u);
  if (i >= m) return; /* warp-uniform */
  fval<N> acc;
  set_zero(acc);
  const size_t arow = i * lda;
  for (size_t k = 0; k < K; ++k) {
    fval<N> a, b, t;
    load_elem<N>(a, A, arow + k);
    load_elem<N>(b, B, k * ldb + j);
    mul<N>(t, b, a);
    add<N, true>(acc, acc, t);
  }
  if (j < n) store_elem<N>(C, i * ldc + j, acc);
}

template <int N, int W>
__global__ void __launch_bounds__(W * 32) k_gemm_c(size_t m, size_t n, size_t K, const uint8_t *A,
                                                            size_t lda, const uint8_t *B, size_t ldb, uint8_t *C,
                                                            size_t ldc) {
  const size_t i = (size_t)blockIdx.y * W + (threadIdx.x >> 5);
  const size_t j = (size_t)blockIdx.x * 32u + (threadIdx.x & 31u);
  if (i >= m) return;
  fval<N> cr, ci;
  set_zero(cr);
  set_zero(ci);
  const size_t arow = i * lda;
  for (size_t k = 0; k < K; ++k) {
    fval<N> ar, ai, br, bi, tr, ti;
    load_celem<N>(ar, ai, A, arow + k);
    load_celem<N>(br, bi, B, k * ldb + j);
    cmul<N, true>(tr, ti, br, bi, ar, ai);
    add<N, true>(cr, cr, tr);
    add<N, true>(ci, ci, ti);
  }
  if (j < n) store_celem<N>(C, i * ldc + j, cr, ci);
}

template <int N>
__global__ void __launch_bounds__(kGemvBlock) k_gemv_r(size_t m, size_t n, const uint8_t *A, size_t lda,
                                                       const uint8_t *x, const uint8_t *y, uint8_t *yo) {
  const size_t mp = tiles_for(m) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < mp; i += (size_t)gridDim.x * blockDim.x) {
    const size_t ir = i < m ? i : m - 1; /* padding lanes recompute the last row */
    fval<N> acc, yv;
    set_zero(acc);
    for (size_t k = 0; k < n; ++k) {
      fval<N> a, xv, t;
      load_elem<N>(a, A, ir * lda + k);
      load_elem<N>(xv, x, k);
      mul<N>(t, a, xv);
      add<N, true>(acc, acc, t);
    }
    load_elem<N>(yv, y, ir);
    add<N, true>(acc, acc, yv);
    if (i < m) store_elem<N>(yo, i, acc);
  }
}

/* GEMV with a group of G lanes per row (the warp-cooperative form for wide
 * operands): the warps of the grid stride over groups of 32/G rows */
template <int L, int G>
__global__ void __launch_bounds__(kGemvBlock) k_gemv_r_coop(size_t m, size_t n, const uint8_t *A, size_t lda,
                                                            const uint8_t *x, const uint8_t *y, uint8_t *yo) {
  constexpr int N = G * L, RPW = 32 / G, SMW = coop_row_smem<N>::words;
  __shared__ uint32_t sm_all[(kGemvBlock / 32) * RPW * SMW];
  const uint32_t warp = threadIdx.x >> 5, gw = (threadIdx.x & 31u) / G;
  uint32_t *sm = sm_all + (warp * RPW + gw) * SMW;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  const size_t rgroups = (m + RPW - 1) / RPW;
  for (size_t rg = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; rg < rgroups; rg += nw) {
    const size_t i = rg * RPW + gw;
    const size_t ir = i < m ? i : m - 1; /* lanes past the last row recompute it */
    coop::cv<L> acc;
    coop_gemv_row<L, G>(acc, A, ir * lda, n, x, y, ir, sm);
    if (i < m) coop::store<L, G>(yo, i, acc);
  }
}

template <int N>
__global__ void __launch_bounds__(kGemvBlock) k_gemv_c(size_t m, size_t n, const uint8_t *A, size_t lda,
                                                       const uint8_t *x, const uint8_t *y, uint8_t *yo) {
  const size_t mp = tiles_for(m) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < mp; i += (size_t)gridDim.x * blockDim.x) {
    const size_t ir = i < m ? i : m - 1;
    fval<N> cr, ci, yr, yi;
    set_zero(cr);
    set_zero(ci);
    for (size_t k = 0; k < n; ++k) {
      fval<N> ar, ai, xr, xi, tr, ti;
      load_celem<N>(ar, ai, A, ir * lda + k);
      load_celem<N>(xr, xi, x, k);
      cmul<N, true>(tr, ti, ar, ai, xr, xi);
      add<N, true>(cr, cr, tr);
      add<N, true>(ci, ci, ti);
    }
    load_celem<N>(yr, yi, y, ir);
    add<N, true>(cr, cr, yr);
    add<N, true>(ci, ci, yi);
    if (i < m) store_celem<N>(yo, i, cr, ci);
  }
}

/* argument checks shared by the matrix entry points; returns 1 for a no-op */
static int mat_args(int prec, size_t rows, size_t cols, size_t ld) {
  if (!prec_ok(prec)) return MPB_ERR_PREC;
  if (rows > kMaxElems || cols > kMaxElems || ld > kMaxElems) return MPB_ERR_SIZE;
  if (rows == 0 || cols == 0) return 1;
  if (ld % 32u != 0 || ld < cols) return MPB_ERR_LD;
  if (rows > kMaxElems / ld) return MPB_ERR_SIZE;
  return MPB_OK;
}
static int bufs_ok(std::initializer_list<const void *> bufs) {
  for (const void *p : bufs) {
    const int rc = check_buf(p);
    if (rc != MPB_OK) return rc;
  }
  return MPB_OK;
}

} /* namespace mpb */

using namespace mpb;

/* GEMV blocks: one warp each when the rows give fewer than four warps per SM
 * (a tall matrix of wide operands is few warps: 4096 rows of one thread each
 * are 32 blocks of 128 on 148 SMs), four warps otherwise */
static int gemv_block(size_t warps) { return warps < 4u * (size_t)sm_count() ? 32 : kGemvBlock; }

template <int L, int G>
static void launch_gemv_coop_lg(size_t m, size_t n, const uint8_t *A, size_t lda, const uint8_t *x, const uint8_t *y,
                                uint8_t *yo, cudaStream_t st) {
  const size_t warps = (m + 32 / G - 1) / (32 / G);
  const int b = gemv_block(warps);
  const int g = grid_for(k_gemv_r_coop<L, G>, b, warps * 32u);
  k_gemv_r_coop<L, G><<<g, b, 0, st>>>(m, n, A, lda, x, y, yo);
}
/* the cooperative GEMV at N limbs with `lanes` lanes per row (1024 bits: 4 or
 * 8 lanes, 2048 bits: 8 or 16; mpb_set_split validates) */
template <int N>
static void launch_gemv_coop(int lanes, size_t m, size_t n, const uint8_t *A, size_t lda, const uint8_t *x,
                             const uint8_t *y, uint8_t *yo, cudaStream_t st) {
  if constexpr (N == 32) {
    if (lanes == 4)
      launch_gemv_coop_lg<8, 4>(m, n, A, lda, x, y, yo, st);
    else
      launch_gemv_coop_lg<4, 8>(m, n, A, lda, x, y, yo, st);
  } else if constexpr (N == 64) {
    if (lanes == 8)
      launch_gemv_coop_lg<8, 8>(m, n, A, lda, x, y, yo, st);
    else
      launch_gemv_coop_lg<4, 16>(m, n, A, lda, x, y, yo, st);
  }
}

template <bool CPLX>
static int gemv_entry(int prec, size_t m, size_t n, const void *A, size_t lda, const void *x, const void *y,
                      void *yo, void *stream) {
  if (!prec_ok(prec)) return MPB_ERR_PREC;
  if (m == 0) return MPB_OK;
  if (n == 0) { /* empty dot: y_out = +0 + y = y */
    if (!y || !yo) return MPB_ERR_NULL;
    int rc = bufs_ok({y, yo});
    if (rc != MPB_OK) return rc;
    const size_t bytes = (CPLX ? 2u : 1u) * tiles_for(m) * tile_bytes_for(prec / 32);
    if (y != yo && cudaMemcpyAsync(yo, y, bytes, cudaMemcpyDeviceToDevice, as_stream(stream)) != cudaSuccess)
      return MPB_ERR_CUDA;
    return MPB_OK;
  }
  int rc = mat_args(prec, m, n, lda);
  if (rc != MPB_OK) return rc > 0 ? MPB_OK : rc;
  rc = bufs_ok({A, x, y, yo});
  if (rc != MPB_OK) return rc;
  MPB_DISPATCH_PREC(prec, {
    const int b = gemv_block(tiles_for(m));
    if (CPLX) {
      const int g = grid_for(k_gemv_c<N>, b, tiles_for(m) * 32u);
      k_gemv_c<N><<<g, b, 0, as_stream(stream)>>>(m, n, (const uint8_t *)A, lda, (const uint8_t *)x,
                                                   (const uint8_t *)y, (uint8_t *)yo);
    } else if (N >= 32 && split_lanes(MPB_SPLIT_GEMV_R, prec) > 1) {
      launch_gemv_coop<N>(split_lanes(MPB_SPLIT_GEMV_R, prec), m, n, (const uint8_t *)A, lda, (const uint8_t *)x,
                          (const uint8_t *)y, (uint8_t *)yo, as_stream(stream));
    } else {
      const int g = grid_for(k_gemv_r<N>, b, tiles_for(m) * 32u);
      k_gemv_r<N><<<g, b, 0, as_stream(stream)>>>(m, n, (const uint8_t *)A, lda, (const uint8_t *)x,
                                                   (const uint8_t *)y, (uint8_t *)yo);
    }
  });
  return launch_status();
}

template <int N, int W, bool CPLX>
static void launch_gemm(size_t m, size_t n, size_t k, const void *A, size_t lda, const void *B, size_t ldb, void *C,
                        size_t ldc, cudaStream_t st) {
  const dim3 grid((unsigned)((n + 31) / 32), (unsigned)((m + W - 1) / W));
  if (CPLX)
    k_gemm_c<N, W><<<grid, W * 32, 0, st>>>(m, n, k, (const uint8_t *)A, lda, (const uint8_t *)B, ldb,
                                            (uint8_t *)C, ldc);
  else
    k_gemm_r<N, W><<<grid, W * 32, 0, st>>>(m, n, k, (const uint8_t *)A, lda, (const uint8_t *)B, ldb,
                                            (uint8_t *)C, ldc);
}

template <bool CPLX>
static int gemm_entry(int prec, size_t m, size_t n, size_t k, const void *A, size_t lda, const void *B, size_t ldb,
                      void *C, size_t ldc, void *stream) {
  int rc = mat_args(prec, m, n, ldc);
  if (rc != MPB_OK) return rc > 0 ? MPB_OK : rc;
  if (k > 0) {
    rc = mat_args(prec, m, k, lda);
    if (rc != MPB_OK) return rc;
    rc = mat_args(prec, k, n, ldb);
    if (rc != MPB_OK) return rc;
    rc = bufs_ok({A, B});
    if (rc != MPB_OK) return rc;
  }
  rc = bufs_ok({C});
  if (rc != MPB_OK) return rc;
  const int w = gemm_warps(CPLX ? 1 : 0, prec);
  if ((m + w - 1) / w > 65535u) return MPB_ERR_SIZE;
  MPB_DISPATCH_PREC(prec, {
    if (w == 4)
      launch_gemm<N, 4, CPLX>(m, n, k, A, lda, B, ldb, C, ldc, as_stream(stream));
    else if (w == 16)
      launch_gemm<N, 16, CPLX>(m, n, k, A, lda, B, ldb, C, ldc, as_stream(stream));
    else
      launch_gemm<N, 8, CPLX>(m, n, k, A, lda, B, ldb, C, ldc, as_stream(stream));
  });
  return launch_status();
}

extern "C" int mpb_gemv_r(int prec, size_t m, size_t n, const void *A, size_t lda, const void *x, const void *y,
                          void *y_out, void *stream) {
  return gemv_entry<false>(prec, m, n, A, lda, x, y, y_out, stream);
}
extern "C" int mpb_gemv_c(int prec, size_t m, size_t n, const void *A, size_t lda, const void *x, const void *y,
                          void *y_out, void *stream) {
  return gemv_entry<true>(prec, m, n, A, lda, x, y, y_out, stream);
}
extern "C" int mpb_gemm_r(int prec, size_t m, size_t n, size_t k, const void *A, size_t lda, const void *B,
                          size_t ldb, void *C, size_t ldc, void *stream) {
  return gemm_entry<false>(prec, m, n, k, A, lda, B, ldb, C, ldc, stream);
}
extern "C" int mpb_gemm_c(int prec, size_t m, size_t n, size_t k, const void *A, size_t lda, const void *B,
                          size_t ldb, void *C, size_t ldc, void *stream) {
  return gemm_entry<true>(prec, m, n, k, A, lda, B, ldb, C, ldc, stream);
}
