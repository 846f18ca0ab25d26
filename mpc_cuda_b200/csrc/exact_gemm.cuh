/* exact_gemm.cuh -- internal: plan, slicing and rounding kernels of the
 * exact-accumulation GEMM, shared by the per-precision translation units
 * exact_gemm_pb*.cu.  The algorithm is described in exact_gemm.cu. */
#ifndef MPB_EXACT_GEMM_CUH
#define MPB_EXACT_GEMM_CUH

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "common.cuh"
#include "sm100.cuh"

namespace mpb {
namespace exact {

constexpr int BM = 128;             /* output rows per tile (UMMA M) */
constexpr int BN = 256;             /* output columns per tile (UMMA N) */
constexpr int BK = 128;             /* K bytes per pipeline stage (one 128B swizzle row) */
constexpr int STAGES = 4;
constexpr uint32_t A_STAGE = BM * BK; /* 16 KB */
constexpr uint32_t B_STAGE = BN * BK; /* 32 KB */
constexpr int kGemmThreads = 192;   /* warp 0 TMA, warp 1 MMA, warps 2-5 epilogue */
constexpr long kSafeTerms = 1L << 17; /* pairs * k < 2^17 keeps |D| < 2^31 */
constexpr int kMaxParts = 16;       /* keeps the rounding's int64 word sums exact */
/* Low-diagonal truncation: the main pass computes diagonals d >= d0 only.
 * d0 is the lowest diagonal for which an entry whose magnitude is up to
 * kDeltaBits below the largest possible product (cancellation or small
 * entries) still certifies its rounding with kMarginBits to spare; an entry
 * fails only when it lies about kDeltaBits + kMarginBits bits or more below
 * that product (or next to a rounding midpoint), and its tile is then
 * recomputed exactly.  For random-sign sums the share of entries more than t
 * bits below falls as ~2^-t (measured: none of 65536 entries of 1024-term
 * dot products below 15 bits), so a failure is rare and costs one tile's low
 * diagonals, while every diagonal skipped saves up to S slice pairs of every
 * tile: 24 bits (d0 = 65 at PB=512) instead of 40 (d0 = 63) skips 4.7% more
 * of the tensor work. */
constexpr int kDeltaBits = 24;
constexpr int kMarginBits = 16;
constexpr size_t kSmemBytes = 1024 /* alignment slack */ + STAGES * (A_STAGE + B_STAGE) + 256 /* barriers */;

/* the per-call geometry (host and device) */
struct Plan {
  int prec, N, S, SP, XL, cplx, nprod;
  int m, n, k, kp, KC; /* kp = k padded to BK, KC = kp / BK chunks */
  int P, cpp;          /* k-parts per diagonal, chunks per part */
  int mt, nt;          /* tiles */
  int d0;              /* lowest diagonal of the main pass (0: all diagonals, no certification) */
  size_t dplane;       /* elements from one diagonal plane to the next (m*n, padded) */
  long cert;           /* log2 of the bound on the omitted diagonals' sum (LSB units); -1 when d0 = 0 */
  long units;          /* units of the main pass, diagonals [d0, 2S-2] */
  size_t off_rowE, off_colE, off_colEmin, off_flags, off_cnt, off_ef, off_tf, off_tiles, off_asl, off_bsl, off_d,
      total;
};

static inline int ceil_log2(long x) {
  int r = 0;
  while ((1L << r) < x) ++r;
  return r;
}

static inline size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

static bool make_plan(int prec, size_t m, size_t n, size_t k, int sp_bits, int cplx, Plan &p) {
  if (sp_bits < 0 || sp_bits > 1024) return false;
  const int guard = cplx ? 3 : 2;
  p.prec = prec;
  p.N = prec / 32;
  p.cplx = cplx ? 1 : 0;
  p.nprod = cplx ? 3 : 1;
  p.S = (prec + sp_bits + guard + 7) / 8;
  p.SP = 8 * p.S - prec - guard;
  const int extra_bits = 8 * p.S - prec;
  const int xl = (extra_bits + 31) / 32;
  p.XL = xl <= 1 ? 1 : xl <= 2 ? 2 : xl <= 4 ? 4 : -1;
  if (p.XL < 0) return false;
  p.m = (int)m;
  p.n = (int)n;
  p.k = (int)k;
  p.kp = (int)((k + BK - 1) / BK * BK);
  p.KC = p.kp / BK;
  const long terms = (long)p.S * p.kp;
  p.P = (int)((terms + kSafeTerms - 1) / kSafeTerms);
  if (p.P < 1) p.P = 1;
  p.cpp = (p.KC + p.P - 1) / p.P;
  p.P = (p.KC + p.cpp - 1) / p.cpp;
  if (p.P > kMaxParts) return false;
  p.mt = (int)((m + BM - 1) / BM);
  p.nt = (int)((n + BN - 1) / BN);
  /* The omitted sum R = sum_{d<d0} 256^d D_d has |D_d| <= c*kp*(d+1)*2^14
   * (c = sum of the |coefficients| of the products in one component: 1 real,
   * at most 3 complex), so |R| < c*kp*d0*2^(6.006)*256^d0 <= 2^cert with
   * cert = 8*d0 + 7 + ceil(log2(c*kp*d0)).  The largest possible product has
   * its top bit at 2*PB + 2*SP - 1; a result kDeltaBits below that has its
   * ULP at PB + 2*SP - kDeltaBits, and cert must stay kMarginBits under it. */
  {
    const int c = cplx ? 3 : 1;
    const long budget = (long)prec + 2L * p.SP - kDeltaBits - kMarginBits;
    p.d0 = 0;
    p.cert = -1;
    for (int d = p.S - 1; d >= 1; --d) {
      const long cert = 8L * d + 7 + ceil_log2((long)c * p.kp * d);
      if (cert <= budget) {
        p.d0 = d;
        p.cert = cert;
        break;
      }
    }
  }
  p.units = (long)p.nprod * (2 * p.S - 1 - p.d0) * p.mt * p.nt * p.P;
  /* Diagonal planes are m*n int32 each; the rounding reads one entry from
   * every plane, so a power-of-two plane size would send all of those loads
   * to the same DRAM channels.  The stride is padded by 4224 bytes (33 x 128)
   * to spread them; it stays a multiple of 128 bytes. */
  p.dplane = (m * n + 31) / 32 * 32 + 1056;
  size_t o = 0;
  p.off_rowE = o;
  o = up256(o + 4 * m);
  p.off_colE = o;
  o = up256(o + 4 * n);
  p.off_colEmin = o;
  o = up256(o + 4 * n);
  p.off_flags = o; /* m row flags then n column flags, one byte each */
  o = up256(o + m + n);
  p.off_cnt = o; /* [0] fallback rows+cols, [1] kernel error, [2] tiles to recompute */
  o = up256(o + 16);
  p.off_ef = o; /* one byte per entry: 1 = rounding not certified, recomputed */
  o = up256(o + m * n);
  p.off_tf = o; /* one int per output tile: marked for recomputation */
  o = up256(o + 4 * (size_t)p.mt * p.nt);
  p.off_tiles = o; /* list of marked tiles */
  o = up256(o + 4 * (size_t)p.mt * p.nt);
  p.off_asl = o;
  o = up256(o + (size_t)p.nprod * p.S * m * p.kp);
  p.off_bsl = o;
  o = up256(o + (size_t)p.nprod * p.S * n * p.kp);
  p.off_d = o;
  o = up256(o + (size_t)p.nprod * p.P * (2 * p.S - 1) * p.dplane * 4);
  p.total = o;
  return true;
}

/* element idx of a real (CPLX=false) or complex tiled matrix */
template <int N, bool CPLX>
__device__ __forceinline__ void load_any(fval<N> &re, fval<N> &im, const uint8_t *base, size_t idx) {
  if (CPLX)
    load_celem<N>(re, im, base, idx);
  else
    load_elem<N>(re, base, idx);
}
/* head word of element idx, part 0 (real / re) or 1 (im) */
template <int N, bool CPLX>
__device__ __forceinline__ uint32_t head_of(const uint8_t *base, size_t idx, int part) {
  constexpr size_t TB = sol<N>::kTileBytes;
  const uint8_t *t = base + (idx >> 5) * (CPLX ? 2u : 1u) * TB + (size_t)part * TB;
  return __ldg((const uint32_t *)(t + sol<N>::kHeadOff) + (idx & 31u));
}

/* ------------------------------------------------------------------ *
 * 1. exponent statistics
 * ------------------------------------------------------------------ */
/* Column statistics of B first: k is split into chunks of kColRows rows, one
 * block per (32 columns, chunk), and each block folds its partial max / min
 * exponent into colE / colEmin with atomics (initialised to kColNone /
 * kColMinNone by a byte memset).  k_row_stats then finalises the columns. */
constexpr int kColRows = 32; /* 32-row chunks: a 512 x 512 B is 256 blocks, enough for every SM */
constexpr int32_t kColNone = (int32_t)0x80808080;    /* memset 0x80: no nonzero entry seen */
constexpr int32_t kColMinNone = (int32_t)0x7f7f7f7f; /* memset 0x7f */
template <int N, bool CPLX>
__global__ void __launch_bounds__(256) k_col_stats(int n, int k, const uint8_t *B, size_t ldb, int32_t *colE,
                                                   int32_t *colEmin) {
  pdl_wait(); /* launched after the previous stage with launch_pdl */
  __shared__ int32_t smax[8][32], smin[8][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int j = blockIdx.x * 32 + lane;
  const int k0 = blockIdx.y * kColRows, k1 = min(k, k0 + kColRows);
  int32_t emax = kColNone, emin = kColMinNone;
  if (j < n) {
    /* unrolled: several rows' head loads in flight per lane */
#pragma unroll 4
    for (int kk = k0 + w; kk < k1; kk += 8) {
#pragma unroll
      for (int part = 0; part < (CPLX ? 2 : 1); ++part) {
        const uint32_t h = head_of<N, CPLX>(B, (size_t)kk * ldb + j, part);
        if (h != kHeadZero) {
          const int32_t e = head_exp(h);
          emax = max(emax, e);
          emin = min(emin, e);
        }
      }
    }
  }
  smax[w][lane] = emax;
  smin[w][lane] = emin;
  __syncthreads();
  if (w == 0 && j < n) {
    for (int q = 1; q < 8; ++q) {
      emax = max(emax, smax[q][lane]);
      emin = min(emin, smin[q][lane]);
    }
    if (emax != kColNone) {
      atomicMax(colE + j, emax);
      atomicMin(colEmin + j, emin);
    }
  }
}

/* one block of kRowWarps warps per row of A, the warps splitting k: E_i =
 * max exponent of the nonzero entries (both parts of a complex entry); flag
 * the row when some nonzero entry lies more than SP bits below E_i.  The same
 * launch finalises the column statistics: an all-zero column gets kExpZero,
 * a column whose spread exceeds SP is flagged; flagged rows and columns are
 * counted. */
constexpr int kRowWarps = 4;
template <int N, bool CPLX>
__global__ void __launch_bounds__(kRowWarps * 32) k_row_stats(int m, int k, const uint8_t *A, size_t lda, int SP,
                                                              int32_t *rowE, uint8_t *rowF, int n, int32_t *colE,
                                                              const int32_t *colEmin, uint8_t *colF, int *count) {
  pdl_wait(); /* launched after the previous stage with launch_pdl */
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int32_t e = colE[j];
    const bool none = e == kColNone;
    const bool flag = !none && (long)e - colEmin[j] > SP;
    colE[j] = none ? kExpZero : e;
    colF[j] = flag ? 1 : 0;
    if (flag) atomicAdd(count, 1);
  }
  __shared__ int32_t smax[kRowWarps], smin[kRowWarps];
  const int row = blockIdx.x, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (row >= m) return; /* block-uniform */
  int32_t emax = kExpZero, emin = 0x7fffffff;
#pragma unroll 4
  for (int k0 = w * 32; k0 < k; k0 += kRowWarps * 32) {
    const int kk = k0 + lane;
    if (kk < k) {
#pragma unroll
      for (int part = 0; part < (CPLX ? 2 : 1); ++part) {
        const uint32_t h = head_of<N, CPLX>(A, (size_t)row * lda + kk, part);
        if (h != kHeadZero) {
          const int32_t e = head_exp(h);
          emax = max(emax, e);
          emin = min(emin, e);
        }
      }
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    emax = max(emax, __shfl_xor_sync(0xffffffffu, emax, o));
    emin = min(emin, __shfl_xor_sync(0xffffffffu, emin, o));
  }
  if (lane == 0) {
    smax[w] = emax;
    smin[w] = emin;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < kRowWarps; ++q) {
      emax = max(emax, smax[q]);
      emin = min(emin, smin[q]);
    }
    rowE[row] = emax;
    const bool flag = emax != kExpZero && (long)emax - emin > SP;
    rowF[row] = flag ? 1 : 0;
    if (flag) atomicAdd(count, 1);
  }
}

/* ------------------------------------------------------------------ *
 * 2. slicing into balanced base-256 digits
 * ------------------------------------------------------------------ */
/* V = (-1)^s * M * 2^sh, 0 <= sh = SP - (Erow - e) <= SP, as a two's
 * complement integer of L+1 limbs (L = N + XL holds M << sh). */
template <int N, int XL>
__device__ __forceinline__ void aligned_twos(uint32_t (&w)[N + XL + 1], const fval<N> &x, int32_t Erow, int SP) {
  constexpr int L = N + XL;
  const bool zero = is_zero(x);
  const uint32_t sh = zero ? 0u : (uint32_t)(SP - (Erow - x.e));
  const uint32_t q = sh >> 5, r = sh & 31u;
#pragma unroll
  for (int i = 0; i <= L; ++i) w[i] = (i < N && !zero) ? x.m[i] : 0u;
#pragma unroll
  for (int b = 0; (1 << b) <= XL; ++b) { /* limb shift q < XL + 1 */
    const int s = 1 << b;
    const bool on = (q >> b) & 1u;
#pragma unroll
    for (int i = L; i >= 0; --i) {
      const uint32_t src = (i - s >= 0) ? w[i - s] : 0u;
      w[i] = on ? src : w[i];
    }
  }
#pragma unroll
  for (int i = L; i > 0; --i) w[i] = fshl(w[i - 1], w[i], r);
  w[0] <<= r;
  if (x.s && !zero) { /* negate */
    uint32_t c = 1u;
#pragma unroll
    for (int i = 0; i <= L; ++i) {
      const uint32_t t = ~w[i] + c;
      c = (c && t == 0u) ? 1u : 0u;
      w[i] = t;
    }
  }
}
/* balanced base-256 digits of a two's complement integer V: the digits in
 * [-128, 127] with V = sum d_s 256^s are the bytes of U = V + 0x8080...80,
 * each XOR 0x80 (adding 128 to every byte produces exactly the carries of
 * the digit-by-digit recoding: byte b plus carry becomes b - 256, carry 1,
 * when it reaches 128).  One carry chain for U, then every digit is a byte
 * extraction.  For |V| < 2^(8S-2) every digit above S-1 is zero, so only
 * the digits s < S are written. */
template <int L1>
__device__ __forceinline__ void offset_words(uint32_t (&u)[L1], const uint32_t (&w)[L1]) {
  uint32_t cf = 0;
  u[0] = add_cc(w[0], 0x80808080u, cf);
#pragma unroll
  for (int i = 1; i < L1; ++i) u[i] = addc_cc(w[i], 0x80808080u, cf);
}

/* elements per thread of the slicing kernels: E consecutive k of one row of
 * A (column of B), so every digit plane gets E bytes per store (one 32-bit
 * store for E = 4) while the E elements' offset words fit in registers */
template <int N, bool CPLX>
struct slice_geo {
  static constexpr int E = CPLX ? (N <= 8 ? 4 : N <= 16 ? 2 : 1) : (N <= 16 ? 4 : N <= 32 ? 2 : 1);
};

/* The digit planes of E consecutive elements for product q (0: the real
 * part, 1: the imaginary part, 2: re + im): ld(e, re, im) loads element e
 * (zero when it is padding or flagged); the digits of plane s go to
 * dst + s * plane, E bytes (E-aligned), element e in byte e. */
template <int N, int XL, bool CPLX, int E, typename Ld>
__device__ __forceinline__ void slice_elements(Ld ld, int32_t Eexp, int SP, int S, int q, int8_t *dst, size_t plane) {
  constexpr int L1 = N + XL + 1;
  uint32_t u[E][L1];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    fval<N> re, im;
    ld(e, re, im);
    uint32_t w[L1];
    aligned_twos<N, XL>(w, q == 1 ? im : re, Eexp, SP);
    if (CPLX && q == 2) {
      uint32_t v[L1];
      aligned_twos<N, XL>(v, im, Eexp, SP);
      uint32_t c = 0;
#pragma unroll
      for (int i = 0; i < L1; ++i) {
        const uint64_t t = (uint64_t)w[i] + v[i] + c;
        w[i] = (uint32_t)t;
        c = (uint32_t)(t >> 32);
      }
    }
    offset_words<L1>(u[e], w);
  }
#pragma unroll
  for (int s = 0; s < 4 * L1; ++s) {
    if (s >= S) continue; /* predicated: the loop stays unrolled, u in registers */
    const int wd = s >> 2, b = s & 3;
    int8_t *o = dst + (size_t)s * plane;
    if (E == 4) {
      /* byte b of each element's word, elements 0..3 in bytes 0..3 */
      const uint32_t t01 = __byte_perm(u[0][wd], u[E > 1 ? 1 : 0][wd], (uint32_t)(b | ((4 + b) << 4)));
      const uint32_t t23 = __byte_perm(u[E > 2 ? 2 : 0][wd], u[E > 3 ? 3 : 0][wd], (uint32_t)(b | ((4 + b) << 4)));
      *(uint32_t *)o = __byte_perm(t01, t23, 0x5410u) ^ 0x80808080u;
    } else if (E == 2) {
      const uint32_t t01 = __byte_perm(u[0][wd], u[E > 1 ? 1 : 0][wd], (uint32_t)(b | ((4 + b) << 4)));
      *(uint16_t *)o = (uint16_t)((t01 ^ 0x8080u) & 0xffffu);
    } else {
      *o = (int8_t)(((u[0][wd] >> (8 * b)) & 0xffu) ^ 0x80u);
    }
  }
}

/* A (m x k, tiles) -> A_sl[q*S+s][i][kp]; thread per (i, E consecutive kk),
 * kk < kp (zero padding) */
template <int N, int XL, bool CPLX>
__global__ void __launch_bounds__(128) k_slice_a(int m, int k, int kp, const uint8_t *A, size_t lda, int SP, int S,
                                                 const int32_t *rowE, const uint8_t *rowF, int8_t *Asl) {
  pdl_wait(); /* launched after the previous stage with launch_pdl */
  constexpr int E = slice_geo<N, CPLX>::E;
  const size_t groups = (size_t)kp / E, total = (size_t)m * groups, plane = (size_t)m * kp;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx / groups), kk0 = (int)(idx % groups) * E;
    const bool live = !rowF[i];
    const int32_t Ex = rowE[i];
    int8_t *dst = Asl + (size_t)i * kp + kk0;
#pragma unroll 1
    for (int q = 0; q < (CPLX ? 3 : 1); ++q)
      slice_elements<N, XL, CPLX, E>(
          [&](int e, fval<N> &re, fval<N> &im) {
            set_zero(im);
            if (live && kk0 + e < k)
              load_any<N, CPLX>(re, im, A, (size_t)i * lda + kk0 + e);
            else
              set_zero(re);
          },
          Ex, SP, S, q, dst + (size_t)q * S * plane, plane);
  }
}

/* B (k x n, tiles) -> B_sl[q*S+s][j][kp]: thread per (j, E consecutive kk)
 * with kk running fastest across the lanes, so each digit plane is written as
 * 32E-byte rows (E bytes per lane) and no staging is needed; the lanes'
 * element loads come from rows of B (16-byte pieces whose tile neighbours
 * are read by the warps of columns j +- 1 soon after, from L2). */
template <int N, int XL, bool CPLX>
__global__ void __launch_bounds__(128) k_slice_b(int n, int k, int kp, const uint8_t *B, size_t ldb, int SP, int S,
                                                 const int32_t *colE, const uint8_t *colF, int8_t *Bsl) {
  pdl_wait(); /* launched after the previous stage with launch_pdl */
  constexpr int E = slice_geo<N, CPLX>::E;
  const size_t groups = (size_t)kp / E, total = (size_t)n * groups, plane = (size_t)n * kp;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(idx / groups), kk0 = (int)(idx % groups) * E;
    const bool live = !colF[j];
    const int32_t Ex = colE[j];
    int8_t *dst = Bsl + (size_t)j * kp + kk0;
#pragma unroll 1
    for (int q = 0; q < (CPLX ? 3 : 1); ++q)
      slice_elements<N, XL, CPLX, E>(
          [&](int e, fval<N> &re, fval<N> &im) {
            set_zero(im);
            if (live && kk0 + e < k)
              load_any<N, CPLX>(re, im, B, (size_t)(kk0 + e) * ldb + j);
            else
              set_zero(re);
          },
          Ex, SP, S, q, dst + (size_t)q * S * plane, plane);
  }
}

/* ------------------------------------------------------------------ *
 * 3. the tcgen05 diagonal GEMM
 * ------------------------------------------------------------------ */
struct GemmArgs {
  int S, nprod, mt, nt, P, cpp, KC, m, n;
  size_t dplane;       /* elements between consecutive diagonal planes */
  int dl, dh;          /* diagonals computed: [dl, dh] */
  long units;          /* all tiles (tiles == nullptr) */
  const int *tiles;    /* or only these output tiles ... */
  const int *ntiles;   /* ... *ntiles of them, counted on the device */
  int32_t *D;          /* [nprod][P][2S-1][dplane], each plane m x n */
  int *err;
  uint64_t wait_ns;    /* limit of every mbarrier wait (sm100::kWaitNs unless a test shortens it) */
  int inject;          /* test of the failure path: 1 = CTA 0 withholds its first accumulator
                        * commit, so its epilogue's wait runs out; 0 otherwise */
};

/* tensor-core phase (exact_gemm.cu): TMA maps over the digit planes and the
 * persistent tcgen05 diagonal-GEMM launch over diagonals [dl, dh] of every
 * tile (tiles == nullptr) or of the device-side tile list; returns an
 * mpb_status */
int launch_diag_gemm(const Plan &p, int8_t *Asl, int8_t *Bsl, int32_t *D, int *err, int dl, int dh,
                     const int *tiles, const int *ntiles, cudaStream_t st);
/* a TMA map over the computed diagonal planes of a rounding pass (exact_gemm.cu):
 * int32 [nprod][nl][entries] from base, plane stride plane_elems, product
 * stride q_elems, box {box_x entries, nl planes, 1 product}, no swizzle */
bool make_plane_tmap(CUtensorMap *tm, const int32_t *base, size_t entries, int nl, int nprod, size_t plane_elems,
                     size_t q_elems, int box_x);

/* ------------------------------------------------------------------ *
 * 4. exact recombination and the single rounding
 * ------------------------------------------------------------------ */
/* Q 32-bit words cover sum_d 256^d D_d (2S-1 diagonals, up to 3 products
 * with coefficients +-1 and 16 parts): 8(2S-2) + 31 + 8 + sign bits */
template <int N, int XL>
struct round_geo {
  static constexpr int SMAX = 4 * (N + XL);
  static constexpr int Q = (8 * (2 * SMAX - 2) + 31 + 8 + 31) / 32 + 1;
  /* the single-part first pass reads at most J planes, from d0 on; their sum
   * (coefficients up to 3) spans 8(J-1) + 35 bits with the sign */
  static constexpr int J = SMAX + 20;
  static constexpr int QJ = (8 * (J - 1) + 35 + 31) / 32 + 1;
  /* threads per block of the first pass: each keeps (QJ | 1) words per
   * component in shared memory, within the 48 KB static limit.  The launch
   * bound asks for 5 (10) resident blocks, i.e. at most ~100 registers: the
   * pass is latency-bound and needs many warps, each with a batch of plane
   * loads in flight, more than registers per thread. */
  template <bool CPLX>
  static constexpr int threads() {
    return 128 * (QJ | 1) * (CPLX ? 2 : 1) * 4 <= 46 * 1024 ? 128 : 64;
  }
};

/* Normalise and round once: v[0..W) is the two's complement integer
 * (LSB weight 2^lsb_exp) of an exact sum; r = RNDN(v) to N limbs.
 *
 * With cert >= 0, v is a truncated sum whose true value differs from it by
 * less than 2^cert (LSB units), and the rounding is accepted only when every
 * value within that distance rounds the same way: the bound must be below a
 * quarter ULP (so no binade change can matter) and the remainder below the
 * ULP, read as the 64-bit fraction G, must stay clear of the midpoint by
 * more than the bound.  Returns false (r unspecified) otherwise; a zero sum
 * is never certified. */
template <int N, int W>
__device__ __forceinline__ bool round_words(fval<N> &r, uint32_t (&v)[W], long lsb_exp, long cert) {
  static_assert(W >= N + 2, "word window too small");
  const uint32_t neg = v[W - 1] >> 31;
  if (neg) {
    uint32_t c = 1;
#pragma unroll
    for (int w = 0; w < W; ++w) {
      const uint32_t t = ~v[w] + c;
      c = (c && t == 0) ? 1u : 0u;
      v[w] = t;
    }
  }
  int lq = W;
  uint32_t top = 0;
#pragma unroll
  for (int w = W - 1; w >= 0; --w) {
    const bool take = (lq == W) && v[w] != 0;
    top = take ? v[w] : top;
    lq = take ? (W - 1 - w) : lq;
  }
  if (lq == W) {
    set_zero(r);
    return cert < 0;
  }
  const uint32_t lr = clz32(top) & 31u;
#pragma unroll
  for (int b = 0; (1 << b) < W; ++b) {
    const int s = 1 << b;
    const bool on = (lq >> b) & 1;
#pragma unroll
    for (int w = W - 1; w >= 0; --w) {
      const uint32_t src = (w - s >= 0) ? v[w - s] : 0u;
      v[w] = on ? src : v[w];
    }
  }
#pragma unroll
  for (int w = W - 1; w > 0; --w) v[w] = fshl(v[w - 1], v[w], lr);
  v[0] <<= lr;
#pragma unroll
  for (int w = 0; w < N; ++w) r.m[w] = v[W - N + w];
  const uint32_t g = v[W - N - 1];
  uint32_t st = g << 1;
#pragma unroll
  for (int w = 0; w < W - N - 1; ++w) st |= v[w];
  /* msb of the exact integer: 32*W - 1 - (32*lq + lr) */
  const long msb = 32L * W - 1 - (32L * lq + lr);
  bool ok = true;
  if (cert >= 0) {
    const long t = cert - (msb - 32L * N + 1); /* log2 of the bound in ULPs */
    const uint64_t G = ((uint64_t)g << 32) | v[W - N - 2];
    /* the bound in 2^-64 ULPs (rounded up); only t <= -3 can certify, so the
     * shift is taken only there, where 64 + t < 62 */
    const uint64_t half = 1ull << 63;
    if (t > -3) {
      ok = false;
    } else {
      const uint64_t thr = (t < -64) ? 1ull : (1ull << (64 + t));
      ok = G <= half - thr - 1 || G > half + thr;
    }
  }
  int32_t ee = (int32_t)(msb + 1 + lsb_exp);
  rndn<N>(r.m, ee, g >> 31, st);
  r.e = ee;
  r.s = neg;
  return ok;
}

/* round_words for a sum held in registers v[0..W) with a shared-memory slot
 * sv[0..W) for this thread: the sign, the magnitude (negation with one carry
 * chain), the top nonzero word and the lowest nonzero word come from the
 * registers; the magnitude words then go to sv once, and only the N + 2
 * words under the leading bit are read back, at indices counted from the top
 * word (no shift network over all W words).  Everything below those words
 * only matters as the sticky bit, which is "the lowest nonzero word lies
 * below them".  Same result and certification as round_words. */
template <int N, int W>
__device__ __forceinline__ bool round_regs(fval<N> &r, uint32_t (&v)[W], uint32_t *sv, long lsb_exp, long cert) {
  static_assert(W >= N + 2, "word window too small");
  const uint32_t neg = v[W - 1] >> 31;
  {
    const uint32_t msk = 0u - neg;
    uint32_t cf = 0;
    cc_set(neg, cf);
#pragma unroll
    for (int w = 0; w < W; ++w) v[w] = addc_cc(v[w] ^ msk, 0u, cf);
  }
  int top = -1, low = W;
#pragma unroll
  for (int w = 0; w < W; ++w) top = v[w] != 0u ? w : top;
#pragma unroll
  for (int w = W - 1; w >= 0; --w) low = v[w] != 0u ? w : low;
  if (top < 0) {
    set_zero(r);
    return cert < 0;
  }
#pragma unroll
  for (int w = 0; w < W; ++w) sv[w] = v[w];
  auto word = [&](int i) -> uint32_t { return i >= 0 ? sv[i] : 0u; };
  const uint32_t lr = clz32(sv[top]) & 31u;
#pragma unroll
  for (int i = 0; i < N; ++i) r.m[N - 1 - i] = fshl(word(top - i - 1), word(top - i), lr);
  const uint32_t g = fshl(word(top - N - 1), word(top - N), lr);
  const uint32_t nx = fshl(word(top - N - 2), word(top - N - 1), lr);
  const uint32_t st = (g << 1) | (word(top - N - 1) << lr) | (low <= top - N - 2 ? 1u : 0u);
  const long msb = 32L * top + 31 - lr;
  bool ok = true;
  if (cert >= 0) {
    const long t = cert - (msb - 32L * N + 1); /* log2 of the bound in ULPs */
    const uint64_t G = ((uint64_t)g << 32) | nx;
    const uint64_t half = 1ull << 63;
    if (t > -3) {
      ok = false;
    } else {
      const uint64_t thr = (t < -64) ? 1ull : (1ull << (64 + t));
      ok = G <= half - thr - 1 || G > half + thr;
    }
  }
  int32_t ee = (int32_t)(msb + 1 + lsb_exp);
  rndn<N>(r.m, ee, g >> 31, st);
  r.e = ee;
  r.s = neg;
  return ok;
}

/* One rounding pass of the exact GEMM (both kernels below).
 * Pass 1 (flagged_only = 0) visits every entry, sums the diagonals
 * [d_first, 2S-2] and, when d_first > 0, certifies the rounding against the
 * omitted diagonals (cert); an entry that does not certify is not stored but
 * marked in ef, and its output tile is appended once to the tile list.
 * Pass 2 (flagged_only = 1) visits the entries of the listed tiles whose ef is
 * set, after the tensor cores have filled in their low diagonals, and rounds
 * the full sum (d_first = 0, no certification). */
struct RoundPass {
  size_t dplane; /* elements between consecutive diagonal planes */
  int d_first;
  long cert;
  int flagged_only;
  int nt;          /* output tiles per row of tiles */
  uint8_t *ef;     /* m*n entry flags */
  int *tf;         /* mt*nt tile marks */
  int *tiles;      /* marked tiles */
  int *ntiles;     /* their count */
};

/* entry u of a pass: false when the entry is not visited */
__device__ __forceinline__ bool pass_entry(const RoundPass &rp, int m, int n, size_t u, int &i, int &j, size_t &idx) {
  if (rp.flagged_only) {
    const int tile = rp.tiles[u / (BM * BN)];
    const int r = (int)(u % (BM * BN));
    i = (tile / rp.nt) * BM + r / BN;
    j = (tile % rp.nt) * BN + r % BN;
    if (i >= m || j >= n) return false;
    idx = (size_t)i * n + j;
    return rp.ef[idx] != 0;
  }
  idx = u;
  if (u < (1ull << 32)) { /* 32-bit division when the index fits */
    i = (int)((uint32_t)u / (uint32_t)n);
    j = (int)((uint32_t)u - (uint32_t)i * (uint32_t)n);
  } else {
    i = (int)(u / n);
    j = (int)(u % n);
  }
  return true;
}
__device__ __forceinline__ size_t pass_total(const RoundPass &rp, int m, int n) {
  return rp.flagged_only ? (size_t)(*rp.ntiles) * (BM * BN) : (size_t)m * n;
}
__device__ __forceinline__ void mark_tile(const RoundPass &rp, int i, int j) {
  const int tile = (i / BM) * rp.nt + j / BN;
  if (atomicExch(rp.tf + tile, 1) == 0) rp.tiles[atomicAdd(rp.ntiles, 1)] = tile;
}

/* One entry (i, j) of a single-part (P == 1) rounding pass over at most J
 * planes from d_first on.  ld(q, jc) returns plane d_first + jc of product q
 * for this entry (jc < nl; plane indices at or past nl are read clamped and
 * count as zero, so every load of a batch is unconditional and all are in
 * flight before any is used).  The planes are taken BATCH at a time and
 * streamed into 32-bit words with an int64 carry -- plane d_first + j lands
 * in word j/4, byte j%4.  The words hold the sum divided by 256^d_first, so
 * the LSB exponent and the certification bound move up by 8 d_first bits
 * instead of the words moving.  round_regs rounds them, reading the few
 * words under the leading bit from this thread's shared-memory slots svr /
 * svi.  Complex outputs read each product's planes once and form both
 * components: re = T0 - T1, im = T2 - T0 - T1.  Every loop is unrolled at
 * compile time. */
template <int N, int XL, bool CPLX, class Ld>
__device__ __forceinline__ void round_entry(int i, int j, size_t idx, int nl, int SP, const int32_t *rowE,
                                            const int32_t *colE, uint8_t *C, size_t ldc, const RoundPass &rp,
                                            uint32_t *svr, uint32_t *svi, Ld ld) {
  constexpr int QJ = round_geo<N, XL>::QJ;
  constexpr int BATCH = CPLX ? 8 : 16; /* a multiple of 4 */
  /* BATCH planes of every product in flight, then their BATCH/4 words:
   * word w = carry + sum of planes 4w..4w+3 (each < 2^31, times 2^(8j)),
   * low 32 bits kept, the rest carried on */
  uint32_t vr[QJ], vi[CPLX ? QJ : 1];
  long long cr = 0, ci = 0;
#pragma unroll
  for (int j0 = 0; j0 < 4 * QJ; j0 += BATCH) {
    int32_t t0v[BATCH], t1v[CPLX ? BATCH : 1], t2v[CPLX ? BATCH : 1];
#pragma unroll
    for (int jj = 0; jj < BATCH; ++jj) {
      /* unconditional loads (a plane past the last one re-reads the last,
       * then counts as 0), so they can all be issued before any is used */
      const bool in = j0 + jj < nl;
      const int jc = min(j0 + jj, nl - 1);
      const int32_t x0 = ld(0, jc);
      t0v[jj] = in ? x0 : 0;
      if (CPLX) {
        const int32_t x1 = ld(1, jc), x2 = ld(2, jc);
        t1v[jj] = in ? x1 : 0;
        t2v[jj] = in ? x2 : 0;
      }
    }
#pragma unroll
    for (int w4 = 0; w4 < BATCH / 4; ++w4) {
      const int w = j0 / 4 + w4;
      if (w < QJ) {
        long long tr = cr, ti = ci;
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const long long scale = 1LL << (8 * jj);
          const long long t0 = t0v[4 * w4 + jj];
          if (CPLX) {
            const long long t1 = t1v[4 * w4 + jj], t2 = t2v[4 * w4 + jj];
            tr += (t0 - t1) * scale;
            ti += (t2 - t0 - t1) * scale;
          } else {
            tr += t0 * scale;
          }
        }
        vr[w] = (uint32_t)tr;
        cr = tr >> 32;
        if (CPLX) {
          vi[w] = (uint32_t)ti;
          ci = ti >> 32;
        }
      }
    }
  }
  const long lsb = (long)rowE[i] + colE[j] - 2L * (32 * N) - 2L * SP + 8L * rp.d_first;
  /* an all-zero row or column has all-zero digits: its sum is exactly 0 */
  const long cert =
      (rowE[i] == kExpZero || colE[j] == kExpZero || rp.cert < 0) ? -1 : rp.cert - 8L * rp.d_first;
  fval<N> re;
  bool ok = round_regs<N, QJ>(re, vr, svr, lsb, cert);
  fval<N> im;
  if (CPLX) ok = round_regs<N, QJ>(im, *reinterpret_cast<uint32_t(*)[QJ]>(vi), svi, lsb, cert) && ok;
  if (!rp.flagged_only) {
    rp.ef[idx] = ok ? 0 : 1;
    if (!ok) {
      mark_tile(rp, i, j);
      return;
    }
  }
  if (CPLX)
    store_celem<N>(C, (size_t)i * ldc + j, re, im);
  else
    store_elem<N>(C, (size_t)i * ldc + j, re);
}

/* The single-part first pass with each thread loading its own planes (the
 * sizes whose shared-memory stage would exceed the TMA kernel's limit). */
template <int N, int XL, bool CPLX>
__global__ void __launch_bounds__(round_geo<N, XL>::template threads<CPLX>(),
                                  round_geo<N, XL>::template threads<CPLX>() == 128 ? 4 : 8)
    k_exact_round(int m, int n, int S, int SP, const int32_t *__restrict__ D, const int32_t *rowE, const int32_t *colE,
                  const uint8_t *rowF, const uint8_t *colF, uint8_t *C, size_t ldc, RoundPass rp) {
  pdl_wait(); /* launched after the previous stage with launch_pdl */
  constexpr int J = round_geo<N, XL>::J;
  constexpr int QJ = round_geo<N, XL>::QJ;
  constexpr int SW = QJ | 1; /* odd word stride per thread: conflict-free banks */
  constexpr int T = round_geo<N, XL>::template threads<CPLX>();
  __shared__ uint32_t swords[T * SW * (CPLX ? 2 : 1)];
  uint32_t *svr = swords + threadIdx.x * SW * (CPLX ? 2 : 1);
  uint32_t *svi = svr + SW;
  static_assert(4 * QJ >= J, "words must cover the planes");
  const size_t total = pass_total(rp, m, n), plane = rp.dplane;
  const int ndiag = 2 * S - 1;
  const int nl = ndiag - rp.d_first; /* <= J, checked on the host */
  const size_t qstride = (size_t)ndiag * plane;
  for (size_t u = (size_t)blockIdx.x * blockDim.x + threadIdx.x; u < total; u += (size_t)gridDim.x * blockDim.x) {
    int i, j;
    size_t idx;
    if (!pass_entry(rp, m, n, u, i, j, idx)) continue;
    if (rowF[i] || colF[j]) { /* computed by the fallback */
      if (!rp.flagged_only) rp.ef[idx] = 0;
      continue;
    }
    const int32_t *base = D + (size_t)rp.d_first * plane + idx;
    round_entry<N, XL, CPLX>(i, j, idx, nl, SP, rowE, colE, C, ldc, rp, svr, svi,
                             [&](int q, int jc) { return base[(size_t)q * qstride + (size_t)jc * plane]; });
  }
}

/* The first pass with the planes staged in shared memory: the T consecutive
 * entries of a block-step arrive for every computed plane (nprod x nl rows
 * of T int32) by one TMA load per product (no multicast) on the block's
 * mbarrier, and round_entry reads them from shared memory.  The plane bytes
 * then stream from HBM while the other blocks of the SM compute, instead of
 * each thread waiting on its own plane loads.  The wait is bounded: on
 * timeout the block records code 6 in err, waits (bounded) for its copy and
 * returns.  Entries past the end of C are zero-filled by the copy and not
 * visited. */
template <int N, int XL, bool CPLX>
__global__ void __launch_bounds__(round_geo<N, XL>::template threads<CPLX>(), 3)
    k_exact_round_tma(const __grid_constant__ CUtensorMap tmD, int m, int n, int SP, const int32_t *rowE,
                      const int32_t *colE, const uint8_t *rowF, const uint8_t *colF, uint8_t *C, size_t ldc,
                      RoundPass rp, int nl, long long wait_ns, int *err) {
  pdl_wait(); /* launched after the previous stage with launch_pdl */
  constexpr int QJ = round_geo<N, XL>::QJ;
  constexpr int SW = QJ | 1;
  constexpr int T = round_geo<N, XL>::template threads<CPLX>();
  constexpr int NP = CPLX ? 3 : 1;
  __shared__ uint32_t swords[T * SW * (CPLX ? 2 : 1)];
  __shared__ uint64_t bar;
  extern __shared__ uint8_t dyn_raw[];
  const int32_t *stage = (const int32_t *)(((uintptr_t)dyn_raw + 127) & ~(uintptr_t)127);
  uint32_t *svr = swords + threadIdx.x * SW * (CPLX ? 2 : 1);
  uint32_t *svi = svr + SW;
  if (threadIdx.x == 0) {
    sm100::mbar_init(&bar, 1);
    sm100::fence_barrier_init();
  }
  __syncthreads();
  const size_t total = (size_t)m * n;
  const uint32_t bytes = (uint32_t)NP * (uint32_t)nl * T * 4u;
  volatile int never = 0;
  uint32_t phase = 0u;
  for (size_t c0 = (size_t)blockIdx.x * T; c0 < total; c0 += (size_t)gridDim.x * T) {
    if (threadIdx.x == 0) {
      sm100::mbar_arrive_expect_tx(&bar, bytes);
      for (int q = 0; q < NP; ++q)
        sm100::tma_load_3d((void *)(stage + (size_t)q * nl * T), &tmD, (int)c0, 0, q, &bar);
    }
    const bool ok = sm100::mbar_wait(&bar, phase, &never, (uint64_t)wait_ns);
    if (__syncthreads_or(ok ? 0 : 1)) {
      if (threadIdx.x == 0) {
        atomicCAS(err, 0, 6);
        sm100::mbar_wait(&bar, phase, &never, (uint64_t)wait_ns); /* the copy still in flight */
      }
      return;
    }
    phase ^= 1u;
    const size_t u = c0 + threadIdx.x;
    int i, j;
    size_t idx;
    if (u < total && pass_entry(rp, m, n, u, i, j, idx)) {
      if (rowF[i] || colF[j]) /* computed by the fallback */
        rp.ef[idx] = 0;
      else
        round_entry<N, XL, CPLX>(i, j, idx, nl, SP, rowE, colE, C, ldc, rp, svr, svi,
                                 [&](int q, int jc) { return stage[((size_t)q * nl + jc) * T + threadIdx.x]; });
    }
    __syncthreads(); /* every row read before the next copy overwrites the stage */
  }
}

/* Several k-parts (P > 1, long k): the same sum with the parts added first.
 * Written with run-time loops over per-thread local words to keep the code
 * small; this path only serves k beyond 2^17/S. */
template <int N, int XL, bool CPLX>
__global__ void __launch_bounds__(128) k_exact_round_parts(int m, int n, int S, int SP, int P, const int32_t *D,
                                                           const int32_t *rowE, const int32_t *colE,
                                                           const uint8_t *rowF, const uint8_t *colF, uint8_t *C,
                                                           size_t ldc, RoundPass rp) {
  pdl_wait(); /* launched after the previous stage with launch_pdl */
  constexpr int Q = round_geo<N, XL>::Q;
  const size_t total = pass_total(rp, m, n), plane = rp.dplane;
  const int ndiag = 2 * S - 1;
  const size_t pstride = (size_t)ndiag * plane, qstride = (size_t)P * pstride;
  for (size_t u = (size_t)blockIdx.x * blockDim.x + threadIdx.x; u < total; u += (size_t)gridDim.x * blockDim.x) {
    int i, j;
    size_t idx;
    if (!pass_entry(rp, m, n, u, i, j, idx)) continue;
    if (rowF[i] || colF[j]) {
      if (!rp.flagged_only) rp.ef[idx] = 0;
      continue;
    }
    const long lsb = (long)rowE[i] + colE[j] - 2L * (32 * N) - 2L * SP;
    const long cert = (rowE[i] == kExpZero || colE[j] == kExpZero) ? -1 : rp.cert;
    fval<N> res[CPLX ? 2 : 1];
    bool ok = true;
#pragma unroll 1
    for (int comp = 0; comp < (CPLX ? 2 : 1); ++comp) {
      /* coefficients of T0, T1, T2 for this component */
      const int c0 = CPLX ? (comp == 0 ? 1 : -1) : 1;
      const int c1 = CPLX ? -1 : 0;
      const int c2 = (CPLX && comp == 1) ? 1 : 0;
      long long acc[Q];
      for (int w = 0; w < Q; ++w) acc[w] = 0;
#pragma unroll 1
      for (int d = rp.d_first; d < ndiag; ++d) {
        long long s = 0;
#pragma unroll 1
        for (int p = 0; p < P; ++p) {
          const int32_t *dp = D + (size_t)p * pstride + (size_t)d * plane + idx;
          s += (long long)c0 * __ldcs(dp);
          if (c1) s += (long long)c1 * __ldcs(dp + qstride);
          if (c2) s += (long long)c2 * __ldcs(dp + 2 * qstride);
        }
        acc[d >> 2] += s * (1LL << (8 * (d & 3)));
      }
      uint32_t v[Q];
      long long carry = 0;
#pragma unroll
      for (int w = 0; w < Q; ++w) {
        const long long t = acc[w] + carry;
        v[w] = (uint32_t)t;
        carry = t >> 32;
      }
      ok = round_words<N, Q>(res[comp], v, lsb, cert) && ok;
    }
    if (!rp.flagged_only) {
      rp.ef[idx] = ok ? 0 : 1;
      if (!ok) {
        mark_tile(rp, i, j);
        continue;
      }
    }
    const size_t e = (size_t)i * ldc + j;
    if (CPLX)
      store_celem<N>(C, e, res[0], res[CPLX ? 1 : 0]);
    else
      store_elem<N>(C, e, res[0]);
  }
}

/* one entry of C by the plain per-operation kernel's order */
template <int N, bool CPLX>
__device__ __forceinline__ void fallback_entry(size_t i, size_t j, size_t K, const uint8_t *A, size_t lda,
                                               const uint8_t *B, size_t ldb, uint8_t *C, size_t ldc) {
  if (CPLX) {
    fval<N> cr, ci;
    set_zero(cr);
    set_zero(ci);
    for (size_t k = 0; k < K; ++k) {
      fval<N> ar, ai, br, bi, tr, ti;
      load_celem<N>(ar, ai, A, i * lda + k);
      load_celem<N>(br, bi, B, k * ldb + j);
      cmul<N, false>(tr, ti, br, bi, ar, ai);
      add<N, false>(cr, cr, tr);
      add<N, false>(ci, ci, ti);
    }
    store_celem<N>(C, i * ldc + j, cr, ci);
  } else {
    fval<N> acc;
    set_zero(acc);
    for (size_t k = 0; k < K; ++k) {
      fval<N> a, b, t;
      load_elem<N>(a, A, i * lda + k);
      load_elem<N>(b, B, k * ldb + j);
      mul<N>(t, b, a);
      add<N, false>(acc, acc, t);
    }
    store_elem<N>(C, i * ldc + j, acc);
  }
}

/* flagged rows / columns: plain sequential-k per-operation rounding */
template <int N, bool CPLX>
__global__ void __launch_bounds__(256) k_fallback(size_t m, size_t n, size_t K, const uint8_t *A, size_t lda,
                                                  const uint8_t *B, size_t ldb, uint8_t *C, size_t ldc,
                                                  const uint8_t *rowF, const uint8_t *colF, const int *cnt,
                                                  int *status) {
  pdl_wait(); /* launched after the previous stage with launch_pdl */
  if (status && blockIdx.x == 0 && threadIdx.x == 0) {
    status[0] = cnt[0]; /* fallback rows + columns, counted by k_row_stats */
    status[1] = cnt[1]; /* error code of the tensor-core launches */
  }
  if (cnt[0] == 0) return; /* nothing flagged: the common case ends here */
  /* blocks of 8 rows x 32 columns of C, strided over a one-wave grid */
  const size_t tj = (n + 31) / 32, nblk = tj * ((m + 7) / 8);
  for (size_t b = blockIdx.x; b < nblk; b += gridDim.x) {
    const size_t i = (b / tj) * 8 + (threadIdx.x >> 5);
    const size_t j = (b % tj) * 32u + (threadIdx.x & 31u);
    if (i >= m || j >= n) continue;
    if (!rowF[i] && !colF[j]) continue;
    fallback_entry<N, CPLX>(i, j, K, A, lda, B, ldb, C, ldc);
  }
}
/* the counters and column statistics every call starts from (one launch in
 * place of four memsets, so the whole chain is kernel to kernel) */
static __global__ void __launch_bounds__(256) k_exact_init(int *cnt, int *tf, size_t ntf, int32_t *colE, int32_t *colEmin,
                                                   size_t n) {
  pdl_wait();
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t0 < 4) cnt[t0] = 0;
  for (size_t i = t0; i < ntf; i += stride) tf[i] = 0;
  for (size_t j = t0; j < n; j += stride) {
    colE[j] = kColNone;
    colEmin[j] = kColMinNone;
  }
}

template <int N, int XL, bool CPLX>
static int run_impl(const Plan &p, const uint8_t *A, size_t lda, const uint8_t *B, size_t ldb, uint8_t *C,
                    size_t ldc, uint8_t *ws, int *n_fallback, cudaStream_t st) {
  int32_t *rowE = (int32_t *)(ws + p.off_rowE), *colE = (int32_t *)(ws + p.off_colE);
  uint8_t *rowF = ws + p.off_flags, *colF = ws + p.off_flags + p.m;
  int *cnt = (int *)(ws + p.off_cnt); /* [0] fallback rows+cols, [1] kernel error code, [2] marked tiles */
  int8_t *Asl = (int8_t *)(ws + p.off_asl), *Bsl = (int8_t *)(ws + p.off_bsl);
  int32_t *D = (int32_t *)(ws + p.off_d);
  RoundPass rp;
  rp.dplane = p.dplane;
  rp.d_first = p.d0;
  rp.cert = p.cert;
  rp.flagged_only = 0;
  rp.nt = p.nt;
  rp.ef = ws + p.off_ef;
  rp.tf = (int *)(ws + p.off_tf);
  rp.tiles = (int *)(ws + p.off_tiles);
  rp.ntiles = cnt + 2;
  /* every stage after the first is launched with launch_pdl: it is scheduled
   * while the previous one finishes and waits for it in pdl_wait() */
  int32_t *colEmin = (int32_t *)(ws + p.off_colEmin);
  {
    const size_t ntf = (size_t)p.mt * p.nt, most = ntf > (size_t)p.n ? ntf : (size_t)p.n;
    const int g = (int)std::min<size_t>((most + 255) / 256 + 1, (size_t)4 * sm_count());
    k_exact_init<<<g, 256, 0, st>>>(cnt, rp.tf, ntf, colE, colEmin, (size_t)p.n);
  }
  if (launch_status() != MPB_OK) return MPB_ERR_CUDA;
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t r) {
    if (r != cudaSuccess && e == cudaSuccess) e = r;
  };
  profile_mark(kPhaseStats, true, st);
  chk(launch_pdl(k_col_stats<N, CPLX>, dim3((p.n + 31) / 32, (p.k + kColRows - 1) / kColRows), dim3(256), 0, st,
                 p.n, p.k, B, ldb, colE, colEmin));
  /* one block per row of A; the column finalisation strides over the grid */
  chk(launch_pdl(k_row_stats<N, CPLX>, dim3(p.m), dim3(kRowWarps * 32), 0, st, p.m, p.k, A, lda, p.SP, rowE, rowF,
                 p.n, colE, (const int32_t *)colEmin, colF, cnt));
  profile_mark(kPhaseStats, false, st);
  profile_mark(kPhaseSlice, true, st);
  chk(launch_pdl(k_slice_a<N, XL, CPLX>, dim3(grid_for(k_slice_a<N, XL, CPLX>, 128, (size_t)p.m * p.kp / slice_geo<N, CPLX>::E)), dim3(128),
                 0, st, p.m, p.k, p.kp, A, lda, p.SP, p.S, (const int32_t *)rowE, (const uint8_t *)rowF, Asl));
  chk(launch_pdl(k_slice_b<N, XL, CPLX>, dim3(grid_for(k_slice_b<N, XL, CPLX>, 128, (size_t)p.n * p.kp / slice_geo<N, CPLX>::E)), dim3(128),
                 0, st, p.n, p.k, p.kp, B, ldb, p.SP, p.S, (const int32_t *)colE, (const uint8_t *)colF, Bsl));
  profile_mark(kPhaseSlice, false, st);
  if (e != cudaSuccess || launch_status() != MPB_OK) return MPB_ERR_CUDA;

  /* main pass: diagonals [d0, 2S-2] of every tile */
  {
    const int rc = launch_diag_gemm(p, Asl, Bsl, D, cnt + 1, p.d0, 2 * p.S - 2, nullptr, nullptr, st);
    if (rc != MPB_OK) return rc;
  }
  auto round_pass = [&](const RoundPass &r, int grid_cap) {
    const int32_t *Dc = D, *rE = rowE, *cE = colE;
    const uint8_t *rF = rowF, *cF = colF;
    const int nl = 2 * p.S - 1 - r.d_first;
    constexpr int TT = round_geo<N, XL>::template threads<CPLX>();
    const size_t stage_bytes = (size_t)p.nprod * nl * TT * 4;
    CUtensorMap tmD;
    /* shared-memory stage of the TMA rounding pass, at most: measured on B200,
     * a 37 KB stage (real 1024^3 at 512 bits, 72 planes) took the pass from
     * 133.7 to 95.7 us, a 61 KB one (complex 512^3 at 256 bits, 3 x 40
     * planes, two blocks per SM) from 43.2 to 54.0 us, and in chunks of 64
     * entries (30 KB, five blocks per SM) to 51.8 us, so larger stages keep
     * the kernel that loads its planes itself */
    constexpr size_t kStageMax = 48 * 1024;
    if (p.P == 1 && !r.flagged_only && nl <= round_geo<N, XL>::J && nl <= 256 && stage_bytes <= kStageMax &&
        make_plane_tmap(&tmD, D + (size_t)r.d_first * r.dplane, (size_t)p.m * p.n, nl, p.nprod, r.dplane,
                        (size_t)(2 * p.S - 1) * r.dplane, TT)) {
      /* planes staged in shared memory by TMA (the first pass of the usual sizes) */
      auto kern = k_exact_round_tma<N, XL, CPLX>;
      const int dsm = (int)stage_bytes + 128;
      /* the opt-in for the largest stage, once per device (the 48 KB default
       * covers static and dynamic shared memory together) */
      static std::atomic<unsigned long long> smem_set{0};
      int dev = 0;
      chk(cudaGetDevice(&dev));
      if (dev >= 0 && dev < 64 && !((smem_set.load(std::memory_order_acquire) >> dev) & 1ull)) {
        const cudaError_t ra =
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStageMax + 128);
        chk(ra);
        if (ra == cudaSuccess) smem_set.fetch_or(1ull << dev, std::memory_order_acq_rel);
      }
      int per = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, TT, dsm) != cudaSuccess || per < 1) per = 1;
      const size_t chunks = ((size_t)p.m * p.n + TT - 1) / TT;
      const int g = (int)std::min(chunks, (size_t)per * sm_count());
      chk(launch_pdl(kern, dim3(g), dim3(TT), (size_t)dsm, st, tmD, p.m, p.n, p.SP, rE, cE, rF, cF, C, ldc, r, nl,
                     (long long)sm100::kWaitNs, cnt + 1));
    } else if (p.P == 1 && !r.flagged_only && nl <= round_geo<N, XL>::J) {
      constexpr int T = round_geo<N, XL>::template threads<CPLX>();
      const int g = std::min(grid_cap, grid_for(k_exact_round<N, XL, CPLX>, T, (size_t)p.m * p.n));
      chk(launch_pdl(k_exact_round<N, XL, CPLX>, dim3(g), dim3(T), 0, st, p.m, p.n, p.S, p.SP, Dc, rE, cE, rF, cF,
                     C, ldc, r));
    } else {
      const int g = std::min(grid_cap, grid_for(k_exact_round_parts<N, XL, CPLX>, 128, (size_t)p.m * p.n));
      chk(launch_pdl(k_exact_round_parts<N, XL, CPLX>, dim3(g), dim3(128), 0, st, p.m, p.n, p.S, p.SP, p.P, Dc, rE,
                     cE, rF, cF, C, ldc, r));
    }
  };
  profile_mark(kPhaseRound, true, st);
  round_pass(rp, 1 << 30);
  profile_mark(kPhaseRound, false, st);
  if (p.d0 > 0) {
    /* tiles holding an entry that did not certify: low diagonals on the
     * tensor cores, then the full sum for those entries (the tile count is
     * read on the device; with no marked tile both launches return at once) */
    const int rc = launch_diag_gemm(p, Asl, Bsl, D, cnt + 1, 0, p.d0 - 1, rp.tiles, rp.ntiles, st);
    if (rc != MPB_OK) return rc;
    RoundPass r2 = rp;
    r2.d_first = 0;
    r2.cert = -1;
    r2.flagged_only = 1;
    round_pass(r2, 4 * sm_count());
  }
  profile_mark(kPhaseFallback, true, st);
  const size_t fb_blocks = (size_t)((p.n + 31) / 32) * ((p.m + 7) / 8);
  chk(launch_pdl(k_fallback<N, CPLX>, dim3((unsigned)std::max<size_t>(1, std::min(fb_blocks, (size_t)2 * sm_count()))), dim3(256), 0, st,
                 (size_t)p.m, (size_t)p.n, (size_t)p.k, A, lda, B, ldb, C, ldc, (const uint8_t *)rowF, (const uint8_t *)colF,
                 (const int *)cnt, n_fallback));
  profile_mark(kPhaseFallback, false, st);
  if (e != cudaSuccess) return MPB_ERR_CUDA;
  return launch_status();
}

template <int N, int XL>
int run_exact(const Plan &p, const uint8_t *A, size_t lda, const uint8_t *B, size_t ldb, uint8_t *C,
                     size_t ldc, uint8_t *ws, int *n_fallback, cudaStream_t st) {
  if (p.cplx) return run_impl<N, XL, true>(p, A, lda, B, ldb, C, ldc, ws, n_fallback, st);
  return run_impl<N, XL, false>(p, A, lda, B, ldb, C, ldc, ws, n_fallback, st);
}

/* one precision, any spread budget (instantiated in exact_gemm_pb<32N>.cu) */
template <int N>
int run_exact_n(const Plan &p, const uint8_t *A, size_t lda, const uint8_t *B, size_t ldb, uint8_t *C, size_t ldc,
                uint8_t *ws, int *n_fallback, cudaStream_t st) {
  switch (p.XL) {
    case 1:
      return run_exact<N, 1>(p, A, lda, B, ldb, C, ldc, ws, n_fallback, st);
    case 2:
      return run_exact<N, 2>(p, A, lda, B, ldb, C, ldc, ws, n_fallback, st);
    case 4:
      return run_exact<N, 4>(p, A, lda, B, ldb, C, ldc, ws, n_fallback, st);
    default:
      return MPB_ERR_ARG;
  }
}

#define MPB_EXACT_DECLARE(N)                                                                                    \
  extern template int run_exact_n<N>(const Plan &, const uint8_t *, size_t, const uint8_t *, size_t, uint8_t *, \
                                     size_t, uint8_t *, int *, cudaStream_t);
MPB_EXACT_DECLARE(2)
MPB_EXACT_DECLARE(4)
MPB_EXACT_DECLARE(8)
MPB_EXACT_DECLARE(16)
MPB_EXACT_DECLARE(32)
MPB_EXACT_DECLARE(64)

} /* namespace exact */
} /* namespace mpb */

#endif /* MPB_EXACT_GEMM_CUH */
