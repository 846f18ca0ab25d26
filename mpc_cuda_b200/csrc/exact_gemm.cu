/* exact_gemm.cu -- exact-accumulation GEMM on the INT8 tensor cores.
 *
 *   C[i,j] = RNDN( sum_k A[i,k] * B[k,j] )      one rounding per entry
 *
 * i.e. the correctly rounded dot product (MPFR mpfr_dot semantics), computed
 * without any floating-point step:
 *
 * 1. Alignment.  Row i of A gets the exponent E_i = max_k exp(A[i,k]); every
 *    entry becomes the exact integer V_ik = +-M_ik * 2^(SP - (E_i - e_ik)) so
 *    that A[i,k] = V_ik * 2^(E_i - PB - SP).  Columns of B likewise (F_j).
 *    SP is the spread budget: an entry more than SP bits below its row's top
 *    would need more bits, so such rows (columns) are flagged and computed by
 *    the fallback (the plain per-operation-rounded kernel), and counted.
 * 2. Slicing.  V (|V| < 2^(8S-2)) is written as S balanced signed base-256
 *    digits in [-128, 127]:  V = sum_s d_s 256^s.  Digit planes are stored
 *    K-major, A_sl[s][i][k], B_sl[s][j][k] (B transposed through shared memory).
 * 3. Tensor cores.  With digits, sum_k V_ik W_kj = sum_d 256^d D_d where
 *    D_d[i,j] = sum_{s+t=d} sum_k a_s[i,k] b_t[k,j]  -- for each diagonal d an
 *    int8 GEMM over the concatenated (s, k) dimension.  |D_d| < pairs*k*2^14
 *    < 2^31 (k is split into parts when needed), so int32 TMEM accumulation
 *    is exact.  A persistent warp-specialised kernel runs one (128x256 output
 *    tile, diagonal, k-part) unit at a time: TMA (128B swizzle, no multicast)
 *    into a 4-stage shared-memory ring, one thread issuing
 *    tcgen05.mma.cta_group::1.kind::i8 (M=128, N=256, K=32), two 256-column
 *    TMEM accumulators so the epilogue warps drain one unit (tcgen05.ld ->
 *    int32 planes in global memory) while the next accumulates.
 * 4. Rounding.  Per output, sum_d 256^d D_d is formed exactly in int64
 *    carry-save words, carried into 32-bit limbs, normalised and rounded once
 *    (RNDN) to PB bits with exponent E_i + F_j - 2PB - 2SP + msb + 1.
 *
 * Work: 2*m*n*k*S^2 int8 operations (S = ceil((PB+SP+2)/8); S = 69 at PB=512
 * with a 32-bit spread budget).  Scratch (caller-provided workspace,
 * mpb_gemm_exact_workspace): digit planes S*(m+n)*kp bytes and the diagonal
 * planes P*(2S-1)*m*n*4 bytes.
 */
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
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
constexpr size_t kSmemBytes = 1024 /* alignment slack */ + STAGES * (A_STAGE + B_STAGE) + 256 /* barriers */;

/* the per-call geometry (host and device) */
struct Plan {
  int prec, N, S, SP, XL;
  int m, n, k, kp, KC; /* kp = k padded to BK, KC = kp / BK chunks */
  int P, cpp;          /* k-parts per diagonal, chunks per part */
  int mt, nt;          /* tiles */
  long units;
  size_t off_rowE, off_colE, off_flags, off_cnt, off_asl, off_bsl, off_d, total;
};

static inline size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

static bool make_plan(int prec, size_t m, size_t n, size_t k, int sp_bits, Plan &p) {
  if (sp_bits < 0 || sp_bits > 1024) return false;
  p.prec = prec;
  p.N = prec / 32;
  p.S = (prec + sp_bits + 2 + 7) / 8;
  p.SP = 8 * p.S - prec - 2;
  const int extra_bits = 8 * p.S - prec;
  int xl = (extra_bits + 31) / 32;
  p.XL = xl <= 1 ? 1 : xl <= 2 ? 2 : xl <= 4 ? 4 : xl <= 8 ? 8 : xl <= 16 ? 16 : xl <= 33 ? 33 : -1;
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
  p.mt = (int)((m + BM - 1) / BM);
  p.nt = (int)((n + BN - 1) / BN);
  p.units = (long)(2 * p.S - 1) * p.mt * p.nt * p.P;
  size_t o = 0;
  p.off_rowE = o;
  o = up256(o + 4 * m);
  p.off_colE = o;
  o = up256(o + 4 * n);
  p.off_flags = o; /* m row flags then n column flags, one byte each */
  o = up256(o + m + n);
  p.off_cnt = o;
  o = up256(o + 16);
  p.off_asl = o;
  o = up256(o + (size_t)p.S * m * p.kp);
  p.off_bsl = o;
  o = up256(o + (size_t)p.S * n * p.kp);
  p.off_d = o;
  o = up256(o + (size_t)p.P * (2 * p.S - 1) * m * n * 4);
  p.total = o;
  return true;
}

/* ------------------------------------------------------------------ *
 * 1. exponent statistics
 * ------------------------------------------------------------------ */
/* one warp per row of A: E_i = max exponent of the nonzero entries; flag the
 * row when some nonzero entry lies more than SP bits below E_i */
template <int N>
__global__ void __launch_bounds__(256) k_row_stats(int m, int k, const uint8_t *A, size_t lda, int SP, int32_t *rowE,
                                                   uint8_t *rowF, int *count) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= m) return;
  int32_t emax = kExpZero, emin = 0x7fffffff;
  const uint8_t *row = A + (size_t)warp * (lda / 32) * sol<N>::kTileBytes;
  for (int k0 = 0; k0 < k; k0 += 32) {
    const int kk = k0 + lane;
    if (kk < k) {
      const uint32_t h = __ldg((const uint32_t *)(row + (size_t)(k0 / 32) * sol<N>::kTileBytes + sol<N>::kHeadOff) + lane);
      if (h != kHeadZero) {
        const int32_t e = head_exp(h);
        emax = max(emax, e);
        emin = min(emin, e);
      }
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    emax = max(emax, __shfl_xor_sync(0xffffffffu, emax, o));
    emin = min(emin, __shfl_xor_sync(0xffffffffu, emin, o));
  }
  if (lane == 0) {
    rowE[warp] = emax;
    const bool flag = emax != kExpZero && (long)emax - emin > SP;
    rowF[warp] = flag ? 1 : 0;
    if (flag) atomicAdd(count, 1);
  }
}
/* column statistics of B (k x n): block = 32 columns x 8 row groups */
template <int N>
__global__ void __launch_bounds__(256) k_col_stats(int n, int k, const uint8_t *B, size_t ldb, int SP, int32_t *colE,
                                                   uint8_t *colF, int *count) {
  __shared__ int32_t smax[8][32], smin[8][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int j = blockIdx.x * 32 + lane;
  int32_t emax = kExpZero, emin = 0x7fffffff;
  const size_t tiles_per_row = ldb / 32;
  for (int kk = w; kk < k; kk += 8) {
    const uint8_t *t = B + ((size_t)kk * tiles_per_row + blockIdx.x) * sol<N>::kTileBytes;
    const uint32_t h = __ldg((const uint32_t *)(t + sol<N>::kHeadOff) + lane);
    if (h != kHeadZero) {
      const int32_t e = head_exp(h);
      emax = max(emax, e);
      emin = min(emin, e);
    }
  }
  smax[w][lane] = emax;
  smin[w][lane] = emin;
  __syncthreads();
  if (w == 0) {
    for (int q = 1; q < 8; ++q) {
      emax = max(emax, smax[q][lane]);
      emin = min(emin, smin[q][lane]);
    }
    if (j < n) {
      colE[j] = emax;
      const bool flag = emax != kExpZero && (long)emax - emin > SP;
      colF[j] = flag ? 1 : 0;
      if (flag) atomicAdd(count, 1);
    }
  }
}

/* ------------------------------------------------------------------ *
 * 2. slicing into balanced base-256 digits
 * ------------------------------------------------------------------ */
/* Digits of V = (-1)^neg * M * 2^sh, M the N-limb significand, 0 <= sh <= SP.
 * L = N + XL limbs hold M << sh; digit s = byte s of |V| balanced into
 * [-128, 127] (positive V) or [-127, 128] then negated (negative V).  Calls
 * put(s, digit) for s < S. */
template <int N, int XL, typename F>
__device__ __forceinline__ void digits_of(const fval<N> &x, int32_t Erow, int SP, int S, F put) {
  constexpr int L = N + XL;
  uint32_t w[L];
  const bool zero = is_zero(x);
  const uint32_t sh = zero ? 0u : (uint32_t)(SP - (Erow - x.e));
  const uint32_t q = sh >> 5, r = sh & 31u;
  /* w = M << sh: limb shift q (< XL + 1 by construction) via a select network */
#pragma unroll
  for (int i = 0; i < L; ++i) w[i] = (i < N) ? x.m[i] : 0u;
#pragma unroll
  for (int b = 0; (1 << b) <= XL; ++b) {
    const int s = 1 << b;
    const bool on = (q >> b) & 1u;
#pragma unroll
    for (int i = L - 1; i >= 0; --i) {
      const uint32_t src = (i - s >= 0) ? w[i - s] : 0u;
      w[i] = on ? src : w[i];
    }
  }
#pragma unroll
  for (int i = L - 1; i > 0; --i) w[i] = fshl(w[i - 1], w[i], r);
  w[0] <<= r;
  const uint32_t thr = x.s ? 129u : 128u;
  uint32_t carry = 0;
#pragma unroll
  for (int s = 0; s < 4 * L; ++s) {
    const uint32_t byte = zero ? 0u : ((w[s >> 2] >> (8 * (s & 3))) & 0xffu);
    const uint32_t t = byte + carry;
    const int d = (t >= thr) ? (int)t - 256 : (int)t;
    carry = (t >= thr) ? 1u : 0u;
    if (s < S) put(s, (int8_t)(x.s ? -d : d));
  }
}

/* A (m x k, tiles) -> A_sl[s][i][kp]; thread per (i, kk), kk < kp (zero padding) */
template <int N, int XL>
__global__ void __launch_bounds__(128) k_slice_a(int m, int k, int kp, const uint8_t *A, size_t lda, int SP, int S,
                                                 const int32_t *rowE, const uint8_t *rowF, int8_t *Asl) {
  const size_t total = (size_t)m * kp, plane = (size_t)m * kp;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx / kp), kk = (int)(idx % kp);
    fval<N> x;
    if (kk < k && !rowF[i]) {
      load_elem<N>(x, A, (size_t)i * lda + kk);
    } else {
      set_zero(x);
    }
    const int32_t E = rowE[i];
    int8_t *dst = Asl + (size_t)i * kp + kk;
    digits_of<N, XL>(x, E, SP, S, [&](int s, int8_t d) { dst[(size_t)s * plane] = d; });
  }
}

/* B (k x n, tiles) -> B_sl[s][j][kp], transposed through shared memory:
 * block = 32 columns (one tile) x 32 rows of B; digits staged per 32-plane
 * chunk as [s][j][32 bytes of k], written out as 32-byte row segments. */
template <int N, int XL>
__global__ void __launch_bounds__(256) k_slice_b(int n, int k, int kp, const uint8_t *B, size_t ldb, int SP, int S,
                                                 const int32_t *colE, const uint8_t *colF, int8_t *Bsl) {
  constexpr int CH = 32; /* digit planes per chunk */
  __shared__ __align__(16) int8_t st[CH][32][32 + 16];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int j0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  const int j = j0 + lane;
  const size_t plane = (size_t)n * kp;
  fval<N> x[4];
  int32_t E = (j < n) ? colE[j] : kExpZero;
  const bool skip = (j >= n) || colF[j];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int kk = k0 + w + 8 * r;
    if (kk < k && !skip)
      load_elem<N>(x[r], B, (size_t)kk * ldb + j);
    else
      set_zero(x[r]);
  }
  for (int c0 = 0; c0 < S; c0 += CH) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int kl = w + 8 * r;
      digits_of<N, XL>(x[r], E, SP, S, [&](int s, int8_t d) {
        if (s >= c0 && s < c0 + CH) st[s - c0][lane][kl] = d;
      });
    }
    __syncthreads();
    /* write: for each plane s and column jl, 32 bytes of k (two uint4) */
    const int nplanes = min(CH, S - c0);
    for (int t = threadIdx.x; t < nplanes * 32 * 2; t += blockDim.x) {
      const int half = t & 1, jl = (t >> 1) & 31, s = t >> 6;
      if (j0 + jl < n && k0 + 16 * half < kp) {
        const uint4 v = *(const uint4 *)&st[s][jl][16 * half];
        *(uint4 *)(Bsl + (size_t)(c0 + s) * plane + (size_t)(j0 + jl) * kp + k0 + 16 * half) = v;
      }
    }
    __syncthreads();
  }
}

/* ------------------------------------------------------------------ *
 * 3. the tcgen05 diagonal GEMM
 * ------------------------------------------------------------------ */
struct GemmArgs {
  int S, mt, nt, P, cpp, KC, m, n;
  long units;
  int32_t *D; /* [P][2S-1][m][n] */
  int *err;
};

struct Unit {
  int d, ti, tj, part, s_lo, s_hi, kc0, kc1;
};
/* units ordered by decreasing diagonal length (longest first) */
__device__ __forceinline__ Unit decode(const GemmArgs &g, long u) {
  Unit x;
  const long per = (long)g.mt * g.nt * g.P;
  const int r = (int)(u / per);
  const long rem = u % per;
  const int tile = (int)(rem / g.P);
  x.part = (int)(rem % g.P);
  const int q = (r + 1) / 2;
  x.d = (r == 0) ? g.S - 1 : ((r & 1) ? g.S - 1 - q : g.S - 1 + q);
  x.ti = tile / g.nt;
  x.tj = tile % g.nt;
  x.s_lo = max(0, x.d - g.S + 1);
  x.s_hi = min(x.d, g.S - 1);
  x.kc0 = x.part * g.cpp;
  x.kc1 = min(x.kc0 + g.cpp, g.KC);
  return x;
}

__global__ void __launch_bounds__(kGemmThreads, 1)
    k_diag_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmArgs g) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t *sA = smem;
  uint8_t *sB = smem + STAGES * A_STAGE;
  uint64_t *bars = (uint64_t *)(sB + STAGES * B_STAGE);
  uint64_t *full = bars, *empty = bars + STAGES, *tfull = bars + 2 * STAGES, *tempty = bars + 2 * STAGES + 2;
  uint64_t *done = bars + 2 * STAGES + 4; /* all MMAs of this CTA retired */
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int s = 0; s < STAGES; ++s) {
      sm100::mbar_init(&full[s], 1);
      sm100::mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      sm100::mbar_init(&tfull[a], 1);
      sm100::mbar_init(&tempty[a], 4);
    }
    sm100::mbar_init(done, 1);
    sm100::fence_barrier_init();
  }
  if (warp == 1) {
    sm100::tmem_alloc(&tmem_base, 512);
    sm100::tmem_relinquish();
  }
  if (warp == 0 && lane == 0) {
    sm100::prefetch_tmap(&tmA);
    sm100::prefetch_tmap(&tmB);
  }
  sm100::tc_fence_before();
  __syncthreads();
  sm100::tc_fence_after();
  const uint32_t tbase = tmem_base;

  auto fail = [&](int code) {
    abort_flag = 1;
    atomicCAS(g.err, 0, code);
  };

  if (warp == 0) {
    /* ---------------- TMA producer ---------------- */
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      for (long u = blockIdx.x; u < g.units && !abort_flag; u += gridDim.x) {
        const Unit x = decode(g, u);
        for (int s = x.s_lo; s <= x.s_hi && !abort_flag; ++s) {
          const int t = x.d - s;
          for (int kc = x.kc0; kc < x.kc1; ++kc) {
            if (!sm100::mbar_wait(&empty[stage], phase ^ 1u, &abort_flag)) {
              fail(1);
              break;
            }
            sm100::mbar_arrive_expect_tx(&full[stage], A_STAGE + B_STAGE);
            sm100::tma_load_3d(sA + stage * A_STAGE, &tmA, kc * BK, x.ti * BM, s, &full[stage]);
            sm100::tma_load_3d(sB + stage * B_STAGE, &tmB, kc * BK, x.tj * BN, t, &full[stage]);
            if (++stage == STAGES) {
              stage = 0;
              phase ^= 1u;
            }
          }
        }
      }
      /* drain: wait until every issued stage has been consumed (bounded) */
      for (int q = 0; q < STAGES && !abort_flag; ++q) {
        if (!sm100::mbar_wait(&empty[stage], phase ^ 1u, &abort_flag)) break;
        if (++stage == STAGES) {
          stage = 0;
          phase ^= 1u;
        }
      }
    }
  } else if (warp == 1) {
    /* ---------------- MMA issuer ---------------- */
    if (lane == 0) {
      constexpr uint32_t idesc = sm100::idesc_i8(BM, BN);
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t aphase = 0;
      for (long u = blockIdx.x; u < g.units && !abort_flag; u += gridDim.x) {
        const Unit x = decode(g, u);
        if (!sm100::mbar_wait(&tempty[acc], aphase ^ 1u, &abort_flag)) {
          fail(2);
          break;
        }
        sm100::tc_fence_after();
        const uint32_t tacc = tbase + (uint32_t)(acc * BN);
        uint32_t accumulate = 0;
        bool ok = true;
        for (int s = x.s_lo; s <= x.s_hi && ok; ++s) {
          for (int kc = x.kc0; kc < x.kc1; ++kc) {
            if (!sm100::mbar_wait(&full[stage], phase, &abort_flag)) {
              fail(3);
              ok = false;
              break;
            }
            sm100::tc_fence_after();
            const uint32_t a0 = sm100::smem_u32(sA + stage * A_STAGE);
            const uint32_t b0 = sm100::smem_u32(sB + stage * B_STAGE);
#pragma unroll
            for (int kk = 0; kk < BK / 32; ++kk) {
              sm100::mma_i8(tacc, sm100::sdesc_k128(a0 + 32u * kk), sm100::sdesc_k128(b0 + 32u * kk), idesc,
                            accumulate);
              accumulate = 1;
            }
            sm100::mma_commit(&empty[stage]);
            if (++stage == STAGES) {
              stage = 0;
              phase ^= 1u;
            }
          }
        }
        if (!ok) break;
        sm100::mma_commit(&tfull[acc]);
        if (++acc == 2) {
          acc = 0;
          aphase ^= 1u;
        }
      }
      /* tensor memory is freed below: wait (bounded) for every MMA issued */
      sm100::mma_commit(done);
      volatile int never = 0;
      sm100::mbar_wait(done, 0, &never);
    }
  } else {
    /* ---------------- epilogue: TMEM -> int32 diagonal planes ---------------- */
    const int q = warp & 3; /* TMEM lane quarter this warp may access */
    int acc = 0;
    uint32_t aphase = 0;
    for (long u = blockIdx.x; u < g.units; u += gridDim.x) {
      /* tcgen05.ld is warp-collective: lane 0 waits and decides for the warp */
      int ok = 1;
      if (lane == 0) ok = (!abort_flag && sm100::mbar_wait(&tfull[acc], aphase, &abort_flag)) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0) fail(4);
        break;
      }
      const Unit x = decode(g, u);
      sm100::tc_fence_after();
      const int row = x.ti * BM + q * 32 + lane;
      int32_t *drow = g.D + (((size_t)x.part * (2 * g.S - 1) + x.d) * g.m + (size_t)row) * g.n;
      const uint32_t tacc = tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * BN);
#pragma unroll 1
      for (int c = 0; c < BN / 32; ++c) {
        uint32_t v[32];
        sm100::tmem_ld32(tacc + 32u * c, v);
        sm100::tmem_ld_wait();
        const int col0 = x.tj * BN + 32 * c;
        if (row < g.m) {
          if (col0 + 32 <= g.n && (g.n & 3) == 0) {
#pragma unroll
            for (int e = 0; e < 32; e += 4)
              *(uint4 *)(drow + col0 + e) = make_uint4(v[e], v[e + 1], v[e + 2], v[e + 3]);
          } else {
#pragma unroll
            for (int e = 0; e < 32; ++e)
              if (col0 + e < g.n) drow[col0 + e] = (int32_t)v[e];
          }
        }
      }
      sm100::tc_fence_before();
      __syncwarp();
      if (lane == 0) sm100::mbar_arrive(&tempty[acc]);
      if (++acc == 2) {
        acc = 0;
        aphase ^= 1u;
      }
    }
  }

  sm100::tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    sm100::tc_fence_after();
    sm100::tmem_dealloc(tbase, 512);
  }
}

/* ------------------------------------------------------------------ *
 * 4. exact recombination and the single rounding
 * ------------------------------------------------------------------ */
/* Q 32-bit words cover sum_d 256^d D_d: 8(2S-2) + 31 + log2(P) + sign bits */
template <int N, int XL>
struct round_geo {
  static constexpr int SMAX = 4 * (N + XL);
  static constexpr int Q = (8 * (2 * SMAX - 2) + 31 + 8 + 31) / 32 + 1;
};

template <int N, int XL>
__global__ void __launch_bounds__(128) k_exact_round(int m, int n, int S, int SP, int P, const int32_t *D,
                                                     const int32_t *rowE, const int32_t *colE, const uint8_t *rowF,
                                                     const uint8_t *colF, uint8_t *C, size_t ldc) {
  constexpr int Q = round_geo<N, XL>::Q;
  constexpr int W = Q; /* window for normalisation */
  const size_t total = (size_t)m * n;
  const size_t plane = (size_t)m * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx / n), j = (int)(idx % n);
    if (rowF[i] || colF[j]) continue; /* computed by the fallback */
    long long acc[Q];
#pragma unroll
    for (int w = 0; w < Q; ++w) acc[w] = 0;
    for (int p = 0; p < P; ++p) {
      const int32_t *dp = D + (size_t)p * (2 * S - 1) * plane + idx;
      /* diagonal d adds D_d * 2^(8d) = D_d * 2^(8(d&3)) at word d>>2 */
#pragma unroll
      for (int d = 0; d < 2 * round_geo<N, XL>::SMAX - 1; ++d) {
        if (d < 2 * S - 1) acc[d >> 2] += (long long)__ldg(dp + (size_t)d * plane) << (8 * (d & 3));
      }
    }
    /* carry into 32-bit two's complement words */
    uint32_t v[W];
    long long carry = 0;
#pragma unroll
    for (int w = 0; w < Q; ++w) {
      const long long t = acc[w] + carry;
      v[w] = (uint32_t)t;
      carry = t >> 32;
    }
    const uint32_t neg = v[Q - 1] >> 31;
    if (neg) {
      uint32_t c = 1;
#pragma unroll
      for (int w = 0; w < Q; ++w) {
        const uint32_t t = ~v[w] + c;
        c = (c && t == 0) ? 1u : 0u;
        v[w] = t;
      }
    }
    /* normalise: leading limb index and bit */
    int lq = W;
    uint32_t top = 0;
#pragma unroll
    for (int w = W - 1; w >= 0; --w) {
      const bool take = (lq == W) && v[w] != 0;
      top = take ? v[w] : top;
      lq = take ? (W - 1 - w) : lq;
    }
    fval<N> r;
    if (lq == W) {
      set_zero(r);
    } else {
      const uint32_t lr = clz32(top) & 31u;
      /* shift left by 32*lq + lr: limb stages then funnel */
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
      /* msb position of the exact integer: 32*W - 1 - (32*lq + lr) */
      const long msb = 32L * W - 1 - (32L * lq + lr);
      const long e = msb + 1 + (long)rowE[i] + colE[j] - 2L * (32 * N) - 2L * SP;
      int32_t ee = (int32_t)e;
      rndn<N>(r.m, ee, g >> 31, st);
      r.e = ee;
      r.s = neg;
    }
    store_elem<N>(C, (size_t)i * ldc + j, r);
  }
}

/* flagged rows / columns: plain sequential-k per-operation rounding */
template <int N>
__global__ void __launch_bounds__(256) k_fallback(size_t m, size_t n, size_t K, const uint8_t *A, size_t lda,
                                                  const uint8_t *B, size_t ldb, uint8_t *C, size_t ldc,
                                                  const uint8_t *rowF, const uint8_t *colF) {
  const size_t i = (size_t)blockIdx.y * 8 + (threadIdx.x >> 5);
  const size_t j = (size_t)blockIdx.x * 32u + (threadIdx.x & 31u);
  if (i >= m || j >= n) return;
  if (!rowF[i] && !colF[j]) return;
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

/* ------------------------------------------------------------------ *
 * host side
 * ------------------------------------------------------------------ */
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  return fn;
}

/* [planes][rows][kp] int8, box = BK x box_rows x 1, 128B swizzle */
static bool make_tmap(CUtensorMap *tm, void *base, int kp, int rows, int planes, int box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)kp, (cuuint64_t)rows, (cuuint64_t)planes};
  const cuuint64_t strides[2] = {(cuuint64_t)kp, (cuuint64_t)kp * rows};
  const cuuint32_t box[3] = {(cuuint32_t)BK, (cuuint32_t)box_rows, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int N, int XL>
static int run_exact(const Plan &p, const uint8_t *A, size_t lda, const uint8_t *B, size_t ldb, uint8_t *C,
                     size_t ldc, uint8_t *ws, int *n_fallback, cudaStream_t st) {
  int32_t *rowE = (int32_t *)(ws + p.off_rowE), *colE = (int32_t *)(ws + p.off_colE);
  uint8_t *rowF = ws + p.off_flags, *colF = ws + p.off_flags + p.m;
  int *cnt = (int *)(ws + p.off_cnt); /* [0] fallback rows+cols, [1] kernel error code */
  int8_t *Asl = (int8_t *)(ws + p.off_asl), *Bsl = (int8_t *)(ws + p.off_bsl);
  int32_t *D = (int32_t *)(ws + p.off_d);
  if (cudaMemsetAsync(cnt, 0, 16, st) != cudaSuccess) return MPB_ERR_CUDA;

  profile_mark(kPhaseStats, true, st);
  k_row_stats<N><<<(p.m + 7) / 8, 256, 0, st>>>(p.m, p.k, A, lda, p.SP, rowE, rowF, cnt);
  k_col_stats<N><<<(p.n + 31) / 32, 256, 0, st>>>(p.n, p.k, B, ldb, p.SP, colE, colF, cnt);
  profile_mark(kPhaseStats, false, st);
  profile_mark(kPhaseSlice, true, st);
  {
    const int g = grid_for(k_slice_a<N, XL>, 128, (size_t)p.m * p.kp);
    k_slice_a<N, XL><<<g, 128, 0, st>>>(p.m, p.k, p.kp, A, lda, p.SP, p.S, rowE, rowF, Asl);
  }
  {
    const dim3 grid((p.n + 31) / 32, p.kp / 32);
    k_slice_b<N, XL><<<grid, 256, 0, st>>>(p.n, p.k, p.kp, B, ldb, p.SP, p.S, colE, colF, Bsl);
  }
  profile_mark(kPhaseSlice, false, st);
  if (launch_status() != MPB_OK) return MPB_ERR_CUDA;

  CUtensorMap tmA, tmB;
  if (!make_tmap(&tmA, Asl, p.kp, p.m, p.S, BM) || !make_tmap(&tmB, Bsl, p.kp, p.n, p.S, BN)) return MPB_ERR_CUDA;
  if (cudaFuncSetAttribute(k_diag_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes) != cudaSuccess)
    return MPB_ERR_CUDA;
  GemmArgs ga;
  ga.S = p.S;
  ga.mt = p.mt;
  ga.nt = p.nt;
  ga.P = p.P;
  ga.cpp = p.cpp;
  ga.KC = p.KC;
  ga.m = p.m;
  ga.n = p.n;
  ga.units = p.units;
  ga.D = D;
  ga.err = cnt + 1;
  const long grid = std::min<long>(p.units, (long)sm_count());
  profile_mark(kPhaseTensor, true, st);
  k_diag_gemm<<<(int)grid, kGemmThreads, kSmemBytes, st>>>(tmA, tmB, ga);
  profile_mark(kPhaseTensor, false, st);
  if (launch_status() != MPB_OK) return MPB_ERR_CUDA;

  profile_mark(kPhaseRound, true, st);
  {
    const int g = grid_for(k_exact_round<N, XL>, 128, (size_t)p.m * p.n);
    k_exact_round<N, XL><<<g, 128, 0, st>>>(p.m, p.n, p.S, p.SP, p.P, D, rowE, colE, rowF, colF, C, ldc);
  }
  profile_mark(kPhaseRound, false, st);
  profile_mark(kPhaseFallback, true, st);
  {
    const dim3 grid((p.n + 31) / 32, (p.m + 7) / 8);
    k_fallback<N><<<grid, 256, 0, st>>>(p.m, p.n, p.k, A, lda, B, ldb, C, ldc, rowF, colF);
  }
  profile_mark(kPhaseFallback, false, st);
  if (n_fallback && cudaMemcpyAsync(n_fallback, cnt, 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return MPB_ERR_CUDA;
  return launch_status();
}

} /* namespace exact */
} /* namespace mpb */

using namespace mpb;

#define MPB_EXACT_XL(XL, ...)        \
  switch (XL) {                      \
    case 1: {                        \
      constexpr int XLC = 1;         \
      __VA_ARGS__;                   \
    } break;                         \
    case 2: {                        \
      constexpr int XLC = 2;         \
      __VA_ARGS__;                   \
    } break;                         \
    case 4: {                        \
      constexpr int XLC = 4;         \
      __VA_ARGS__;                   \
    } break;                         \
    default:                         \
      return MPB_ERR_ARG;            \
  }

extern "C" size_t mpb_gemm_exact_workspace(int prec, size_t m, size_t n, size_t k, int sp_bits) {
  exact::Plan p;
  if (!prec_ok(prec) || m == 0 || n == 0 || k == 0 || m > (1u << 24) || n > (1u << 24) || k > (1u << 24))
    return 0;
  if (!exact::make_plan(prec, m, n, k, sp_bits, p) || p.XL > 4) return 0;
  return p.total;
}

extern "C" int mpb_gemm_exact_r(int prec, size_t m, size_t n, size_t k, const void *A, size_t lda, const void *B,
                                size_t ldb, void *C, size_t ldc, int sp_bits, void *workspace, size_t ws_bytes,
                                int *status, void *stream) {
  if (!prec_ok(prec)) return MPB_ERR_PREC;
  if (m == 0 || n == 0) return MPB_OK;
  if (m > (1u << 24) || n > (1u << 24) || k > (1u << 24)) return MPB_ERR_SIZE;
  if (ldc % 32 || ldc < n) return MPB_ERR_LD;
  if (k > 0 && (lda % 32 || lda < k || ldb % 32 || ldb < n)) return MPB_ERR_LD;
  if (!C || (k > 0 && (!A || !B))) return MPB_ERR_NULL;
  if (!aligned16(C) || (k > 0 && (!aligned16(A) || !aligned16(B)))) return MPB_ERR_ALIGN;
  if (k == 0) /* empty sums: +0 everywhere */
    return mpb_gemm_r(prec, m, n, 0, nullptr, 32, nullptr, 32, C, ldc, stream);
  exact::Plan p;
  if (!exact::make_plan(prec, m, n, k, sp_bits, p) || p.XL > 4) return MPB_ERR_ARG;
  if (!workspace || ws_bytes < p.total) return MPB_ERR_WORKSPACE;
  if (((uintptr_t)workspace & 255u) != 0) return MPB_ERR_ALIGN;
  cudaStream_t st = as_stream(stream);
  MPB_DISPATCH_PREC(prec, {
    MPB_EXACT_XL(p.XL, {
      return exact::run_exact<N, XLC>(p, (const uint8_t *)A, lda, (const uint8_t *)B, ldb, (uint8_t *)C, ldc,
                                      (uint8_t *)workspace, status, st);
    });
  });
  return MPB_OK;
}

/* ------------------------------------------------------------------ *
 * Exact GEMM without any allocation.
 *
 * For callers that cannot call cudaMalloc: code that runs after start-up in
 * a latency-critical loop where an allocation (and its implicit device
 * synchronisation) is not allowed, or code inside a framework that owns the
 * whole device memory pool so a foreign cudaMalloc would fail or fragment it.
 * Such callers still pass A, B and C; the scratch the exact GEMM needs (digit
 * planes, diagonal planes, statistics) comes from this fixed area instead of
 * a caller-provided workspace.
 *
 * kStaticScratchBytes (16 MiB) is reserved on every GPU that loads this
 * library, for the life of the process.  Problems whose
 * mpb_gemm_exact_workspace(...) exceeds it are rejected with MPB_ERR_SIZE
 * (e.g. PB=512 up to about 128 x 128 x 128).  Every call shares the area: calls
 * that overlap on the GPU (other streams, other host threads) race and must
 * be serialised by the caller.  The counters that must start at zero are
 * cleared by each call; everything else is overwritten.
 * ------------------------------------------------------------------ */
namespace {
constexpr size_t kStaticScratchBytes = (size_t)16 << 20;
static __device__ __align__(256) uint8_t g_exact_scratch[kStaticScratchBytes];

/* Device address of g_exact_scratch on the current device.  The host-side
 * name is only a stand-in, so the address is looked up once per device (the
 * first call on a device, which should therefore come before any stream
 * capture) with that device current. */
uint8_t *static_scratch() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  static std::once_flag once[64];
  static uint8_t *addr[64];
  std::call_once(once[dev], [dev] {
    void *p = nullptr;
    addr[dev] = (cudaGetSymbolAddress(&p, g_exact_scratch) == cudaSuccess) ? (uint8_t *)p : nullptr;
  });
  return addr[dev];
}
}  // namespace

extern "C" int mpb_gemm_exact_r_static(int prec, size_t m, size_t n, size_t k, const void *A, size_t lda,
                                       const void *B, size_t ldb, void *C, size_t ldc, int sp_bits, int *status,
                                       void *stream) {
  if (!prec_ok(prec)) return MPB_ERR_PREC;
  if (m == 0 || n == 0) return MPB_OK;
  if (m > (1u << 24) || n > (1u << 24) || k > (1u << 24)) return MPB_ERR_SIZE;
  if (ldc % 32 || ldc < n) return MPB_ERR_LD;
  if (k > 0 && (lda % 32 || lda < k || ldb % 32 || ldb < n)) return MPB_ERR_LD;
  if (!C || (k > 0 && (!A || !B))) return MPB_ERR_NULL;
  if (!aligned16(C) || (k > 0 && (!aligned16(A) || !aligned16(B)))) return MPB_ERR_ALIGN;
  if (k == 0) return mpb_gemm_r(prec, m, n, 0, nullptr, 32, nullptr, 32, C, ldc, stream);
  exact::Plan p;
  if (!exact::make_plan(prec, m, n, k, sp_bits, p) || p.XL > 4) return MPB_ERR_ARG;
  if (p.total > kStaticScratchBytes) return MPB_ERR_SIZE; /* larger than the static scratch area */
  uint8_t *ws = static_scratch();
  if (!ws) return MPB_ERR_CUDA;
  cudaStream_t st = as_stream(stream);
  MPB_DISPATCH_PREC(prec, {
    MPB_EXACT_XL(p.XL, {
      return exact::run_exact<N, XLC>(p, (const uint8_t *)A, lda, (const uint8_t *)B, ldb, (uint8_t *)C, ldc, ws,
                                      status, st);
    });
  });
  return MPB_OK;
}
