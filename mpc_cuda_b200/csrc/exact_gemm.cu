/* exact_gemm.cu -- exact-accumulation GEMM on the INT8 tensor cores.
 *
 *   C[i,j] = RNDN( sum_k A[i,k] * B[k,j] )      one rounding per entry
 *
 * i.e. the correctly rounded dot product (MPFR mpfr_dot / MPC mpc_dot
 * semantics), computed without any floating-point step:
 *
 * 1. Alignment.  Row i of A gets the exponent E_i = max_k exp(A[i,k]) (over
 *    real and imaginary parts); every entry becomes the exact integer
 *    V_ik = +-M_ik * 2^(SP - (E_i - e_ik)), so A[i,k] = V_ik * 2^(E_i - PB - SP).
 *    Columns of B likewise (F_j).  SP is the spread budget: an entry more than
 *    SP bits below its row's top would need more bits, so such rows (columns)
 *    are flagged, computed by the fallback (the plain per-operation-rounded
 *    kernel) and counted.
 * 2. Slicing.  V (two's complement, |V| < 2^(8S-2)) is written as S balanced
 *    signed base-256 digits in [-128, 127]: V = sum_s d_s 256^s.  Digit planes
 *    are stored K-major, A_sl[q*S+s][i][k] and B_sl[q*S+s][j][k] (B transposed
 *    through shared memory) for each real product q.  A complex product uses
 *    the 3-multiplication (Gauss) form on exact integers:
 *      T0 = Vr*Wr, T1 = Vi*Wi, T2 = (Vr+Vi)*(Wr+Wi);  re = T0 - T1, im = T2 - T0 - T1
 *    so q runs over {re, im, re+im} (one more bit: S from PB + SP + 3).
 * 3. Tensor cores.  With digits, sum_k V_ik W_kj = sum_d 256^d D_d where
 *    D_d[i,j] = sum_{s+t=d} sum_k a_s[i,k] b_t[k,j]  -- for each diagonal d an
 *    int8 GEMM over the concatenated (s, k) dimension.  |D_d| < pairs*k*2^14
 *    < 2^31 (k is split into parts when needed), so int32 TMEM accumulation
 *    is exact.  A persistent warp-specialised kernel runs one (product,
 *    128x256 output tile, diagonal, k-part) unit at a time, longest diagonals
 *    first: TMA (128B swizzle, no multicast) into a 4-stage shared-memory ring,
 *    one thread issuing tcgen05.mma.cta_group::1.kind::i8 (M=128, N=256,
 *    K=32), two 256-column TMEM accumulators so the epilogue warps drain one
 *    unit (tcgen05.ld -> int32 planes in global memory) while the next
 *    accumulates.
 * 4. Rounding.  Per output (component), the signed combination of the
 *    products' sum_d 256^d D_d is streamed word by word into 32-bit limbs with
 *    an int64 carry, normalised and rounded once (RNDN) to PB bits with
 *    exponent E_i + F_j - 2PB - 2SP + msb + 1.
 * 5. Truncation.  The low diagonals d < d0 only reach the bits far below the
 *    result's ULP, so the main pass skips them (about 40% of the pairs at
 *    PB=512): their sum is bounded, |R| < 2^cert, and the rounding of the
 *    truncated sum is accepted only when no value within 2^cert of it rounds
 *    differently (round_words).  An entry that fails -- heavy cancellation,
 *    or a sum within 2^cert of a rounding midpoint -- marks its output tile;
 *    the tensor cores then compute the low diagonals of the marked tiles only,
 *    and a second rounding pass rounds those entries from the full, exact
 *    sum.  Every entry is therefore still the correctly rounded dot product.
 *
 * This file holds the kernels and the entry points; each precision's
 * instantiations are compiled in their own translation unit
 * (exact_gemm_pb*.cu) so the build runs them in parallel.
 *
 * Work: nprod*2*m*n*k*pairs int8 operations, pairs = the slice pairs on the
 * diagonals [d0, 2S-2] (mpb_gemm_exact_plan_info; S = ceil((PB+SP+2)/8)
 * real, ceil((PB+SP+3)/8) complex; S = 69, d0 = 65, 2616 of S^2 = 4761
 * pairs at PB=512, k=1024 with a 32-bit budget).
 * Scratch (caller-provided workspace, mpb_gemm_exact_workspace /
 * mpb_gemm_exact_c_workspace): digit planes nprod*S*(m+n)*kp bytes and the
 * diagonal planes nprod*P*(2S-1)*m*n*4 bytes.
 */
#include <atomic>

#include "exact_gemm.cuh"

namespace mpb {
namespace exact {

struct Unit {
  int d, q, ti, tj, part, s_lo, s_hi, kc0, kc1;
};
/* unit u of a launch over T tiles: units ordered by decreasing diagonal
 * length (the r-th longest diagonal of [dl, dh], alternating around S-1),
 * then product, tile, k-part */
__device__ __forceinline__ Unit decode(const GemmArgs &g, long u, long T) {
  Unit x;
  const long per = (long)g.nprod * T * g.P;
  const int r = (int)(u / per);
  long rem = u % per;
  x.q = (int)(rem / (T * g.P));
  rem %= T * g.P;
  const long t = rem / g.P;
  x.part = (int)(rem % g.P);
  const int tile = g.tiles ? g.tiles[t] : (int)t;
  const int c = min(max(g.S - 1, g.dl), g.dh);
  const int a = c - g.dl, b = g.dh - c, mm = min(a, b);
  if (r <= 2 * mm)
    x.d = (r == 0) ? c : ((r & 1) ? c - (r + 1) / 2 : c + r / 2);
  else
    x.d = (a > b) ? c - (r - mm) : c + (r - mm);
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
  pdl_wait(); /* launched after the previous stage with launch_pdl */
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
  /* tiles in this launch, and its unit count (a tile list is counted by the
   * previous kernel on the stream) */
  const long T = g.tiles ? (long)*g.ntiles : (long)g.mt * g.nt;
  const long units = g.tiles ? T * g.nprod * (g.dh - g.dl + 1) * g.P : g.units;
  if (units == 0) return; /* an empty recomputation pass: no set-up at all */
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
      uint32_t issued = 0u, iphase = 0u; /* per stage: a load pending on it, and its phase */
      for (long u = blockIdx.x; u < units && !abort_flag; u += gridDim.x) {
        const Unit x = decode(g, u, T);
        for (int s = x.s_lo; s <= x.s_hi && !abort_flag; ++s) {
          const int t = x.d - s;
          for (int kc = x.kc0; kc < x.kc1; ++kc) {
            if (!sm100::mbar_wait(&empty[stage], phase ^ 1u, &abort_flag, g.wait_ns)) {
              fail(1);
              break;
            }
            sm100::mbar_arrive_expect_tx(&full[stage], A_STAGE + B_STAGE);
            issued |= 1u << stage;
            iphase = (iphase & ~(1u << stage)) | (phase << stage);
            sm100::tma_load_3d(sA + stage * A_STAGE, &tmA, kc * BK, x.ti * BM, x.q * g.S + s, &full[stage]);
            sm100::tma_load_3d(sB + stage * B_STAGE, &tmB, kc * BK, x.tj * BN, x.q * g.S + t, &full[stage]);
            if (++stage == STAGES) {
              stage = 0;
              phase ^= 1u;
            }
          }
        }
      }
      /* drain: wait until every issued stage has been consumed (bounded) */
      for (int q = 0; q < STAGES && !abort_flag; ++q) {
        if (!sm100::mbar_wait(&empty[stage], phase ^ 1u, &abort_flag, g.wait_ns)) break;
        if (++stage == STAGES) {
          stage = 0;
          phase ^= 1u;
        }
      }
      if (abort_flag) {
        /* the consumer is gone: wait (bounded) for this CTA's own copies still
         * in flight, so none lands in shared memory after the CTA exits */
        volatile int never = 0;
        for (int s2 = 0; s2 < STAGES; ++s2)
          if ((issued >> s2) & 1u) sm100::mbar_wait(&full[s2], (iphase >> s2) & 1u, &never, g.wait_ns);
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
      for (long u = blockIdx.x; u < units && !abort_flag; u += gridDim.x) {
        const Unit x = decode(g, u, T);
        if (!sm100::mbar_wait(&tempty[acc], aphase ^ 1u, &abort_flag, g.wait_ns)) {
          fail(2);
          break;
        }
        sm100::tc_fence_after();
        const uint32_t tacc = tbase + (uint32_t)(acc * BN);
        uint32_t accumulate = 0;
        bool ok = true;
        for (int s = x.s_lo; s <= x.s_hi && ok; ++s) {
          for (int kc = x.kc0; kc < x.kc1; ++kc) {
            if (!sm100::mbar_wait(&full[stage], phase, &abort_flag, g.wait_ns)) {
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
        if (!(g.inject == 1 && blockIdx.x == 0 && u == 0)) sm100::mma_commit(&tfull[acc]);
        if (++acc == 2) {
          acc = 0;
          aphase ^= 1u;
        }
      }
      /* tensor memory is freed below: wait (bounded) for every MMA issued */
      sm100::mma_commit(done);
      volatile int never = 0;
      sm100::mbar_wait(done, 0, &never, g.wait_ns);
    }
  } else {
    /* ---------------- epilogue: TMEM -> int32 diagonal planes ---------------- */
    const int q = warp & 3; /* TMEM lane quarter this warp may access */
    int acc = 0;
    uint32_t aphase = 0;
    for (long u = blockIdx.x; u < units; u += gridDim.x) {
      /* tcgen05.ld is warp-collective: lane 0 waits and decides for the warp */
      int ok = 1;
      if (lane == 0) ok = (!abort_flag && sm100::mbar_wait(&tfull[acc], aphase, &abort_flag, g.wait_ns)) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0) fail(4);
        break;
      }
      const Unit x = decode(g, u, T);
      sm100::tc_fence_after();
      const int row = x.ti * BM + q * 32 + lane;
      int32_t *drow = g.D + (((size_t)x.q * g.P + x.part) * (2 * g.S - 1) + x.d) * g.dplane + (size_t)row * g.n;
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

bool make_plane_tmap(CUtensorMap *tm, const int32_t *base, size_t entries, int nl, int nprod, size_t plane_elems,
                     size_t q_elems, int box_x) {
  auto fn = encode_fn();
  if (!fn || nl < 1 || nl > 256 || box_x < 4 || box_x > 256) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)entries, (cuuint64_t)nl, (cuuint64_t)nprod};
  const cuuint64_t strides[2] = {(cuuint64_t)plane_elems * 4u, (cuuint64_t)q_elems * 4u};
  const cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)nl, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_INT32, 3, (void *)base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

/* failure-path test: consumed by the next tensor-core launch of the process */
static std::atomic<int> g_inject{0};
static std::atomic<long long> g_inject_wait_ns{0};

int launch_diag_gemm(const Plan &p, int8_t *Asl, int8_t *Bsl, int32_t *D, int *err, int dl, int dh,
                     const int *tiles, const int *ntiles, cudaStream_t st) {
  CUtensorMap tmA, tmB;
  if (!make_tmap(&tmA, Asl, p.kp, p.m, p.nprod * p.S, BM) || !make_tmap(&tmB, Bsl, p.kp, p.n, p.nprod * p.S, BN))
    return MPB_ERR_CUDA;
  /* the shared-memory opt-in, once per device (a call made while a stream is
   * being captured then issues nothing but the launches) */
  static std::atomic<unsigned long long> smem_set{0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return MPB_ERR_CUDA;
  if (!((smem_set.load(std::memory_order_acquire) >> dev) & 1ull)) {
    if (cudaFuncSetAttribute(k_diag_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes) !=
        cudaSuccess)
      return MPB_ERR_CUDA;
    smem_set.fetch_or(1ull << dev, std::memory_order_acq_rel);
  }
  GemmArgs ga;
  ga.S = p.S;
  ga.nprod = p.nprod;
  ga.mt = p.mt;
  ga.nt = p.nt;
  ga.P = p.P;
  ga.cpp = p.cpp;
  ga.KC = p.KC;
  ga.m = p.m;
  ga.n = p.n;
  ga.dplane = p.dplane;
  ga.dl = dl;
  ga.dh = dh;
  ga.units = (long)p.nprod * (dh - dl + 1) * p.mt * p.nt * p.P;
  ga.tiles = tiles;
  ga.ntiles = ntiles;
  ga.D = D;
  ga.err = err;
  ga.inject = g_inject.exchange(0);
  const long long wns = g_inject_wait_ns.exchange(0);
  ga.wait_ns = (ga.inject && wns > 0) ? (uint64_t)wns : sm100::kWaitNs;
  const long grid = std::min<long>(ga.units, (long)sm_count());
  const int phase = tiles ? kPhaseTensorLow : kPhaseTensor;
  profile_mark(phase, true, st);
  const cudaError_t e = launch_pdl(k_diag_gemm, dim3((unsigned)grid), dim3(kGemmThreads), kSmemBytes, st, tmA, tmB, ga);
  profile_mark(phase, false, st);
  if (e != cudaSuccess) return MPB_ERR_CUDA;
  return launch_status();
}

} /* namespace exact */
} /* namespace mpb */

using namespace mpb;

static size_t workspace_bytes(int prec, size_t m, size_t n, size_t k, int sp_bits, int cplx) {
  exact::Plan p;
  if (!prec_ok(prec) || m == 0 || n == 0 || k == 0 || m > (1u << 24) || n > (1u << 24) || k > (1u << 24))
    return 0;
  if (!exact::make_plan(prec, m, n, k, sp_bits, cplx, p)) return 0;
  return p.total;
}

extern "C" size_t mpb_gemm_exact_workspace(int prec, size_t m, size_t n, size_t k, int sp_bits) {
  return workspace_bytes(prec, m, n, k, sp_bits, 0);
}
extern "C" size_t mpb_gemm_exact_c_workspace(int prec, size_t m, size_t n, size_t k, int sp_bits) {
  return workspace_bytes(prec, m, n, k, sp_bits, 1);
}

extern "C" int mpb_gemm_exact_plan_info(int prec, size_t m, size_t n, size_t k, int sp_bits, int cplx, int *slices,
                                        int *first_diag, long long *pairs) {
  if (!prec_ok(prec)) return MPB_ERR_PREC;
  if (m == 0 || n == 0 || k == 0 || m > (1u << 24) || n > (1u << 24) || k > (1u << 24)) return MPB_ERR_SIZE;
  exact::Plan p;
  if (!exact::make_plan(prec, m, n, k, sp_bits, cplx, p)) return MPB_ERR_ARG;
  long long pr = 0;
  for (int d = p.d0; d <= 2 * p.S - 2; ++d) pr += std::min(d, 2 * p.S - 2 - d) + 1;
  if (slices) *slices = p.S;
  if (first_diag) *first_diag = p.d0;
  if (pairs) *pairs = pr;
  return MPB_OK;
}

static int exact_entry(int cplx, int prec, size_t m, size_t n, size_t k, const void *A, size_t lda, const void *B,
                       size_t ldb, void *C, size_t ldc, int sp_bits, void *workspace, size_t ws_bytes, int *status,
                       void *stream) {
  if (!prec_ok(prec)) return MPB_ERR_PREC;
  /* an empty product still reports: nothing fell back, no kernel error */
  auto clear_status = [&]() -> int {
    if (status && cudaMemsetAsync(status, 0, 2 * sizeof(int), as_stream(stream)) != cudaSuccess) return MPB_ERR_CUDA;
    return MPB_OK;
  };
  if (m == 0 || n == 0) return clear_status();
  if (m > (1u << 24) || n > (1u << 24) || k > (1u << 24)) return MPB_ERR_SIZE;
  if (ldc % 32 || ldc < n) return MPB_ERR_LD;
  if (k > 0 && (lda % 32 || lda < k || ldb % 32 || ldb < n)) return MPB_ERR_LD;
  if (!C || (k > 0 && (!A || !B))) return MPB_ERR_NULL;
  if (!aligned16(C) || (k > 0 && (!aligned16(A) || !aligned16(B)))) return MPB_ERR_ALIGN;
  if (k == 0) { /* empty sums: +0 everywhere */
    const int rc = cplx ? mpb_gemm_c(prec, m, n, 0, nullptr, 32, nullptr, 32, C, ldc, stream)
                        : mpb_gemm_r(prec, m, n, 0, nullptr, 32, nullptr, 32, C, ldc, stream);
    return rc != MPB_OK ? rc : clear_status();
  }
  exact::Plan p;
  if (!exact::make_plan(prec, m, n, k, sp_bits, cplx, p)) return MPB_ERR_ARG;
  if (!workspace || ws_bytes < p.total) return MPB_ERR_WORKSPACE;
  if (((uintptr_t)workspace & 255u) != 0) return MPB_ERR_ALIGN;
  cudaStream_t st = as_stream(stream);
  MPB_DISPATCH_PREC(prec, {
    return exact::run_exact_n<N>(p, (const uint8_t *)A, lda, (const uint8_t *)B, ldb, (uint8_t *)C, ldc,
                                 (uint8_t *)workspace, status, st);
  });
  return MPB_OK;
}

extern "C" int mpb_gemm_exact_r(int prec, size_t m, size_t n, size_t k, const void *A, size_t lda, const void *B,
                                size_t ldb, void *C, size_t ldc, int sp_bits, void *workspace, size_t ws_bytes,
                                int *status, void *stream) {
  return exact_entry(0, prec, m, n, k, A, lda, B, ldb, C, ldc, sp_bits, workspace, ws_bytes, status, stream);
}
extern "C" int mpb_gemm_exact_c(int prec, size_t m, size_t n, size_t k, const void *A, size_t lda, const void *B,
                                size_t ldb, void *C, size_t ldc, int sp_bits, void *workspace, size_t ws_bytes,
                                int *status, void *stream) {
  return exact_entry(1, prec, m, n, k, A, lda, B, ldb, C, ldc, sp_bits, workspace, ws_bytes, status, stream);
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
 * name is only a stand-in, so the address is looked up with that device
 * current, by the first call on the device that succeeds in doing so (that
 * first call should come before any stream capture).  Only a successful
 * lookup is kept: a lookup that fails (no context yet, a capture in progress)
 * returns nullptr for that call, and the next call tries again. */
uint8_t *static_scratch() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  static std::atomic<uint8_t *> addr[64];
  uint8_t *a = addr[dev].load(std::memory_order_acquire);
  if (a) return a;
  void *p = nullptr;
  if (cudaGetSymbolAddress(&p, g_exact_scratch) != cudaSuccess || !p) {
    (void)cudaGetLastError(); /* do not leave the failure for the caller's next check */
    return nullptr;
  }
  addr[dev].store((uint8_t *)p, std::memory_order_release); /* the same address whichever thread wins */
  return (uint8_t *)p;
}
}  // namespace

extern "C" int mpb_gemm_exact_r_static(int prec, size_t m, size_t n, size_t k, const void *A, size_t lda,
                                       const void *B, size_t ldb, void *C, size_t ldc, int sp_bits, int *status,
                                       void *stream) {
  if (!prec_ok(prec)) return MPB_ERR_PREC;
  auto clear_status = [&]() -> int { /* an empty product reports no fallback, no error */
    if (status && cudaMemsetAsync(status, 0, 2 * sizeof(int), as_stream(stream)) != cudaSuccess) return MPB_ERR_CUDA;
    return MPB_OK;
  };
  if (m == 0 || n == 0) return clear_status();
  if (m > (1u << 24) || n > (1u << 24) || k > (1u << 24)) return MPB_ERR_SIZE;
  if (ldc % 32 || ldc < n) return MPB_ERR_LD;
  if (k > 0 && (lda % 32 || lda < k || ldb % 32 || ldb < n)) return MPB_ERR_LD;
  if (!C || (k > 0 && (!A || !B))) return MPB_ERR_NULL;
  if (!aligned16(C) || (k > 0 && (!aligned16(A) || !aligned16(B)))) return MPB_ERR_ALIGN;
  if (k == 0) {
    const int rc = mpb_gemm_r(prec, m, n, 0, nullptr, 32, nullptr, 32, C, ldc, stream);
    return rc != MPB_OK ? rc : clear_status();
  }
  exact::Plan p;
  if (!exact::make_plan(prec, m, n, k, sp_bits, 0, p)) return MPB_ERR_ARG;
  if (p.total > kStaticScratchBytes) return MPB_ERR_SIZE; /* larger than the static scratch area */
  uint8_t *ws = static_scratch();
  if (!ws) return MPB_ERR_CUDA;
  cudaStream_t st = as_stream(stream);
  MPB_DISPATCH_PREC(prec, {
    return exact::run_exact_n<N>(p, (const uint8_t *)A, lda, (const uint8_t *)B, ldb, (uint8_t *)C, ldc, ws, status,
                                 st);
  });
  return MPB_OK;
}

/* failure-path test of the tensor-core kernel: the next launch runs with one
 * accumulator commit withheld in its first CTA and every mbarrier wait limited
 * to wait_ns, so that CTA's epilogue wait runs out, it raises its abort flag,
 * records the error in status[1], waits for its own MMAs and copies, frees its
 * tensor memory and returns */
extern "C" int mpb_gemm_exact_test_inject(int what, long long wait_ns) {
  if (what != 1 || wait_ns < 1000 || wait_ns > (long long)mpb::sm100::kWaitNs) return MPB_ERR_ARG;
  mpb::exact::g_inject_wait_ns.store(wait_ns);
  mpb::exact::g_inject.store(what);
  return MPB_OK;
}
