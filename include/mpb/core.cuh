/* mpb/core.cuh -- register-resident fixed-precision limb arithmetic for sm_100a
 * (and, through the same code, for the host CPU).
 *
 * A value with N 32-bit limbs (precision PB = 32*N bits) is
 *     value = (-1)^s * M * 2^(e - 32*N),   M = sum m[i] * 2^(32 i)
 * with M left-justified (bit 31 of m[N-1] set) unless the value is zero, in
 * which case e == kExpZero and every limb is 0.  e is the MPFR exponent, so an
 * N-limb value has exactly the significand and exponent MPFR stores for the
 * same number at PB bits (MPFR limbs are 64-bit; their 32-bit halves are these
 * limbs), and exactly those of the mpc_cuda cu_freal<PB> struct.
 *
 * Every operation is round-to-nearest-even (MPFR_RNDN) with one rounding per
 * operation:
 *   mul          round(a*b)                (upper half of the N x N product, certified)
 *   add_round    round(x + y)              (x, y exact NX-limb terms, result NM limbs)
 *   fma          round(a*b + c)            (single rounding)
 *   fmms/fmma    round(a*b -/+ c*d)        (single rounding, certified upper-column products; complex multiply)
 *   sum3_round   round(t1 + t2 + t3)       (three exact terms; complex fma: cfma)
 *   div, sqrt_   round(a/b), round(sqrt(a)) (exact long division / integer square root)
 * Zero is unsigned (+0), as in cu_freal (cu_freal.cuh:79-81 of mpc_cuda).
 *
 * B200 design points:
 *  - 32-bit limbs: the integer datapath is 32 bits wide (IMAD / IMAD.HI with
 *    carry), 64-bit limbs would be emulated.
 *  - Products are N^2 32x32->64 multiply-adds in product-scanning order over
 *    PTX carry chains (mad.lo.cc / madc.hi.cc / addc).
 *  - No runtime-indexed local arrays: every shift (alignment, normalisation)
 *    is a compile-time-unrolled log-depth network of predicated selects and
 *    funnel shifts, so all limbs stay in registers.
 *  - Kernels that keep their warps converged may pass kVote=true, which lets a
 *    warp skip the rare normalisation/negation networks when no lane needs them.
 *
 * The host build emulates each PTX carry-chain instruction with an explicit
 * carry flag (same call sequence), so the chain logic is exercised by CPU
 * tests against MPFR.
 */
#ifndef MPB_CORE_CUH
#define MPB_CORE_CUH

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define MPB_HD __host__ __device__ __forceinline__
#define MPB_HDI __host__ __device__ inline
#else
#define MPB_HD inline
#define MPB_HDI inline
#endif

#if defined(__CUDACC__)
#define MPB_UNROLL _Pragma("unroll")
#define MPB_NOINLINE __host__ __device__ __noinline__
#else
#define MPB_UNROLL
#define MPB_NOINLINE
#endif

namespace mpb {

/* exponent of zero: below MPFR's default emin (1 - 2^30) */
constexpr int32_t kExpZero = -(1 << 30);

template <int N>
struct fval {
  uint32_t m[N];
  int32_t e;
  uint32_t s; /* 1 = negative */
};

/* ------------------------------------------------------------------ *
 * carry-chain primitives.  cf is the carry flag; on the device it is
 * the hardware CC.CF and the argument is unused.
 * ------------------------------------------------------------------ */
#if defined(__CUDA_ARCH__)
MPB_HD uint32_t cc_set(uint32_t cin, uint32_t &) { /* CF = (cin != 0), cin in {0,1} */
  uint32_t d;
  asm volatile("add.cc.u32 %0, %1, 0xffffffff;" : "=r"(d) : "r"(cin));
  return d;
}
MPB_HD uint32_t add_cc(uint32_t a, uint32_t b, uint32_t &) {
  uint32_t d;
  asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
MPB_HD uint32_t addc_cc(uint32_t a, uint32_t b, uint32_t &) {
  uint32_t d;
  asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
MPB_HD uint32_t addc(uint32_t a, uint32_t b, uint32_t &) {
  uint32_t d;
  asm volatile("addc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
MPB_HD uint32_t madlo_cc(uint32_t a, uint32_t b, uint32_t c, uint32_t &) {
  uint32_t d;
  asm volatile("mad.lo.cc.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}
MPB_HD uint32_t madclo_cc(uint32_t a, uint32_t b, uint32_t c, uint32_t &) {
  uint32_t d;
  asm volatile("madc.lo.cc.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}
MPB_HD uint32_t madhi_cc(uint32_t a, uint32_t b, uint32_t c, uint32_t &) {
  uint32_t d;
  asm volatile("mad.hi.cc.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}
MPB_HD uint32_t madchi_cc(uint32_t a, uint32_t b, uint32_t c, uint32_t &) {
  uint32_t d;
  asm volatile("madc.hi.cc.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}
MPB_HD uint32_t madchi(uint32_t a, uint32_t b, uint32_t c, uint32_t &) {
  uint32_t d;
  asm volatile("madc.hi.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}
MPB_HD uint32_t sub_cc(uint32_t a, uint32_t b, uint32_t &) { /* CF = borrow */
  uint32_t d;
  asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
MPB_HD uint32_t subc_cc(uint32_t a, uint32_t b, uint32_t &) {
  uint32_t d;
  asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
MPB_HD uint32_t subc(uint32_t a, uint32_t b, uint32_t &) {
  uint32_t d;
  asm volatile("subc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
MPB_HD uint32_t mulhi(uint32_t a, uint32_t b) { return __umulhi(a, b); }
MPB_HD uint32_t fshl(uint32_t lo, uint32_t hi, uint32_t s) { return __funnelshift_l(lo, hi, s); }
MPB_HD uint32_t fshr(uint32_t lo, uint32_t hi, uint32_t s) { return __funnelshift_r(lo, hi, s); }
MPB_HD uint32_t clz32(uint32_t x) { return (uint32_t)__clz(x); }
#else
MPB_HD uint32_t cc_set(uint32_t cin, uint32_t &cf) {
  cf = cin ? 1u : 0u;
  return cin + 0xffffffffu;
}
MPB_HD uint32_t add_cc(uint32_t a, uint32_t b, uint32_t &cf) {
  uint64_t t = (uint64_t)a + b;
  cf = (uint32_t)(t >> 32);
  return (uint32_t)t;
}
MPB_HD uint32_t addc_cc(uint32_t a, uint32_t b, uint32_t &cf) {
  uint64_t t = (uint64_t)a + b + cf;
  cf = (uint32_t)(t >> 32);
  return (uint32_t)t;
}
MPB_HD uint32_t addc(uint32_t a, uint32_t b, uint32_t &cf) { return a + b + cf; }
MPB_HD uint32_t madlo_cc(uint32_t a, uint32_t b, uint32_t c, uint32_t &cf) {
  uint64_t t = (uint64_t)(uint32_t)(a * b) + c;
  cf = (uint32_t)(t >> 32);
  return (uint32_t)t;
}
MPB_HD uint32_t madclo_cc(uint32_t a, uint32_t b, uint32_t c, uint32_t &cf) {
  uint64_t t = (uint64_t)(uint32_t)(a * b) + c + cf;
  cf = (uint32_t)(t >> 32);
  return (uint32_t)t;
}
MPB_HD uint32_t madhi_cc(uint32_t a, uint32_t b, uint32_t c, uint32_t &cf) {
  uint64_t t = (((uint64_t)a * b) >> 32) + c;
  cf = (uint32_t)(t >> 32);
  return (uint32_t)t;
}
MPB_HD uint32_t madchi_cc(uint32_t a, uint32_t b, uint32_t c, uint32_t &cf) {
  uint64_t t = (((uint64_t)a * b) >> 32) + c + cf;
  cf = (uint32_t)(t >> 32);
  return (uint32_t)t;
}
MPB_HD uint32_t madchi(uint32_t a, uint32_t b, uint32_t c, uint32_t &cf) {
  return (uint32_t)(((uint64_t)a * b) >> 32) + c + cf;
}
MPB_HD uint32_t sub_cc(uint32_t a, uint32_t b, uint32_t &cf) {
  cf = a < b ? 1u : 0u;
  return a - b;
}
MPB_HD uint32_t subc_cc(uint32_t a, uint32_t b, uint32_t &cf) {
  const uint64_t t = (uint64_t)a - b - cf;
  cf = (uint32_t)(t >> 63);
  return (uint32_t)t;
}
MPB_HD uint32_t subc(uint32_t a, uint32_t b, uint32_t &cf) { return a - b - cf; }
MPB_HD uint32_t mulhi(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) >> 32); }
MPB_HD uint32_t fshl(uint32_t lo, uint32_t hi, uint32_t s) {
  return (uint32_t)((((uint64_t)hi << 32) | lo) << (s & 31) >> 32);
}
MPB_HD uint32_t fshr(uint32_t lo, uint32_t hi, uint32_t s) {
  return (uint32_t)((((uint64_t)hi << 32) | lo) >> (s & 31));
}
MPB_HD uint32_t clz32(uint32_t x) { return x ? (uint32_t)__builtin_clz(x) : 32u; }
#endif

/* warp-uniform "does any lane need this" vote (device, converged warps only) */
template <bool kVote>
MPB_HD bool any_lane(bool p) {
#if defined(__CUDA_ARCH__)
  if (kVote) return __any_sync(0xffffffffu, p);
#endif
  return p;
}

/* ------------------------------------------------------------------ *
 * exact N x N -> 2N product, schoolbook in product-scanning (column) order:
 * column c accumulates every a[i]*b[c-i] into a 96-bit accumulator with one
 * carry chain per partial product (mad.lo.cc, madc.hi.cc, addc), then emits
 * its low word.  Measured on sm_100a this runs 1.3-1.45x faster than
 * row-by-row lo/hi chains at N = 8..32, at lower register pressure.
 * ------------------------------------------------------------------ */
template <int N>
MPB_HD void mul_full(uint32_t *p, const uint32_t *a, const uint32_t *b) {
  uint32_t c0 = 0u, c1 = 0u, c2 = 0u;
  MPB_UNROLL
  for (int c = 0; c < 2 * N - 1; ++c) {
    MPB_UNROLL
    for (int i = 0; i < N; ++i) {
      const int j = c - i;
      if (j < 0 || j >= N) continue;
      uint32_t cf = 0;
      c0 = madlo_cc(a[i], b[j], c0, cf);
      c1 = madchi_cc(a[i], b[j], c1, cf);
      c2 = addc(c2, 0u, cf);
    }
    p[c] = c0;
    c0 = c1;
    c1 = c2;
    c2 = 0u;
  }
  p[2 * N - 1] = c0;
}

/* m[0..n) += inc (inc in {0,1}); returns the carry out */
template <int n>
MPB_HD uint32_t inc_n(uint32_t *m, uint32_t inc) {
  uint32_t cf = 0;
  m[0] = add_cc(m[0], inc, cf);
  MPB_UNROLL
  for (int i = 1; i < n; ++i) m[i] = addc_cc(m[i], 0u, cf);
  return addc(0u, 0u, cf);
}

/* Round-to-nearest-even increment of the NM-limb mantissa m given the round
 * bit rb and a nonzero-if-sticky word st; renormalises on carry-out. */
/* round the mantissa m given the round bit rb and the sticky word st: to
 * nearest-even (kRnd = 0), or to odd (kRnd = 1: truncate, then set the last
 * bit when anything was lost -- the intermediate rounding that makes a later
 * rounding to nearest at 2 or more bits fewer correct, Boldo and Melquiond,
 * "Emulation of FMA and correctly rounded sums: proved algorithms using
 * rounding to odd", IEEE Trans. Computers 2008) */
template <int NM, int kRnd = 0>
MPB_HD void rndn(uint32_t *m, int32_t &e, uint32_t rb, uint32_t st) {
  if (kRnd == 1) {
    m[0] |= (rb | st) != 0u ? 1u : 0u;
    return;
  }
  const uint32_t inc = rb & ((st != 0u) | (m[0] & 1u));
  const uint32_t c = inc_n<NM>(m, inc);
  m[NM - 1] |= c << 31; /* all-ones + 1 -> 1000...0 */
  e += (int32_t)c;
}

/* ------------------------------------------------------------------ *
 * r = round(a * b)
 * ------------------------------------------------------------------ */
/* Round an exact normalised-or-half-normalised 2N-limb product p (leading
 * one at bit 64N-1 or 64N-2) with exponent e (for the 64N-1 case) to N limbs. */
template <int N, int kRnd = 0>
MPB_HD void round_prod(fval<N> &r, const uint32_t *p, int32_t e, uint32_t s) {
  const uint32_t sh = (p[2 * N - 1] >> 31) ^ 1u;
  MPB_UNROLL
  for (int i = 0; i < N; ++i) r.m[i] = fshl(p[N + i - 1], p[N + i], sh);
  const uint32_t below = (N >= 2) ? p[N - 2] : 0u;
  const uint32_t low = fshl(below, p[N - 1], sh);
  uint32_t st = low << 1;
  MPB_UNROLL
  for (int i = 0; i < N - 1; ++i) st |= p[i];
  r.e = e - (int32_t)sh;
  rndn<N, kRnd>(r.m, r.e, low >> 31, st);
  r.s = s;
}

template <int N>
MPB_HD void set_zero(fval<N> &r) {
  MPB_UNROLL
  for (int i = 0; i < N; ++i) r.m[i] = 0u;
  r.e = kExpZero;
  r.s = 0u;
}
template <int N>
MPB_HD bool is_zero(const fval<N> &x) {
  return x.e == kExpZero;
}

/* the upper columns only: p[N-2 .. 2N-1] of T = sum_{i+j >= N-2} a_i b_j
 * 2^(32(i+j)), in the same product-scanning order as mul_full; the omitted
 * pairs sum to L < (N-2) 2^(32(N-1)), below 2^38 units of word N-2 (N <= 64) */
template <int N>
MPB_HD void mul_high(uint32_t *p, const uint32_t *a, const uint32_t *b) {
  uint32_t c0 = 0u, c1 = 0u, c2 = 0u;
  MPB_UNROLL
  for (int c = N - 2; c < 2 * N - 1; ++c) {
    MPB_UNROLL
    for (int i = 0; i < N; ++i) {
      const int j = c - i;
      if (j < 0 || j >= N) continue;
      uint32_t cf = 0;
      c0 = madlo_cc(a[i], b[j], c0, cf);
      c1 = madchi_cc(a[i], b[j], c1, cf);
      c2 = addc(c2, 0u, cf);
    }
    p[c] = c0;
    c0 = c1;
    c1 = c2;
    c2 = 0u;
  }
  p[2 * N - 1] = c0;
}

/* the full product and its rounding, out of line: the rare case of mul.
 * Up to kByValueLimbs limbs the operands and the result travel by value: the
 * call passes them in registers, whereas references to a caller's registers
 * make the caller keep those values in local memory (a stack frame) for the
 * call.  Above it the argument registers run out and by-value passing spills,
 * so wider operands go by reference. */
constexpr int kByValueLimbs = 20;
template <int N, int kRnd = 0>
MPB_NOINLINE fval<N> mul_full_round_v(fval<N> a, fval<N> b) {
  uint32_t p[2 * N];
  mul_full<N>(p, a.m, b.m);
  fval<N> r;
  round_prod<N, kRnd>(r, p, a.e + b.e, a.s ^ b.s);
  return r;
}
template <int N, int kRnd = 0>
MPB_NOINLINE void mul_full_round_r(fval<N> &r, const fval<N> &a, const uint32_t *bm, int32_t be, uint32_t bs) {
  uint32_t p[2 * N];
  mul_full<N>(p, a.m, bm);
  round_prod<N, kRnd>(r, p, a.e + be, a.s ^ bs);
}
template <int N, int kRnd = 0>
MPB_HD void mul_full_round(fval<N> &r, const fval<N> &a, const uint32_t *bm, int32_t be, uint32_t bs) {
  if constexpr (N <= kByValueLimbs) {
    fval<N> b;
    MPB_UNROLL
    for (int i = 0; i < N; ++i) b.m[i] = bm[i];
    b.e = be;
    b.s = bs;
    r = mul_full_round_v<N, kRnd>(a, b);
  } else {
    mul_full_round_r<N, kRnd>(r, a, bm, be, bs);
  }
}

/* r = round(a * b), b given by its limbs (which may live in shared memory:
 * mul_high reads them one at a time) and exponent / sign.  From N = 4 limbs
 * up only the upper columns are computed (about half the partial products).  With X the 64 bits under the
 * mantissa (words N-1 and N-2 of T after the normalisation shift), the exact
 * product has X + lambda there, 0 <= lambda < 2^39: X <= 2^63 - 2^39 - 1
 * rounds down and X > 2^63 rounds up (a carry into the mantissa gives the
 * same result) whatever lambda is.  X in between -- about 2^-25 of random
 * operands, exact ties included -- rounds the full product instead. */
template <int N, int kRnd = 0>
MPB_HD void mul_limbs(fval<N> &r, const fval<N> &a, const uint32_t *bm, int32_t be, uint32_t bs) {
  uint32_t p[2 * N];
  if (kRnd == 1) { /* rounding to odd needs exactness: the full product */
    mul_full_round<N, 1>(r, a, bm, be, bs);
  } else if (N >= 4) {
    mul_high<N>(p, a.m, bm);
    MPB_UNROLL
    for (int i = 0; i < N - 2; ++i) p[i] = 0u;
    const uint32_t sh = (p[2 * N - 1] >> 31) ^ 1u;
    const uint64_t X = ((((uint64_t)p[N - 1]) << 32) | p[N - 2]) << sh;
    const bool sure = X <= (1ull << 63) - (1ull << 39) - 1ull || X > (1ull << 63);
    if (sure)
      round_prod<N>(r, p, a.e + be, a.s ^ bs);
    else
      mul_full_round<N>(r, a, bm, be, bs);
  } else {
    mul_full<N>(p, a.m, bm);
    round_prod<N>(r, p, a.e + be, a.s ^ bs);
  }
  if (is_zero(a) || be == kExpZero) set_zero(r);
}
/* the same with b as a value */
template <int N, int kRnd = 0>
MPB_HD void mul(fval<N> &r, const fval<N> &a, const fval<N> &b) {
  mul_limbs<N, kRnd>(r, a, b.m, b.e, b.s);
}

/* r = round(a * b) for a b whose limbs below the top K are zero (a scalar
 * converted from a double has K <= 2, a small integer K = 1): the exact
 * N x K product (N+K words, N*K partial products in the column order of
 * mul_full) lands in the top of the 2N-word array and is rounded once, so no
 * certification is needed. */
template <int N, int K>
MPB_HD void mul_short(fval<N> &r, const fval<N> &a, const uint32_t *bm, int32_t be, uint32_t bs) {
  static_assert(K >= 1 && K < N, "short operand");
  uint32_t p[2 * N];
  MPB_UNROLL
  for (int i = 0; i < N - K; ++i) p[i] = 0u;
  uint32_t c0 = 0u, c1 = 0u, c2 = 0u;
  MPB_UNROLL
  for (int c = 0; c < N + K - 1; ++c) {
    MPB_UNROLL
    for (int j = 0; j < K; ++j) {
      const int i = c - j;
      if (i < 0 || i >= N) continue;
      uint32_t cf = 0;
      c0 = madlo_cc(a.m[i], bm[N - K + j], c0, cf);
      c1 = madchi_cc(a.m[i], bm[N - K + j], c1, cf);
      c2 = addc(c2, 0u, cf);
    }
    p[N - K + c] = c0;
    c0 = c1;
    c1 = c2;
    c2 = 0u;
  }
  p[2 * N - 1] = c0;
  round_prod<N>(r, p, a.e + be, a.s ^ bs);
  if (is_zero(a) || be == kExpZero) set_zero(r);
}
/* the number of limbs of b from the top down to its lowest nonzero limb (1 for zero) */
template <int N>
MPB_HD int limb_length(const uint32_t *bm) {
  int k = N;
  while (k > 1 && bm[N - k] == 0u) --k;
  return k;
}

/* exact product, normalised so that bit 31 of p[2N-1] is set (zero stays 0) */
template <int N>
MPB_HD void mul_exact_norm(uint32_t *p, int32_t &e, const fval<N> &a, const fval<N> &b) {
  mul_full<N>(p, a.m, b.m);
  const uint32_t sh = (p[2 * N - 1] >> 31) ^ 1u;
  MPB_UNROLL
  for (int i = 2 * N - 1; i > 0; --i) p[i] = fshl(p[i - 1], p[i], sh);
  p[0] <<= sh;
  e = a.e + b.e - (int32_t)sh;
  if (is_zero(a) || is_zero(b)) e = kExpZero;
}

/* ------------------------------------------------------------------ *
 * r = round(x + y) for exact NX-limb terms x, y (each normalised, or zero
 * with kExpZero and zero limbs), rounded once to NM <= NX limbs.
 *
 * Window of W = NX + 2 limbs: the larger-exponent term sits in the top NX
 * limbs, the other is shifted right by the exponent difference d; bits that
 * fall below the window only matter as sticky.  For opposite signs, a sticky
 * window makes the window difference one unit too large, so one unit is
 * subtracted (borrow-in) and sticky stays set; the cancellation can then be
 * at most one bit (d >= 2), well inside the 64-bit guard.  A negative window
 * difference (possible only for d = 0) is negated exactly.
 * ------------------------------------------------------------------ */
template <int W>
struct log2_ceil {
  static constexpr int v = (W <= 1) ? 0 : 1 + log2_ceil<(W + 1) / 2>::v;
};
template <>
struct log2_ceil<1> {
  static constexpr int v = 0;
};

/* kCertBits > 0: the terms are known only to within a total error below
 * 2^(ea - kCertBits) (ea = the larger term exponent), and the function also
 * reports whether every value within that error rounds to the same r: the
 * error must stay under a quarter ULP of r and the bits under the mantissa,
 * read as the 64-bit fraction G, clear of the midpoint by more than it (a
 * zero sum never certifies).  Without it the return value is true. */
template <int NX, int NM, bool kVote = false, int kCertBits = 0, int kRnd = 0>
MPB_HD bool add_round(fval<NM> &r, const uint32_t *xm, int32_t xe, uint32_t xs,
                      const uint32_t *ym, int32_t ye, uint32_t ys) {
  constexpr int W = NX + 2;
  constexpr int KQ = log2_ceil<W + 1>::v; /* limb-shift stages: 2^KQ > W */
  const bool sw = ye > xe;
  uint32_t D[W + 1], Y[W];
  D[0] = 0u;
  D[1] = 0u;
  Y[0] = 0u;
  Y[1] = 0u;
  MPB_UNROLL
  for (int i = 0; i < NX; ++i) {
    D[i + 2] = sw ? ym[i] : xm[i];
    Y[i + 2] = sw ? xm[i] : ym[i];
  }
  const int32_t ea = sw ? ye : xe;
  const int32_t eb = sw ? xe : ye;
  const uint32_t sa = sw ? ys : xs;
  const uint32_t sb = sw ? xs : ys;

  /* ---- align Y right by d = ea - eb bits (limb part q, bit part rs) ---- */
  const uint32_t d = (uint32_t)(ea - eb);
  const uint32_t q = (d >> 5) < (uint32_t)W ? (d >> 5) : (uint32_t)W;
  const uint32_t rs = d & 31u;
  uint32_t st = 0u;
  /* whole-word part of the shift: a log-depth select network.  Only as many
   * stages run as the warp needs: none when no lane shifts by a word or more
   * (exponents within 32 bits), two when every lane shifts by at most 3 words
   * (the common case of AXPY and dot-product operands), else all KQ. */
  const int kq_run = any_lane<kVote>(q >= 4u) ? KQ : (any_lane<kVote>(q != 0u) ? 2 : 0);
  if (kq_run != 0) {
    MPB_UNROLL
    for (int k = 0; k < KQ; ++k) {
      if (k >= 2 && kq_run == 2) break;
      const int sh = 1 << k;
      const bool on = (q >> k) & 1u;
      uint32_t lost = 0u;
      MPB_UNROLL
      for (int i = 0; i < sh && i < W; ++i) lost |= Y[i];
      st |= on ? lost : 0u;
      MPB_UNROLL
      for (int i = 0; i < W; ++i) {
        const uint32_t src = (i + sh < W) ? Y[i + sh] : 0u;
        Y[i] = on ? src : Y[i];
      }
    }
  }
  st |= Y[0] & ((1u << rs) - 1u);
  MPB_UNROLL
  for (int i = 0; i < W - 1; ++i) Y[i] = fshr(Y[i], Y[i + 1], rs);
  Y[W - 1] >>= rs;

  /* ---- D = X + Y   or   X - Y - sticky ---- */
  const uint32_t sub = sa ^ sb;
  const uint32_t msk = 0u - sub;
  const uint32_t cin = sub & (st == 0u ? 1u : 0u);
  uint32_t cf = 0;
  cc_set(cin, cf);
  MPB_UNROLL
  for (int i = 0; i < W; ++i) D[i] = addc_cc(D[i], Y[i] ^ msk, cf);
  const uint32_t c = addc(0u, 0u, cf);

  /* negative difference (d == 0 and |y| > |x|): negate exactly */
  const uint32_t neg = sub & (c ^ 1u);
  if (any_lane<kVote>(neg != 0u)) {
    const uint32_t nm = 0u - neg;
    uint32_t cf2 = 0;
    cc_set(neg, cf2);
    MPB_UNROLL
    for (int i = 0; i < W; ++i) D[i] = addc_cc(D[i] ^ nm, 0u, cf2);
  }
  uint32_t s = sa ^ neg;

  /* same-sign carry-out: shift right by one, the lost bit joins sticky */
  const uint32_t cs = (sub ^ 1u) & c;
  st |= D[0] & cs;
  D[W] = c;
  MPB_UNROLL
  for (int i = 0; i < W; ++i) D[i] = fshr(D[i], D[i + 1], cs);

  /* ---- normalise left (cancellation after subtraction) ---- */
  /* the leading word is the top one unless a subtraction cancelled 32 bits or
   * more: search the window only when some lane needs it */
  uint32_t lq = 0u, top = D[W - 1];
  if (any_lane<kVote>(top == 0u)) {
    lq = (uint32_t)W;
    MPB_UNROLL
    for (int i = W - 1; i >= 0; --i) {
      const bool take = (lq == (uint32_t)W) && (D[i] != 0u);
      top = take ? D[i] : top;
      lq = take ? (uint32_t)(W - 1 - i) : lq;
    }
  }
  const bool zero = (lq == (uint32_t)W);
  const uint32_t lr = clz32(top) & 31u;
  if (any_lane<kVote>(lq != 0u && !zero)) {
    const uint32_t qq = zero ? 0u : lq;
    MPB_UNROLL
    for (int k = 0; k < KQ; ++k) {
      const int sh = 1 << k;
      const bool on = (qq >> k) & 1u;
      MPB_UNROLL
      for (int i = W - 1; i >= 0; --i) {
        const uint32_t src = (i - sh >= 0) ? D[i - sh] : 0u;
        D[i] = on ? src : D[i];
      }
    }
  }
  MPB_UNROLL
  for (int i = W - 1; i > 0; --i) D[i] = fshl(D[i - 1], D[i], lr);
  D[0] <<= lr;

  /* ---- round to NM limbs ---- */
  MPB_UNROLL
  for (int i = 0; i < NM; ++i) r.m[i] = D[W - NM + i];
  const uint32_t g = D[W - NM - 1];
  st |= g << 1;
  MPB_UNROLL
  for (int i = 0; i < W - NM - 1; ++i) st |= D[i];
  int32_t e = ea + (int32_t)cs - (int32_t)(32u * lq + lr);
  bool ok = true;
  if (kCertBits > 0) {
    static_assert(W - NM - 2 >= 0, "no word under the guard word");
    const int64_t t = ((int64_t)ea - kCertBits) - ((int64_t)e - 32 * NM); /* log2 of the error in ULPs */
    const uint64_t G = ((uint64_t)g << 32) | D[W - NM - 2];
    const uint64_t thr = (t < -64) ? 1ull : (1ull << (64 + (t < -3 ? t : -3)));
    const uint64_t half = 1ull << 63;
    ok = !zero && t <= -3 && (G <= half - thr - 1 || G > half + thr);
  }
  rndn<NM, kRnd>(r.m, e, g >> 31, st);
  r.e = e;
  r.s = s;
  if (any_lane<kVote>(zero) && zero) set_zero(r); /* x = -y exactly */
  return ok;
}

/* r = round(x + y), r = round(x - y) */
template <int N, bool kVote = false, int kRnd = 0>
MPB_HD void add(fval<N> &r, const fval<N> &x, const fval<N> &y) {
  add_round<N, N, kVote, 0, kRnd>(r, x.m, x.e, x.s, y.m, y.e, y.s);
}
template <int N, bool kVote = false, int kRnd = 0>
MPB_HD void sub(fval<N> &r, const fval<N> &x, const fval<N> &y) {
  add_round<N, N, kVote, 0, kRnd>(r, x.m, x.e, x.s, y.m, y.e, y.s ^ (is_zero(y) ? 0u : 1u));
}

/* r = round(a*b + c), one rounding (MPFR mpfr_fma semantics) */
template <int N, bool kVote = false, int kRnd = 0>
MPB_HD void fma(fval<N> &r, const fval<N> &a, const fval<N> &b, const fval<N> &c) {
  uint32_t p[2 * N], cw[2 * N];
  int32_t pe;
  mul_exact_norm<N>(p, pe, a, b);
  MPB_UNROLL
  for (int i = 0; i < N; ++i) {
    cw[i] = 0u;
    cw[N + i] = c.m[i];
  }
  add_round<2 * N, N, kVote, 0, kRnd>(r, p, pe, a.s ^ b.s, cw, c.e, c.s);
}

/* round(a*b - c*d) and round(a*b + c*d), one rounding each (MPFR
 * mpfr_fmms / mpfr_fmma semantics; the exact-intermediate complex product
 * of MPC_RNDNN, mpc_cuda cu_fcomplex.cuh:91-96) */
template <int N>
MPB_NOINLINE fval<N> fmms_full_v(fval<N> a, fval<N> b, fval<N> c, fval<N> d, uint32_t negate_cd) {
  uint32_t p1[2 * N], p2[2 * N];
  int32_t e1, e2;
  mul_exact_norm<N>(p1, e1, a, b);
  mul_exact_norm<N>(p2, e2, c, d);
  fval<N> r;
  add_round<2 * N, N>(r, p1, e1, a.s ^ b.s, p2, e2, c.s ^ d.s ^ negate_cd);
  return r;
}
template <int N>
MPB_NOINLINE void fmms_full_r(fval<N> &r, const fval<N> &a, const fval<N> &b, const fval<N> &c, const fval<N> &d,
                              uint32_t negate_cd) {
  uint32_t p1[2 * N], p2[2 * N];
  int32_t e1, e2;
  mul_exact_norm<N>(p1, e1, a, b);
  mul_exact_norm<N>(p2, e2, c, d);
  add_round<2 * N, N>(r, p1, e1, a.s ^ b.s, p2, e2, c.s ^ d.s ^ negate_cd);
}
template <int N>
MPB_HD void fmms_full(fval<N> &r, const fval<N> &a, const fval<N> &b, const fval<N> &c, const fval<N> &d,
                      uint32_t negate_cd) {
  if constexpr (N <= kByValueLimbs)
    r = fmms_full_v<N>(a, b, c, d, negate_cd);
  else
    fmms_full_r<N>(r, a, b, c, d, negate_cd);
}

/* upper columns of a*b (mul_high), normalised like mul_exact_norm; zero stays 0 */
template <int N>
MPB_HD void mul_high_norm(uint32_t *p, int32_t &e, const fval<N> &a, const fval<N> &b) {
  mul_high<N>(p, a.m, b.m);
  MPB_UNROLL
  for (int i = 0; i < N - 2; ++i) p[i] = 0u;
  const uint32_t sh = (p[2 * N - 1] >> 31) ^ 1u;
  MPB_UNROLL
  for (int i = 2 * N - 1; i > 0; --i) p[i] = fshl(p[i - 1], p[i], sh);
  p[0] <<= sh;
  e = a.e + b.e - (int32_t)sh;
  if (is_zero(a) || is_zero(b)) e = kExpZero;
}

/* From N = 4 limbs up both products are taken from their upper columns
 * only: each then misses less than N 2^(32(N-1)) units of its lowest word,
 * i.e. below 2^(e_i - 32N - 25) for |product| < 2^(e_i), so the sum is off by
 * less than 2^(e_max - 32N - 24).  add_round certifies the rounding against
 * that (it fails under heavy cancellation -- more than about 20 bits -- or
 * next to a midpoint), and the exact products decide otherwise.  The words
 * under column N-2 of a normalised upper-column product are zero, so the sum
 * takes the top N+2 words of each (an (N+4)-word window instead of 2N+2). */
template <int N, bool kVote = false>
MPB_HD void fmms(fval<N> &r, const fval<N> &a, const fval<N> &b, const fval<N> &c,
                 const fval<N> &d, uint32_t negate_cd = 1u) {
  uint32_t p1[2 * N], p2[2 * N];
  int32_t e1, e2;
  uint32_t s2 = c.s ^ d.s ^ negate_cd;
  if (N >= 4) {
    mul_high_norm<N>(p1, e1, a, b);
    mul_high_norm<N>(p2, e2, c, d);
    const bool ok = add_round<N + 2, N, kVote, 32 * N + 24>(r, p1 + (N - 2), e1, a.s ^ b.s, p2 + (N - 2), e2, s2);
    if (!ok && !(e1 == kExpZero && e2 == kExpZero)) fmms_full<N>(r, a, b, c, d, negate_cd);
  } else {
    mul_exact_norm<N>(p1, e1, a, b);
    mul_exact_norm<N>(p2, e2, c, d);
    add_round<2 * N, N, kVote>(r, p1, e1, a.s ^ b.s, p2, e2, s2);
  }
}
template <int N, bool kVote = false>
MPB_HD void fmma(fval<N> &r, const fval<N> &a, const fval<N> &b, const fval<N> &c,
                 const fval<N> &d) {
  fmms<N, kVote>(r, a, b, c, d, 0u);
}

/* complex (MPC_RNDNN): re = round(ar*br - ai*bi), im = round(ar*bi + ai*br) */
template <int N, bool kVote = false>
MPB_HD void cmul(fval<N> &rr, fval<N> &ri, const fval<N> &ar, const fval<N> &ai,
                 const fval<N> &br, const fval<N> &bi) {
  fmms<N, kVote>(rr, ar, br, ai, bi, 1u);
  fmms<N, kVote>(ri, ar, bi, ai, br, 0u);
}

/* ------------------------------------------------------------------ *
 * r = round(t1 + t2 + t3) for three exact terms, one rounding.
 * ------------------------------------------------------------------ */
/* Window sum of two exact L-limb terms: x (the larger exponent; zero only if
 * y is zero too) sits in the top L of WS = 2L + 2 words, y is shifted right
 * by d = xe - ye.  When d <= 32 (L + 1) every bit of y lands in words 1..WS-1
 * and the sum is exact; otherwise the bits of y below the window become the
 * sticky-borrow of add_round and are folded into the lowest bit, which makes
 * the sum round-to-odd at 32 WS bits.  o is normalised (top bit set), zero is
 * kExpZero with zero words.  Exponents follow add_round: the alignment shift
 * of two terms is their exponent difference. */
template <int L>
MPB_HD void sum2_odd(uint32_t (&o)[2 * L + 2], int32_t &oe, uint32_t &os, const uint32_t *xm, int32_t xe,
                     uint32_t xs, const uint32_t *ym, int32_t ye, uint32_t ys) {
  constexpr int WS = 2 * L + 2;
  constexpr int KQ = log2_ceil<WS + 1>::v;
  uint32_t D[WS + 1], Y[WS];
  MPB_UNROLL
  for (int i = 0; i < WS; ++i) {
    D[i] = (i >= WS - L) ? xm[i - (WS - L)] : 0u;
    Y[i] = (i >= WS - L) ? ym[i - (WS - L)] : 0u;
  }
  const uint32_t d = (uint32_t)(xe - ye);
  const uint32_t q = (d >> 5) < (uint32_t)WS ? (d >> 5) : (uint32_t)WS;
  const uint32_t rs = d & 31u;
  uint32_t st = 0u;
  MPB_UNROLL
  for (int k = 0; k < KQ; ++k) {
    const int sh = 1 << k;
    const bool on = (q >> k) & 1u;
    uint32_t lost = 0u;
    MPB_UNROLL
    for (int i = 0; i < sh && i < WS; ++i) lost |= Y[i];
    st |= on ? lost : 0u;
    MPB_UNROLL
    for (int i = 0; i < WS; ++i) {
      const uint32_t src = (i + sh < WS) ? Y[i + sh] : 0u;
      Y[i] = on ? src : Y[i];
    }
  }
  st |= Y[0] & ((1u << rs) - 1u);
  MPB_UNROLL
  for (int i = 0; i < WS - 1; ++i) Y[i] = fshr(Y[i], Y[i + 1], rs);
  Y[WS - 1] >>= rs;

  const uint32_t sub = xs ^ ys;
  const uint32_t msk = 0u - sub;
  uint32_t cf = 0;
  cc_set(sub & (st == 0u ? 1u : 0u), cf);
  MPB_UNROLL
  for (int i = 0; i < WS; ++i) D[i] = addc_cc(D[i], Y[i] ^ msk, cf);
  const uint32_t c = addc(0u, 0u, cf);
  const uint32_t neg = sub & (c ^ 1u); /* only when d == 0: exact negation */
  {
    const uint32_t nm = 0u - neg;
    uint32_t cf2 = 0;
    cc_set(neg, cf2);
    MPB_UNROLL
    for (int i = 0; i < WS; ++i) D[i] = addc_cc(D[i] ^ nm, 0u, cf2);
  }
  const uint32_t cs = (sub ^ 1u) & c;
  st |= D[0] & cs;
  D[WS] = c;
  MPB_UNROLL
  for (int i = 0; i < WS; ++i) D[i] = fshr(D[i], D[i + 1], cs);
  D[0] |= (st != 0u) ? 1u : 0u; /* round to odd */

  uint32_t lq = (uint32_t)WS, top = 0u;
  MPB_UNROLL
  for (int i = WS - 1; i >= 0; --i) {
    const bool take = (lq == (uint32_t)WS) && (D[i] != 0u);
    top = take ? D[i] : top;
    lq = take ? (uint32_t)(WS - 1 - i) : lq;
  }
  const bool zero = (lq == (uint32_t)WS);
  const uint32_t lr = clz32(top) & 31u;
  const uint32_t qq = zero ? 0u : lq;
  MPB_UNROLL
  for (int k = 0; k < KQ; ++k) {
    const int sh = 1 << k;
    const bool on = (qq >> k) & 1u;
    MPB_UNROLL
    for (int i = WS - 1; i >= 0; --i) {
      const uint32_t src = (i - sh >= 0) ? D[i - sh] : 0u;
      D[i] = on ? src : D[i];
    }
  }
  MPB_UNROLL
  for (int i = WS - 1; i > 0; --i) D[i] = fshl(D[i - 1], D[i], lr);
  D[0] <<= lr;
  MPB_UNROLL
  for (int i = 0; i < WS; ++i) o[i] = zero ? 0u : D[i];
  oe = zero ? kExpZero : xe + (int32_t)cs - (int32_t)(32u * lq + lr);
  os = zero ? 0u : (xs ^ neg);
}

/* round(t1 + t2 + t3), each term exact with L limbs (normalised or zero).
 * With the terms ordered by exponent: if the second fits the window of the
 * first (gap <= 32 (L + 1) bits), their sum is exact and is rounded together
 * with the third by add_round; otherwise the first term is more than 32(L+1)
 * bits above the other two, their window sum is rounded to odd at 32(2L+2)
 * bits -- its last bit lies below add_round's window, where only the sign
 * and the non-zeroness of the remainder matter, and rounding to odd keeps
 * both -- and it is rounded together with the first. */
template <int L, int NM, bool kVote = false>
MPB_HD void sum3_round(fval<NM> &r, const uint32_t *am, int32_t ae, uint32_t as, const uint32_t *bm, int32_t be,
                       uint32_t bs, const uint32_t *cm, int32_t ce, uint32_t cs) {
  constexpr int WS = 2 * L + 2;
  /* order by exponent: t1 >= t2 >= t3 (selects, no runtime-indexed arrays) */
  uint32_t t1[L], t2[L], t3[L];
  int32_t e1 = ae, e2 = be, e3 = ce;
  uint32_t s1 = as, s2 = bs, s3 = cs;
  MPB_UNROLL
  for (int i = 0; i < L; ++i) {
    t1[i] = am[i];
    t2[i] = bm[i];
    t3[i] = cm[i];
  }
  auto cswap = [&](uint32_t(&x)[L], int32_t &xe, uint32_t &xs, uint32_t(&y)[L], int32_t &ye, uint32_t &ys) {
    const bool sw = ye > xe;
    MPB_UNROLL
    for (int i = 0; i < L; ++i) {
      const uint32_t a = x[i], b = y[i];
      x[i] = sw ? b : a;
      y[i] = sw ? a : b;
    }
    const int32_t ea = xe, eb = ye;
    xe = sw ? eb : ea;
    ye = sw ? ea : eb;
    const uint32_t sa = xs, sb = ys;
    xs = sw ? sb : sa;
    ys = sw ? sa : sb;
  };
  cswap(t1, e1, s1, t2, e2, s2);
  cswap(t2, e2, s2, t3, e3, s3);
  cswap(t1, e1, s1, t2, e2, s2);

  /* near: sum t1 + t2 exactly, then round with t3; far: t2 + t3 (exact or
   * rounded to odd), then round with t1 -- one window sum either way */
  const bool near = (int64_t)e1 - e2 <= 32 * (L + 1);
  uint32_t P[L], Q[L], X[WS], S[WS];
  MPB_UNROLL
  for (int i = 0; i < L; ++i) {
    P[i] = near ? t1[i] : t2[i];
    Q[i] = near ? t2[i] : t3[i];
  }
  MPB_UNROLL
  for (int i = 0; i < WS; ++i) X[i] = (i >= WS - L) ? (near ? t3[i - (WS - L)] : t1[i - (WS - L)]) : 0u;
  int32_t se;
  uint32_t ss;
  sum2_odd<L>(S, se, ss, P, near ? e1 : e2, near ? s1 : s2, Q, near ? e2 : e3, near ? s2 : s3);
  add_round<WS, NM, kVote>(r, X, near ? e3 : e1, near ? s3 : s1, S, se, ss);
}

/* round(a*b + c*d + e) with one rounding (negate_cd flips the sign of c*d):
 * one component of a complex fused multiply-add */
template <int N, bool kVote = false>
MPB_HD void fmma_add(fval<N> &r, const fval<N> &a, const fval<N> &b, const fval<N> &c, const fval<N> &d,
                     const fval<N> &e, uint32_t negate_cd) {
  uint32_t p1[2 * N], p2[2 * N], ew[2 * N];
  int32_t e1, e2;
  mul_exact_norm<N>(p1, e1, a, b);
  mul_exact_norm<N>(p2, e2, c, d);
  MPB_UNROLL
  for (int i = 0; i < N; ++i) {
    ew[i] = 0u;
    ew[N + i] = e.m[i];
  }
  const uint32_t s2 = (e2 == kExpZero) ? 0u : (c.s ^ d.s ^ negate_cd);
  sum3_round<2 * N, N, kVote>(r, p1, e1, (e1 == kExpZero) ? 0u : (a.s ^ b.s), p2, e2, s2, ew, e.e, e.s);
}

/* complex (MPC_RNDNN) fused multiply-add: re = round(ar*br - ai*bi + cr),
 * im = round(ar*bi + ai*br + ci), each with one rounding (MPC mpc_fma).  The
 * two components run through one instance of the three-term sum (a loop
 * over the component with selected operands) to halve the code. */
template <int N, bool kVote = false>
MPB_HD void cfma(fval<N> &rr, fval<N> &ri, const fval<N> &ar, const fval<N> &ai, const fval<N> &br,
                 const fval<N> &bi, const fval<N> &cr, const fval<N> &ci) {
#ifdef __CUDA_ARCH__
#pragma unroll 1
#endif
  for (int comp = 0; comp < 2; ++comp) {
    const bool im = comp == 1;
    fval<N> y, z, r;
    MPB_UNROLL
    for (int i = 0; i < N; ++i) {
      y.m[i] = im ? bi.m[i] : br.m[i];
      z.m[i] = im ? br.m[i] : bi.m[i];
    }
    y.e = im ? bi.e : br.e;
    y.s = im ? bi.s : br.s;
    z.e = im ? br.e : bi.e;
    z.s = im ? br.s : bi.s;
    fmma_add<N, kVote>(r, ar, y, ai, z, im ? ci : cr, im ? 0u : 1u);
    if (im)
      ri = r;
    else
      rr = r;
  }
}

/* ------------------------------------------------------------------ *
 * Division and square root, correctly rounded (MPFR mpfr_div / mpfr_sqrt)
 * ------------------------------------------------------------------ */
/* Long division of limb integers (Knuth's algorithm D, base 2^32), every
 * index known at compile time: q[0 .. NU-NV) = floor(U / V) and u[0 .. NV)
 * becomes U mod V.  V must be normalised (top bit of v[NV-1] set) and
 * U < V * 2^(32 (NU - NV)).  Each quotient limb is estimated from the top two
 * remainder limbs and the top divisor limb d by the 2-by-1 division of
 * Moeller and Granlund ("Improved division by invariant integers", IEEE
 * Trans. Computers 2011) with the reciprocal floor((2^64 - 1) / d) - 2^32
 * computed once, corrected with the second divisor limb (at most twice,
 * Knuth's test), and fixed by one add-back when the multiply-subtract -- a
 * carry chain over the limb product and a borrow chain over the remainder
 * -- goes negative. */
template <int NU, int NV>
MPB_HD void divmod_limbs(uint32_t *q, uint32_t *u, const uint32_t *v) {
  const uint32_t d = v[NV - 1];
  const uint64_t v2 = NV >= 2 ? v[NV - 2 >= 0 ? NV - 2 : 0] : 0u;
  const uint32_t rcp = (uint32_t)(0xffffffffffffffffull / d - (1ull << 32));
  MPB_UNROLL
  for (int j = NU - NV - 1; j >= 0; --j) {
    const uint32_t u1 = u[j + NV], u0 = u[j + NV - 1];
    uint64_t qh, rh;
    if (u1 >= d) { /* (u1 = d): the estimate is 2^32 - 1 */
      qh = 0xffffffffull;
      rh = (uint64_t)u0 + d;
    } else { /* 2-by-1 division with the reciprocal */
      const uint64_t qq = (uint64_t)rcp * u1 + (((uint64_t)u1 << 32) | u0);
      uint32_t q1 = (uint32_t)(qq >> 32) + 1u;
      const uint32_t q0 = (uint32_t)qq;
      uint32_t r = u0 - q1 * d;
      if (r > q0) {
        --q1;
        r += d;
      }
      if (r >= d) {
        ++q1;
        r -= d;
      }
      qh = q1;
      rh = r;
    }
    const uint64_t u3 = (j + NV - 2 >= 0) ? u[j + NV - 2 >= 0 ? j + NV - 2 : 0] : 0u;
    MPB_UNROLL
    for (int c = 0; c < 2; ++c) {
      if (rh < (1ull << 32) && qh * v2 > ((rh << 32) | u3)) {
        --qh;
        rh += d;
      }
    }
    const uint32_t qd = (uint32_t)qh;
    /* P = qd * v (NV + 1 limbs), then u[j .. j+NV] -= P */
    uint32_t pl[NV + 1];
    {
      uint32_t cf = 0;
      pl[0] = qd * v[0];
      MPB_UNROLL
      for (int i = 1; i < NV; ++i) pl[i] = (i == 1) ? add_cc(qd * v[i], mulhi(qd, v[i - 1]), cf)
                                                    : addc_cc(qd * v[i], mulhi(qd, v[i - 1]), cf);
      pl[NV] = (NV == 1) ? mulhi(qd, v[NV - 1]) : addc(mulhi(qd, v[NV - 1]), 0u, cf);
    }
    uint32_t bf = 0;
    u[j] = sub_cc(u[j], pl[0], bf);
    MPB_UNROLL
    for (int i = 1; i < NV; ++i) u[j + i] = subc_cc(u[j + i], pl[i], bf);
    u[j + NV] = subc_cc(u[j + NV], pl[NV], bf);
    const uint32_t neg = subc(0u, 0u, bf); /* all ones when the result went negative */
    if (neg) { /* estimate one too large: add v back */
      qh = qd - 1u;
      uint32_t cf = 0;
      u[j] = add_cc(u[j], v[0], cf);
      MPB_UNROLL
      for (int i = 1; i < NV; ++i) u[j + i] = addc_cc(u[j + i], v[i], cf);
      u[j + NV] = addc(u[j + NV], 0u, cf);
    }
    q[j] = (uint32_t)qh;
  }
}

/* r = round(a / b), one rounding.  With A, B the significands (a = A 2^(ea-32N)),
 * Q = floor(A 2^(32(N+1)) / B) has 32(N+1) or 32(N+1)+1 bits: the top 32N
 * are the result, the next bit the round bit, the rest plus a nonzero
 * remainder the sticky bit.  b = 0 has no result in this format (no
 * infinities): r is 0. */
template <int N, int kRnd = 0>
MPB_HD void div(fval<N> &r, const fval<N> &a, const fval<N> &b) {
  if (is_zero(a) || is_zero(b)) { /* no integer division by a zero divisor */
    set_zero(r);
    return;
  }
  uint32_t u[2 * N + 2], q[N + 2];
  MPB_UNROLL
  for (int i = 0; i < 2 * N + 2; ++i) u[i] = (i >= N + 1 && i <= 2 * N) ? a.m[i - N - 1] : 0u;
  divmod_limbs<2 * N + 2, N>(q, u, b.m);
  uint32_t rem = 0u;
  MPB_UNROLL
  for (int i = 0; i < N; ++i) rem |= u[i];
  const uint32_t big = q[N + 1] & 1u; /* A >= B: one more quotient bit */
  MPB_UNROLL
  for (int i = 0; i < N; ++i) r.m[i] = big ? fshr(q[i + 1], q[i + 2], 1) : q[i + 1];
  const uint32_t rb = big ? (q[1] & 1u) : (q[0] >> 31);
  const uint32_t st = (big ? q[0] : (q[0] << 1)) | rem;
  int32_t e = a.e - b.e + (int32_t)big;
  rndn<N, kRnd>(r.m, e, rb, st);
  r.e = e;
  r.s = a.s ^ b.s;
}

/* r = round(sqrt(a)), one rounding.  With a = M 2^E (E = e - 32N), X = M 2^(2K)
 * for K = 16N + 32 (E even) or X = 2M 2^(2K) for K = 16N + 31 (E odd) lies in
 * [2^(64N+62), 2^(64N+64)), so S = floor(sqrt(X)) has exactly 32(N+1) bits.
 * S comes from the integer Newton iteration s <- (s + floor(X / s)) / 2,
 * started at or above sqrt(X) from a double-precision estimate of the top
 * 64 bits; it decreases to S and stops when it no longer decreases.  The top
 * 32N bits of S are the result, the next the round bit, the rest plus
 * S^2 != X the sticky bit.  Negative a has no result in this format: r is 0. */
template <int N, int kRnd = 0>
MPB_HD void sqrt_(fval<N> &r, const fval<N> &a) {
  constexpr int NX = 2 * N + 2, NS = N + 1;
  if (is_zero(a) || a.s) { /* the iteration below needs a nonzero root */
    set_zero(r);
    return;
  }
  const int32_t E = a.e - 32 * N;
  const uint32_t odd = (uint32_t)E & 1u;
  uint32_t x[NX + 1];
  /* X = M << (32(N+2)) (even) or M << (32(N+1) + 31) (odd) */
  MPB_UNROLL
  for (int i = 0; i < NX + 1; ++i) {
    const uint32_t even_w = (i >= N + 2 && i < 2 * N + 2) ? a.m[i - N - 2] : 0u;
    const uint32_t lo = (i >= N + 1 && i - N - 1 < N) ? a.m[i - N - 1 >= 0 ? i - N - 1 : 0] : 0u;
    const uint32_t hi = (i >= N + 2 && i - N - 2 < N) ? a.m[i - N - 2 >= 0 ? i - N - 2 : 0] : 0u;
    x[i] = odd ? fshl(hi, lo, 31) : even_w; /* limb of M << 31: (m[k] << 31) | (m[k-1] >> 1) */
  }
  /* start: t >= sqrt(top 64 bits + 1), s0 = t 2^(32N), or all ones */
  const uint64_t T = ((uint64_t)x[NX - 1] << 32) | x[NX - 2];
  uint64_t t = (uint64_t)sqrt((double)T) + 2u;
  uint32_t s[NS];
  MPB_UNROLL
  for (int i = 0; i < NS; ++i) s[i] = (t >> 32) ? 0xffffffffu : (i == NS - 1 ? (uint32_t)t : 0u);
  for (int it = 0; it < 64; ++it) {
    uint32_t u[NX + 1], qq[NX + 1 - NS];
    MPB_UNROLL
    for (int i = 0; i < NX + 1; ++i) u[i] = x[i];
    divmod_limbs<NX + 1, NS>(qq, u, s);
    /* s_new = (s + q) >> 1; q has NS + 1 limbs */
    uint32_t w[NS + 1];
    uint32_t cf = 0;
    w[0] = add_cc(s[0], qq[0], cf);
    MPB_UNROLL
    for (int i = 1; i < NS; ++i) w[i] = addc_cc(s[i], qq[i], cf);
    w[NS] = addc(0u, qq[NS], cf);
    uint32_t sn[NS];
    MPB_UNROLL
    for (int i = 0; i < NS; ++i) sn[i] = fshr(w[i], w[i + 1], 1);
    /* continue while sn < s */
    int cmp = 0;
    MPB_UNROLL
    for (int i = 0; i < NS; ++i) cmp = (sn[i] != s[i]) ? (sn[i] < s[i] ? -1 : 1) : cmp;
    if (cmp >= 0) break;
    MPB_UNROLL
    for (int i = 0; i < NS; ++i) s[i] = sn[i];
  }
  /* sticky: S^2 != X */
  uint32_t sq[2 * NS];
  mul_full<NS>(sq, s, s);
  uint32_t diff = 0u;
  MPB_UNROLL
  for (int i = 0; i < 2 * NS; ++i) diff |= sq[i] ^ (i < NX ? x[i] : 0u);
  MPB_UNROLL
  for (int i = 0; i < N; ++i) r.m[i] = s[i + 1];
  const uint32_t rb = s[0] >> 31;
  const uint32_t st = (s[0] << 1) | diff;
  int32_t e = (a.e + (int32_t)odd) >> 1; /* e/2 (E even) or (e+1)/2 (E odd), exactly */
  rndn<N, kRnd>(r.m, e, rb, st);
  r.e = e;
  r.s = 0u;
}

/* magnitude / signed compare (-1, 0, 1) */
template <int N>
MPB_HD int cmpmag(const fval<N> &a, const fval<N> &b) {
  if (a.e != b.e) return a.e > b.e ? 1 : -1;
  for (int i = N - 1; i >= 0; --i)
    if (a.m[i] != b.m[i]) return a.m[i] > b.m[i] ? 1 : -1;
  return 0;
}

/* ------------------------------------------------------------------ *
 * head word of the in-memory format: (e << 1) | s, zero = 0x80000000
 * ------------------------------------------------------------------ */
MPB_HD uint32_t pack_head(int32_t e, uint32_t s) { return ((uint32_t)e << 1) | s; }
MPB_HD int32_t head_exp(uint32_t h) { return (int32_t)h >> 1; }
MPB_HD uint32_t head_sign(uint32_t h) { return h & 1u; }
constexpr uint32_t kHeadZero = 0x80000000u;

} /* namespace mpb */

#endif /* MPB_CORE_CUH */
