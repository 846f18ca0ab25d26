/* mpc_cuda/cu_freal.cuh -- drop-in cu_fp::cu_freal<PB> for the mpb engine.
 *
 * Same names, struct layout, operators and semantics as the mpc_cuda header of
 * the same path (reference include/mpc_cuda/cu_freal.cuh:34-366):
 *
 *   template<int PB> struct cu_freal { int sign; long exp; cu_limb m[N]; };
 *   value = sign * M * 2^(exp - 64N), M left-justified in N = ceil(PB/64)
 *   64-bit limbs, low SB = 64N-PB bits zero, zero = exp == CU_FREAL_ZERO_EXP.
 *
 * so AoS buffers of cu_freal<PB> written by code built against the reference
 * are read unchanged.  Every arithmetic operation is bit-exact with MPFR RNDN
 * (the reference's contract, cu_freal.cuh:1-16).  The arithmetic itself is
 * the mpb core (mpb/core.cuh): 32-bit limbs, PTX carry chains, and shift
 * networks unrolled at compile time instead of the reference's runtime-indexed
 * local arrays, so on sm_100a the operands stay in registers.  Added over the
 * reference: cu_ffma (one rounding of a*b+c, MPFR mpfr_fma semantics).
 *
 * Exponents are carried in 32 bits inside the core: values must stay inside
 * MPFR's default exponent range |exp| < 2^30 (the reference uses a 64-bit
 * exponent without a range check; MPFR's own default range is the same bound).
 */
#ifndef MPB_DROPIN_CU_FREAL_CUH
#define MPB_DROPIN_CU_FREAL_CUH

#include <cmath>
#include <cstdint>

#include "../mpb/rprec.cuh"

#if !defined(__CUDACC__)
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#endif

namespace cu_fp {

typedef unsigned long long cu_limb;
#define CU_FREAL_ZERO_EXP (-0x7fffffffffffffLL)

/* 64x64 -> 128 (reference cu_freal.cuh:39-49) */
__host__ __device__ static inline void cu_umul(cu_limb &hi, cu_limb &lo, cu_limb a, cu_limb b) {
#if defined(__CUDA_ARCH__)
  lo = a * b;
  hi = __umul64hi(a, b);
#else
  __uint128_t p = (__uint128_t)a * b;
  lo = (cu_limb)p;
  hi = (cu_limb)(p >> 64);
#endif
}
/* bit i of the little-endian limb array W[len]; bits outside it read as 0
 * (reference cu_freal.cuh:52-54) */
__host__ __device__ static inline cu_limb cu_wbit(const cu_limb *W, int len, long i) {
  const unsigned long u = (unsigned long)i; /* negative i wraps to a huge index */
  return u < 64ul * (unsigned long)len ? (W[u / 64] >> (u % 64)) & 1ull : 0ull;
}
/* 1 when some bit of W below position i is set, else 0 (reference
 * cu_freal.cuh:56-64): every limb is masked to the part of it that lies
 * below i and the masked limbs are ORed */
__host__ __device__ static inline cu_limb cu_wsticky_below(const cu_limb *W, int len, long i) {
  cu_limb any = 0;
  for (int j = 0; j < len; j++) {
    const long below = i - 64L * j; /* bits of limb j under position i */
    if (below <= 0) break;
    any |= below >= 64 ? W[j] : W[j] & ~(~0ull << below);
  }
  return any ? 1ull : 0ull;
}

template <int PB>
struct cu_freal;

namespace detail {
/* limb i of D[len], 0 outside the array */
__host__ __device__ inline cu_limb limb_or0(const cu_limb *D, int len, long i) {
  return (i >= 0 && i < len) ? D[i] : 0ull;
}
/* the 32 bits [pos, pos + 32) of the magnitude D[len] (64-bit limbs); bits
 * outside [0, 64 len) read as 0 */
__host__ __device__ inline uint32_t dbits32(const cu_limb *D, int len, long pos) {
  if (pos <= -32) return 0u;
  if (pos < 0) return (uint32_t)(limb_or0(D, len, 0) << (-pos));
  const long w = pos >> 6;
  const int b = (int)(pos & 63);
  const cu_limb lo = limb_or0(D, len, w), hi = limb_or0(D, len, w + 1);
  return (uint32_t)(b ? (lo >> b) | (hi << (64 - b)) : lo);
}
}  // namespace detail

template <int PB>
struct cu_freal {
  static_assert(PB > 0 && (PB % 32) == 0, "PB must be a positive multiple of 32");
  static const int P = PB;
  static const int N = (PB + 63) / 64;
  static const int SB = N * 64 - PB;

  int sign;
  long exp;
  cu_limb m[N];

  __host__ __device__ bool is_zero() const { return exp == CU_FREAL_ZERO_EXP; }
  __host__ __device__ void set_zero() {
    sign = 1;
    exp = CU_FREAL_ZERO_EXP;
    for (int i = 0; i < N; i++) m[i] = 0;
  }

  /* Round a magnitude to PB bits, RNDN, and give it the sign sgn (the
   * argument meaning of the reference's finalize, cu_freal.cuh:83-138):
   * D[len] holds the significant bits (little-endian 64-bit limbs), its
   * leading one at bit msb (msb < 0: the value is zero) with weight 2^Ehi,
   * and brnd / bsti are the round bit and the sticky bit of what lies below
   * D's bit 0 (used only when the result's last bit is at or above D's bit 0;
   * a result with fewer than PB significant bits in D is exact).
   * The PB bits under the leading one are read as PB/32 words of the mpb
   * core, rounded there (mpb::rndn) and packed into the 64-bit limbs. */
  __host__ __device__ static cu_freal finalize(const cu_limb *D, int len, int msb, long Ehi, cu_limb brnd,
                                               cu_limb bsti, int sgn);

  /* exact for PB >= 53, rounded to PB bits below that (reference cu_freal.cuh:141-149) */
  __host__ __device__ static cu_freal from_double(double d);
  /* RNDN to 53 bits (reference cu_freal.cuh:150-165) */
  __host__ __device__ double to_double() const;

  __host__ __device__ cu_freal() {}
  __host__ __device__ cu_freal(double d) { *this = from_double(d); }
  __host__ __device__ explicit operator double() const { return to_double(); }
};

/* ---------------- bridge to the mpb core (32-bit limbs) ---------------- */
namespace detail {
template <int PB>
struct core_of {
  static const int N32 = PB / 32;
  static const int OFF = cu_freal<PB>::SB / 32; /* zero low 32-bit halves */
  typedef mpb::fval<N32> type;
};
/* 32-bit half k of a 64-bit limb array */
__host__ __device__ inline uint32_t half32(const cu_limb *m, int n64, int k) {
  return (k >= 0 && k < 2 * n64) ? (uint32_t)(m[k >> 1] >> (32 * (k & 1))) : 0u;
}
template <int PB>
__host__ __device__ inline void to_core(typename core_of<PB>::type &r, const cu_freal<PB> &x) {
  typedef core_of<PB> C;
  if (x.is_zero()) {
    mpb::set_zero(r);
    return;
  }
  for (int i = 0; i < C::N32; i++) r.m[i] = half32(x.m, cu_freal<PB>::N, i + C::OFF);
  r.e = (int32_t)x.exp;
  r.s = x.sign < 0 ? 1u : 0u;
}
/* the core words of r in the 64-bit limbs of x (the low SB bits stay 0) */
template <int PB>
__host__ __device__ inline void pack_limbs(cu_freal<PB> &x, const typename core_of<PB>::type &r) {
  typedef core_of<PB> C;
  for (int k = 0; k < cu_freal<PB>::N; k++) {
    const int lo = 2 * k - C::OFF, hi = 2 * k + 1 - C::OFF;
    const cu_limb l = (lo >= 0 && lo < C::N32) ? r.m[lo] : 0u;
    const cu_limb h = (hi >= 0 && hi < C::N32) ? r.m[hi] : 0u;
    x.m[k] = (h << 32) | l;
  }
}
template <int PB>
__host__ __device__ inline cu_freal<PB> from_core(const typename core_of<PB>::type &r) {
  cu_freal<PB> x;
  if (mpb::is_zero(r)) {
    x.set_zero();
    return x;
  }
  pack_limbs<PB>(x, r);
  x.exp = r.e;
  x.sign = r.s ? -1 : 1;
  return x;
}
}  // namespace detail

/* ---------------- conversions through the core ---------------- */
namespace detail {
/* r = sign s, a left-justified 64-bit magnitude T (bit 63 set) times
 * 2^(e - 64), rounded to the core's N words (only N = 1 loses bits) */
template <int N>
__host__ __device__ inline void from_top64(mpb::fval<N> &r, uint64_t T, int32_t e, uint32_t s) {
  for (int i = 0; i < N; i++) r.m[i] = 0u;
  r.m[N - 1] = (uint32_t)(T >> 32);
  uint32_t rb = 0u, st = 0u;
  if (N >= 2)
    r.m[N - 2] = (uint32_t)T;
  else {
    rb = (uint32_t)(T >> 31) & 1u;
    st = (uint32_t)T & 0x7fffffffu;
  }
  r.e = e;
  r.s = s;
  mpb::rndn<N>(r.m, r.e, rb, st);
}
/* the core value x rounded (RNDN) or widened (exactly) to NT words */
template <int NT, int NF>
__host__ __device__ inline void resize(mpb::fval<NT> &r, const mpb::fval<NF> &x) {
  if (mpb::is_zero(x)) {
    mpb::set_zero(r);
    return;
  }
  /* word i of r is word i + NF - NT of x (0 below x) */
  for (int i = 0; i < NT; i++) r.m[i] = (i + NF - NT >= 0) ? x.m[i + NF - NT] : 0u;
  r.e = x.e;
  r.s = x.s;
  if (NT < NF) {
    const uint32_t g = x.m[NF - NT - 1];
    uint32_t st = g << 1;
    for (int i = 0; i < NF - NT - 1; i++) st |= x.m[i];
    mpb::rndn<NT>(r.m, r.e, g >> 31, st);
  }
}
}  // namespace detail

template <int PB>
__host__ __device__ cu_freal<PB> cu_freal<PB>::finalize(const cu_limb *D, int len, int msb, long Ehi, cu_limb brnd,
                                                        cu_limb bsti, int sgn) {
  typedef typename detail::core_of<PB>::type V;
  const int NW = detail::core_of<PB>::N32;
  if (msb < 0) {
    cu_freal r;
    r.set_zero();
    return r;
  }
  /* word NW-1-w of the result holds D's bits [msb - 32 w - 31, msb - 32 w] */
  V v;
  for (int w = 0; w < NW; w++) v.m[NW - 1 - w] = detail::dbits32(D, len, (long)msb - 32L * w - 31);
  const long last = (long)msb - PB + 1; /* D position of the result's last bit */
  uint32_t rb = 0u, st = 0u;
  if (last > 0) { /* the round bit is a bit of D; D's lower bits and brnd/bsti are sticky */
    rb = (uint32_t)cu_wbit(D, len, last - 1);
    st = (uint32_t)(cu_wsticky_below(D, len, last - 1) | brnd | bsti);
  } else if (last == 0) { /* the round bit is the bit just under D */
    rb = (uint32_t)(brnd & 1ull);
    st = (uint32_t)(bsti != 0ull);
  } /* last < 0: every significant bit fits, the value is exact */
  v.e = (int32_t)(Ehi + 1);
  v.s = sgn < 0 ? 1u : 0u;
  const int32_t e0 = v.e;
  mpb::rndn<NW>(v.m, v.e, rb, st);
  cu_freal r;
  detail::pack_limbs<PB>(r, v);
  r.exp = (long)Ehi + 1 + (long)(v.e - e0); /* the 64-bit exponent, plus the rounding's carry */
  r.sign = sgn;
  return r;
}

template <int PB>
__host__ __device__ cu_freal<PB> cu_freal<PB>::from_double(double d) {
  typename detail::core_of<PB>::type v;
  if (d == 0.0) {
    mpb::set_zero(v);
    return detail::from_core<PB>(v);
  }
  int k;
  const double f = frexp(fabs(d), &k);                     /* |d| = f 2^k, f in [1/2, 1) */
  const uint64_t F = (uint64_t)ldexp(f, 64);               /* f's 53 bits, left-justified */
  detail::from_top64(v, F, (int32_t)k, d < 0 ? 1u : 0u);
  return detail::from_core<PB>(v);
}

template <int PB>
__host__ __device__ double cu_freal<PB>::to_double() const {
  if (is_zero()) return 0.0;
  const int NW = detail::core_of<PB>::N32;
  typename detail::core_of<PB>::type v;
  detail::to_core<PB>(v, *this);
  if (PB > 53) mpb::round_to_bits<NW>(v, 53); /* the nearest 53-bit value */
  /* the value is (top two words) * 2^(e - 64); for PB = 32 only one word */
  const uint64_t T = ((uint64_t)v.m[NW - 1] << 32) | (NW >= 2 ? v.m[NW - 2] : 0u);
  const double mag = ldexp((double)T, v.e - 64); /* T has at most 53 significant bits: exact */
  return sign < 0 ? -mag : mag;
}

/* N x N -> 2N (64-bit limbs) exact product (reference cu_freal.cuh:173-200) */
template <int PB>
__host__ __device__ static void cu_mul_full(cu_limb r[2 * cu_freal<PB>::N], const cu_limb a[cu_freal<PB>::N],
                                            const cu_limb b[cu_freal<PB>::N]) {
  const int N = cu_freal<PB>::N;
  uint32_t a32[2 * N], b32[2 * N], p32[4 * N];
  for (int k = 0; k < 2 * N; k++) {
    a32[k] = detail::half32(a, N, k);
    b32[k] = detail::half32(b, N, k);
  }
  mpb::mul_full<2 * N>(p32, a32, b32);
  for (int k = 0; k < 2 * N; k++) r[k] = ((cu_limb)p32[2 * k + 1] << 32) | p32[2 * k];
}

/* round(a*b) (reference cu_fmul, cu_freal.cuh:202-213) */
template <int PB>
__host__ __device__ static cu_freal<PB> cu_fmul(const cu_freal<PB> &a, const cu_freal<PB> &b) {
  typename detail::core_of<PB>::type x, y, r;
  detail::to_core<PB>(x, a);
  detail::to_core<PB>(y, b);
  mpb::mul(r, x, y);
  return detail::from_core<PB>(r);
}

/* magnitude compare, -1 / 0 / 1 (reference cu_cmpmag, cu_freal.cuh:215-222):
 * the exponents first, then the significands word by word from the top, by
 * the core */
template <int PB>
__host__ __device__ static int cu_cmpmag(const cu_freal<PB> &a, const cu_freal<PB> &b) {
  typename detail::core_of<PB>::type x, y;
  detail::to_core<PB>(x, a);
  detail::to_core<PB>(y, b);
  if (a.is_zero() || b.is_zero()) return (int)!a.is_zero() - (int)!b.is_zero(); /* zero is the smallest */
  return mpb::cmpmag(x, y);
}

/* round(|a| + |b|) with sign sgn (reference cu_addmag, cu_freal.cuh:224-245) */
template <int PB>
__host__ __device__ static cu_freal<PB> cu_addmag(cu_freal<PB> a, cu_freal<PB> b, int sgn) {
  a.sign = 1;
  b.sign = 1;
  typename detail::core_of<PB>::type x, y, r;
  detail::to_core<PB>(x, a);
  detail::to_core<PB>(y, b);
  mpb::add(r, x, y);
  cu_freal<PB> o = detail::from_core<PB>(r);
  if (!o.is_zero()) o.sign = sgn;
  return o;
}
/* round(|a| - |b|), |a| > |b|, sign sgn (reference cu_submag, cu_freal.cuh:247-277) */
template <int PB>
__host__ __device__ static cu_freal<PB> cu_submag(const cu_freal<PB> &a, const cu_freal<PB> &b, int sgn) {
  typename detail::core_of<PB>::type x, y, r;
  detail::to_core<PB>(x, a);
  detail::to_core<PB>(y, b);
  x.s = 0u;
  y.s = 0u;
  mpb::sub(r, x, y);
  cu_freal<PB> o = detail::from_core<PB>(r);
  if (!o.is_zero()) o.sign = sgn;
  return o;
}

/* round(a + b), round(a - b) (reference cu_fadd/cu_fsub, cu_freal.cuh:279-292) */
template <int PB>
__host__ __device__ static cu_freal<PB> cu_fadd(const cu_freal<PB> &a, const cu_freal<PB> &b) {
  typename detail::core_of<PB>::type x, y, r;
  detail::to_core<PB>(x, a);
  detail::to_core<PB>(y, b);
  mpb::add(r, x, y);
  return detail::from_core<PB>(r);
}
template <int PB>
__host__ __device__ static cu_freal<PB> cu_fsub(const cu_freal<PB> &a, cu_freal<PB> b) {
  typename detail::core_of<PB>::type x, y, r;
  detail::to_core<PB>(x, a);
  detail::to_core<PB>(y, b);
  mpb::sub(r, x, y);
  return detail::from_core<PB>(r);
}
/* round(a*b + c), a single rounding (MPFR mpfr_fma semantics; not in the reference) */
template <int PB>
__host__ __device__ static cu_freal<PB> cu_ffma(const cu_freal<PB> &a, const cu_freal<PB> &b,
                                                const cu_freal<PB> &c) {
  typename detail::core_of<PB>::type x, y, z, r;
  detail::to_core<PB>(x, a);
  detail::to_core<PB>(y, b);
  detail::to_core<PB>(z, c);
  mpb::fma(r, x, y, z);
  return detail::from_core<PB>(r);
}

/* utilities (reference cu_freal.cuh:294-356) */
template <int PB>
__host__ __device__ static inline cu_freal<PB> cu_neg(cu_freal<PB> a) {
  if (!a.is_zero()) a.sign = -a.sign;
  return a;
}
template <int PB>
__host__ __device__ static inline cu_freal<PB> cu_abs(cu_freal<PB> a) {
  if (!a.is_zero()) a.sign = 1;
  return a;
}
template <int PB>
__host__ __device__ static inline cu_freal<PB> cu_scale2(cu_freal<PB> a, long k) {
  if (!a.is_zero()) a.exp += k;
  return a;
}
template <int PB>
__host__ __device__ static inline int cu_sgn(const cu_freal<PB> &a) {
  return a.is_zero() ? 0 : a.sign;
}
/* signed compare, -1 / 0 / 1 (reference cu_cmp, cu_freal.cuh:304-314):
 * values of different signs (zero counting as sign 0) order by their sign;
 * equal signs by magnitude, reversed for negative values */
template <int PB>
__host__ __device__ static int cu_cmp(const cu_freal<PB> &a, const cu_freal<PB> &b) {
  const int sa = cu_sgn<PB>(a), sb = cu_sgn<PB>(b);
  if (sa != sb) return sa < sb ? -1 : 1;
  return sa * cu_cmpmag<PB>(a, b); /* 0 when both are zero */
}
/* the value at another precision: widened exactly or rounded to nearest-even
 * (reference cu_convert, cu_freal.cuh:316-323), through the core words */
template <int TO, int FROM>
__host__ __device__ static inline cu_freal<TO> cu_convert(const cu_freal<FROM> &x) {
  typename detail::core_of<FROM>::type v;
  typename detail::core_of<TO>::type r;
  detail::to_core<FROM>(v, x);
  detail::resize(r, v);
  return detail::from_core<TO>(r);
}
/* an integer, exact from PB = 64 up and rounded to nearest below (reference
 * cu_from_si, cu_freal.cuh:325-334): the magnitude is left-justified by its
 * leading-zero count and handed to the core */
template <int PB>
__host__ __device__ static cu_freal<PB> cu_from_si(long v) {
  typename detail::core_of<PB>::type r;
  if (v == 0) {
    mpb::set_zero(r);
    return detail::from_core<PB>(r);
  }
  const uint64_t mag = v < 0 ? 0ull - (uint64_t)v : (uint64_t)v; /* |v|, LONG_MIN included */
  int lz = 0;
  while (!((mag << lz) >> 63)) lz++;
  detail::from_top64(r, mag << lz, (int32_t)(64 - lz), v < 0 ? 1u : 0u);
  return detail::from_core<PB>(r);
}
/* the nearest integer, ties to even (reference cu_lround, cu_freal.cuh:336-356;
 * |x| must stay below 2^62 as there): with MPFR exponent e, |x| < 2^e, so
 * rounding the significand to its top e bits (the core's round_to_bits) leaves
 * the integer in those bits; e <= 0 means |x| < 1/2 (0) or, for e = 0,
 * |x| in [1/2, 1), which is 1 except for the tie 1/2 (0, the even neighbour) */
template <int PB>
__host__ __device__ static long cu_lround(const cu_freal<PB> &x) {
  if (x.is_zero() || x.exp < 0) return 0;
  const int NW = detail::core_of<PB>::N32;
  typename detail::core_of<PB>::type v;
  detail::to_core<PB>(v, x);
  long mag;
  if (x.exp == 0) {
    bool tie = v.m[NW - 1] == 0x80000000u;
    for (int i = 0; i < NW - 1; i++) tie = tie && v.m[i] == 0u;
    mag = tie ? 0 : 1;
  } else {
    if (x.exp < PB) mpb::round_to_bits<NW>(v, (int)x.exp); /* may carry: v.e = e + 1 */
    const uint64_t T = ((uint64_t)v.m[NW - 1] << 32) | (NW >= 2 ? v.m[NW - 2] : 0u);
    mag = v.e >= 64 ? (long)T : (long)(T >> (64 - v.e)); /* the top v.e bits */
  }
  return x.sign < 0 ? -mag : mag;
}

/* operators (reference cu_freal.cuh:358-364) */
template <int PB>
__host__ __device__ static inline cu_freal<PB> operator*(const cu_freal<PB> &a, const cu_freal<PB> &b) {
  return cu_fmul<PB>(a, b);
}
template <int PB>
__host__ __device__ static inline cu_freal<PB> operator+(const cu_freal<PB> &a, const cu_freal<PB> &b) {
  return cu_fadd<PB>(a, b);
}
template <int PB>
__host__ __device__ static inline cu_freal<PB> operator-(const cu_freal<PB> &a, const cu_freal<PB> &b) {
  return cu_fsub<PB>(a, b);
}

} /* namespace cu_fp */

#endif /* MPB_DROPIN_CU_FREAL_CUH */
