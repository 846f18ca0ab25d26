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

#include "../mpb/core.cuh"

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
/* bit i of W[len], 0 outside (reference cu_freal.cuh:52-54) */
__host__ __device__ static inline cu_limb cu_wbit(const cu_limb *W, int len, long i) {
  if (i < 0 || i >= (long)len * 64) return 0;
  return (W[i >> 6] >> (i & 63)) & 1;
}
/* 1 if any of bits [0, i) of W is set (reference cu_freal.cuh:56-64) */
__host__ __device__ static inline cu_limb cu_wsticky_below(const cu_limb *W, int len, long i) {
  if (i <= 0) return 0;
  long full = i >> 6;
  cu_limb s = 0;
  for (long j = 0; j < full && j < len; j++) s |= W[j];
  int rem = (int)(i & 63);
  if (rem && full < len) s |= W[full] & ((((cu_limb)1) << rem) - 1);
  return s != 0;
}

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

  /* Round the exact magnitude D[len] (leading one at bit msb, of weight 2^Ehi,
   * with round/sticky material brnd/bsti strictly below bit 0) to P bits,
   * RNDN (reference cu_freal.cuh:83-138).  General-purpose, used by the
   * conversions; the arithmetic goes through the mpb core instead. */
  __host__ __device__ static cu_freal finalize(const cu_limb *D, int len, int msb, long Ehi,
                                               cu_limb brnd, cu_limb bsti, int sgn) {
    cu_freal r;
    if (msb < 0) {
      r.set_zero();
      return r;
    }
    const long lo = (long)msb - P + 1;
    cu_limb V[N];
    for (int i = 0; i < N; i++) { /* bits [lo + 64i, lo + 64i + 64) */
      const long pos = lo + 64L * i;
      const long w = pos >= 0 ? pos / 64 : -((-pos + 63) / 64);
      const int b = (int)(pos - 64 * w);
      const cu_limb a0 = (w >= 0 && w < len) ? D[w] : 0;
      const cu_limb a1 = (w + 1 >= 0 && w + 1 < len) ? D[w + 1] : 0;
      V[i] = b ? (a0 >> b) | (a1 << (64 - b)) : a0;
    }
    if (SB) V[N - 1] &= (((cu_limb)1) << (64 - SB)) - 1;
    cu_limb rb = 0, st = 0;
    if (lo > 0) {
      rb = cu_wbit(D, len, lo - 1);
      st = brnd | bsti | cu_wsticky_below(D, len, lo - 1);
    } else if (lo == 0) {
      rb = brnd;
      st = bsti;
    }
    long E = Ehi;
    if (rb && (st || (V[0] & 1))) {
      cu_limb c = 1;
      for (int i = 0; i < N && c; i++) {
        V[i] += c;
        c = (V[i] == 0);
      }
      const bool ov = SB ? (((V[N - 1] >> (64 - SB)) & 1) != 0) : (c != 0);
      if (ov) {
        for (int i = 0; i < N; i++) V[i] = 0;
        V[(P - 1) >> 6] = ((cu_limb)1) << ((P - 1) & 63);
        E++;
      }
    }
    for (int i = N - 1; i >= 0; i--) {
      const cu_limb hi = V[i], lo2 = (i > 0) ? V[i - 1] : 0;
      r.m[i] = SB ? (hi << SB) | (lo2 >> (64 - SB)) : hi;
    }
    r.sign = sgn;
    r.exp = E + 1;
    return r;
  }

  /* exact for PB >= 53 (reference cu_freal.cuh:141-149) */
  __host__ __device__ static cu_freal from_double(double d) {
    cu_freal r;
    if (d == 0.0) {
      r.set_zero();
      return r;
    }
    const int sgn = d < 0 ? -1 : 1;
    d = d < 0 ? -d : d;
    int k;
    const double f = frexp(d, &k);
    cu_limb F = (cu_limb)ldexp(f, 53);
    return finalize(&F, 1, 52, (long)k - 1, 0, 0, sgn);
  }
  /* RNDN to 53 bits (reference cu_freal.cuh:150-165) */
  __host__ __device__ double to_double() const {
    if (is_zero()) return 0.0;
    const int hb = N * 64 - 53;
    const int w = hb >> 6, b = hb & 63;
    cu_limb F = b ? (m[w] >> b) | (w + 1 < N ? m[w + 1] << (64 - b) : 0) : m[w];
    const cu_limb rbit = cu_wbit(m, N, hb - 1);
    const cu_limb sticky = cu_wsticky_below(m, N, hb - 1);
    long e = exp;
    if (rbit && (sticky || (F & 1))) {
      F++;
      if (F == (1ULL << 53)) {
        F >>= 1;
        e++;
      }
    }
    return (double)sign * ldexp((double)F, (int)(e - 53));
  }

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
template <int PB>
__host__ __device__ inline cu_freal<PB> from_core(const typename core_of<PB>::type &r) {
  typedef core_of<PB> C;
  cu_freal<PB> x;
  if (mpb::is_zero(r)) {
    x.set_zero();
    return x;
  }
  for (int k = 0; k < cu_freal<PB>::N; k++) {
    const int lo = 2 * k - C::OFF, hi = 2 * k + 1 - C::OFF;
    const cu_limb l = (lo >= 0 && lo < C::N32) ? r.m[lo] : 0u;
    const cu_limb h = (hi >= 0 && hi < C::N32) ? r.m[hi] : 0u;
    x.m[k] = (h << 32) | l;
  }
  x.exp = r.e;
  x.sign = r.s ? -1 : 1;
  return x;
}
}  // namespace detail

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

/* magnitude compare (reference cu_cmpmag, cu_freal.cuh:215-222) */
template <int PB>
__host__ __device__ static int cu_cmpmag(const cu_freal<PB> &a, const cu_freal<PB> &b) {
  if (a.exp != b.exp) return a.exp > b.exp ? 1 : -1;
  for (int i = cu_freal<PB>::N - 1; i >= 0; i--)
    if (a.m[i] != b.m[i]) return a.m[i] > b.m[i] ? 1 : -1;
  return 0;
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
template <int PB>
__host__ __device__ static int cu_cmp(const cu_freal<PB> &a, const cu_freal<PB> &b) {
  if (a.is_zero() && b.is_zero()) return 0;
  if (a.is_zero()) return b.sign > 0 ? -1 : 1;
  if (b.is_zero()) return a.sign > 0 ? 1 : -1;
  if (a.sign != b.sign) return a.sign > 0 ? 1 : -1;
  const int m = cu_cmpmag<PB>(a, b);
  return a.sign > 0 ? m : -m;
}
/* re-round to another precision, exact when widening (reference cu_freal.cuh:316-323) */
template <int TO, int FROM>
__host__ __device__ static inline cu_freal<TO> cu_convert(const cu_freal<FROM> &x) {
  if (x.is_zero()) {
    cu_freal<TO> r;
    r.set_zero();
    return r;
  }
  return cu_freal<TO>::finalize(x.m, cu_freal<FROM>::N, cu_freal<FROM>::N * 64 - 1, x.exp - 1, 0, 0, x.sign);
}
/* exact small integer (reference cu_freal.cuh:325-334) */
template <int PB>
__host__ __device__ static cu_freal<PB> cu_from_si(long v) {
  cu_freal<PB> r;
  if (v == 0) {
    r.set_zero();
    return r;
  }
  const int sgn = v < 0 ? -1 : 1;
  unsigned long long a = v < 0 ? (unsigned long long)(-(v + 1)) + 1ULL : (unsigned long long)v;
  int nb = 64;
  while (!((a >> (nb - 1)) & 1)) nb--;
  return cu_freal<PB>::finalize(&a, 1, nb - 1, (long)nb - 1, 0, 0, sgn);
}
/* round to nearest integer, ties to even (reference cu_freal.cuh:336-356) */
template <int PB>
__host__ __device__ static long cu_lround(const cu_freal<PB> &x) {
  if (x.is_zero()) return 0;
  const int N = cu_freal<PB>::N;
  const long e = x.exp;
  if (e <= 0) {
    if (e == 0) {
      bool half = (x.m[N - 1] == (1ULL << 63));
      for (int i = 0; i < N - 1; i++) half &= (x.m[i] == 0);
      const long r = half ? 0 : 1;
      return x.sign < 0 ? -r : r;
    }
    return 0;
  }
  unsigned long long ip = 0;
  for (long b = 0; b < e; b++) {
    const long bit = (long)N * 64 - e + b;
    ip |= ((x.m[bit >> 6] >> (bit & 63)) & 1ULL) << b;
  }
  const long rb = (long)N * 64 - e - 1;
  const unsigned long long rbit = rb >= 0 ? ((x.m[rb >> 6] >> (rb & 63)) & 1ULL) : 0;
  const unsigned long long st = cu_wsticky_below(x.m, N, rb);
  if (rbit && (st || (ip & 1))) ip++;
  const long r = (long)ip;
  return x.sign < 0 ? -r : r;
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
