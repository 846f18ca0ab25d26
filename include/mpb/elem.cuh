/* mpb/elem.cuh -- elementary functions on the mpb core (host and device).
 *
 * Faithful (at most 1 ULP from the exact value; in practice almost always the
 * correctly rounded one), the contract of the reference's cu_fmath /
 * cu_fcmath functions (mpc_cuda include/mpc_cuda/cu_fmath.cuh:1-14,
 * cu_fcmath.cuh:1-5).  Every function widens its N-limb operands exactly to
 * NW = N + 4 limbs (128 guard bits), computes there with the core's
 * correctly rounded operations and rounds once to N limbs at the end.
 *
 *   expm1 core  |r| < 1: r' = r / 2^s, expm1(r') by its Taylor series in
 *               Horner form (1 + r' h / i, the division by the small integer
 *               i is O(NW)), then s doublings e <- e (e + 2) (expm1(2y) =
 *               expm1(y) (expm1(y) + 2)); the relative error grows only
 *               linearly in s, s ~ sqrt(38 NW) balances terms and doublings.
 *   exp         x = k ln2 + r (k from a double estimate), 2^k (1 + expm1(r)).
 *   log         x = m 2^e with m in [1/sqrt2, sqrt2); near 1, log m =
 *               2 atanh((m-1)/(m+1)) directly; elsewhere log m = y0 +
 *               log(m exp(-y0)) with y0 = log m in double, the second term
 *               from a few atanh terms; then + e ln2.
 *   sin/cos/tan x = k pi/2 + r with pi carried at 2N + 4 limbs and the exact
 *               difference rounded once, so that r keeps its relative
 *               accuracy even when x is close to a multiple of pi/2; then
 *               sin and 1 - cos of r / 2^s by their series and s doublings
 *               (sin 2y = 2 sin y cos y, 1 - cos 2y = 2 sin^2 y).
 *   atan        1/x above 1 (then pi/2 - .); atan a = y0 + atan w with
 *               y0 = atan a in double and w = tan(atan a - y0) from sin / cos
 *               of y0, a few terms of the alternating odd series.
 *   others      from these: asin, acos, atanh, sinh, cosh, expm1, log1p,
 *               pow, cbrt (Newton), atan2 and the complex functions.
 *
 * ln 2 and pi come from consts.cuh (generated by make_consts.py).  Results
 * with no value in this format -- no NaN or infinity: exp / sinh / cosh of
 * |x| >= 2^29, sin / cos / tan of |x| >= 2^30, log / log1p outside their
 * domain, atanh of |x| >= 1, pow of a negative base and a non-integer
 * exponent, a complex division by zero -- are 0.
 */
#ifndef MPB_ELEM_CUH
#define MPB_ELEM_CUH

#include "core.cuh"
#include "consts.cuh"

namespace mpb {

/* ------------------------------------------------------------------ *
 * compile-time parameters of the series
 * ------------------------------------------------------------------ */
constexpr int ilog2_floor(uint32_t v) { return v <= 1u ? 0 : 1 + ilog2_floor(v >> 1); }
constexpr int isqrt_step(int v, int r) { return (r + 1) * (r + 1) <= v ? isqrt_step(v, r + 1) : r; }
constexpr int isqrt_floor(int v) { return isqrt_step(v, 0); }

/* expm1: argument halvings and Taylor terms (|r'| < 2^-s, the term ratio
 * r'/i, the product of ratios 2..T at least 2^-(32 NW + 8)) */
constexpr int em1_halvings(int NW) { return isqrt_floor(38 * NW); }
constexpr int em1_terms_from(int T, int bits, int need, int s) {
  return bits >= need ? T : em1_terms_from(T + 1, bits + s + ilog2_floor((uint32_t)(T + 1)), need, s);
}
constexpr int em1_terms(int NW) { return em1_terms_from(1, 0, 32 * NW + 8, em1_halvings(NW)); }

/* sin / 1 - cos: halvings and terms (ratio r'^2 / ((2i)(2i+1))) */
constexpr int sc_halvings(int NW) { return (9 * isqrt_floor(NW) - 5) / 2 < 4 ? 4 : (9 * isqrt_floor(NW) - 5) / 2; }
constexpr int sc_terms_from(int T, int bits, int need, int s) {
  return bits >= need ? T
                      : sc_terms_from(T + 1, bits + 2 * s + ilog2_floor((uint32_t)((2 * T + 2) * (2 * T + 3))), need, s);
}
constexpr int sc_terms(int NW) { return sc_terms_from(0, 0, 32 * NW + 8, sc_halvings(NW)); }

/* log / log1p / atanh: arguments below 2^-kNearBits (from 1, for log) go
 * straight to the atanh series */
constexpr int kNearBits = 12;
/* odd series sum z^(2i) / (2i+1), |z| < 2^-ZB: the first omitted term is
 * below 2^-(32 NW + 8) */
constexpr int odd_terms(int NW, int ZB) { return (32 * NW + 8 + 2 * ZB - 1) / (2 * ZB); }

/* ------------------------------------------------------------------ *
 * conversions and constants
 * ------------------------------------------------------------------ */
template <int NW>
MPB_HD void from_i32(fval<NW> &r, int32_t k) {
  MPB_UNROLL
  for (int i = 0; i < NW; ++i) r.m[i] = 0u;
  if (k == 0) {
    r.e = kExpZero;
    r.s = 0u;
    return;
  }
  const uint32_t a = k < 0 ? 0u - (uint32_t)k : (uint32_t)k;
  const uint32_t lz = clz32(a);
  r.m[NW - 1] = a << lz;
  r.e = 32 - (int32_t)lz;
  r.s = k < 0 ? 1u : 0u;
}

/* exact conversion of an unsigned 64-bit integer */
template <int NW>
MPB_HD void from_u64(fval<NW> &r, uint64_t v) {
  static_assert(NW >= 2, "a 64-bit integer needs two limbs");
  MPB_UNROLL
  for (int i = 0; i < NW; ++i) r.m[i] = 0u;
  r.s = 0u;
  if (v == 0u) {
    r.e = kExpZero;
    return;
  }
  const uint32_t hi = (uint32_t)(v >> 32);
  const int lz = hi ? (int)clz32(hi) : 32 + (int)clz32((uint32_t)v);
  const uint64_t m = v << lz;
  r.m[NW - 1] = (uint32_t)(m >> 32);
  r.m[NW - 2] = (uint32_t)m;
  r.e = 64 - lz;
}

/* exact conversion of a finite double */
template <int NW>
MPB_HD void from_dbl(fval<NW> &r, double v) {
  MPB_UNROLL
  for (int i = 0; i < NW; ++i) r.m[i] = 0u;
  if (v == 0.0) {
    r.e = kExpZero;
    r.s = 0u;
    return;
  }
  int k;
  const double f = frexp(v < 0 ? -v : v, &k);
  const uint64_t M = (uint64_t)ldexp(f, 64); /* f in [0.5, 1): top bit set, 53 bits */
  r.m[NW - 1] = (uint32_t)(M >> 32);
  if (NW >= 2) r.m[NW >= 2 ? NW - 2 : 0] = (uint32_t)M;
  r.e = k;
  r.s = v < 0 ? 1u : 0u;
}

/* the top 64 bits as a fraction in [0.5, 1) */
template <int NW>
MPB_HD double top_fraction(const fval<NW> &x) {
  const uint64_t m = ((uint64_t)x.m[NW - 1] << 32) | (NW >= 2 ? x.m[NW >= 2 ? NW - 2 : 0] : 0u);
  return ldexp((double)m, -64);
}

/* the value as a double (no range check: |exponent| stays small where used) */
template <int NW>
MPB_HD double to_dbl_approx(const fval<NW> &x) {
  return is_zero(x) ? 0.0 : ldexp(top_fraction<NW>(x), x.e) * (x.s ? -1.0 : 1.0);
}

template <int N, int NW>
MPB_HD void widen(fval<NW> &r, const fval<N> &x) {
  MPB_UNROLL
  for (int i = 0; i < NW; ++i) r.m[i] = (i >= NW - N) ? x.m[i - (NW - N)] : 0u;
  r.e = x.e;
  r.s = x.s;
}

template <int NW, int N>
MPB_HD void narrow(fval<N> &r, const fval<NW> &x) {
  uint32_t z[NW];
  MPB_UNROLL
  for (int i = 0; i < NW; ++i) z[i] = 0u;
  add_round<NW, N>(r, x.m, x.e, x.s, z, kExpZero, 0u);
}

template <int NW>
MPB_HD void ln2_w(fval<NW> &r) {
  static_assert(NW <= kLn2WordCount, "precision above the ln 2 table");
  MPB_UNROLL
  for (int i = 0; i < NW; ++i) r.m[i] = ln2_word(kLn2WordCount - NW + i);
  r.e = 0;
  r.s = 0u;
}

/* pi * 2^(e - 2): e = 2 gives pi, 1 pi/2, 0 pi/4 */
template <int NW>
MPB_HD void pi_w(fval<NW> &r, int32_t e) {
  static_assert(NW <= kPiWordCount, "precision above the pi table");
  MPB_UNROLL
  for (int i = 0; i < NW; ++i) r.m[i] = pi_word(kPiWordCount - NW + i);
  r.e = e;
  r.s = 0u;
}

template <int NW>
MPB_HD void one_w(fval<NW> &r) {
  from_i32<NW>(r, 1);
}

template <int NW>
MPB_HD void neg_w(fval<NW> &x) {
  if (!is_zero(x)) x.s ^= 1u;
}

/* ------------------------------------------------------------------ *
 * division by a small integer, exact products by one
 * ------------------------------------------------------------------ */
/* r = round(a / D) for a positive integer D of NV limbs (top limb nonzero),
 * one rounding.  Q = floor(A 2^(32(NV+1)) / D) comes from the long division
 * by D 2^sh, normalised (numerator shifted alike); Q >= 2^(32N+31), so its
 * top 32N bits are the result, the next the round bit and the rest plus a
 * nonzero remainder the sticky bit -- O(N NV) work. */
template <int N, int NV>
MPB_HD void div_int(fval<N> &r, const fval<N> &a, const uint32_t *d) {
  constexpr int NU = N + NV + 2;
  const uint32_t sh = clz32(d[NV - 1]);
  uint32_t v[NV], u[NU], q[N + 2];
  MPB_UNROLL
  for (int i = 0; i < NV; ++i) v[i] = fshl(i > 0 ? d[i > 0 ? i - 1 : 0] : 0u, d[i], sh);
  MPB_UNROLL
  for (int i = 0; i < NV + 1; ++i) u[i] = 0u;
  MPB_UNROLL
  for (int i = 0; i < N; ++i) u[NV + 1 + i] = fshl(i > 0 ? a.m[i > 0 ? i - 1 : 0] : 0u, a.m[i], sh);
  u[NU - 1] = fshl(a.m[N - 1], 0u, sh);
  divmod_limbs<NU, NV>(q, u, v);
  uint32_t rem = 0u;
  MPB_UNROLL
  for (int i = 0; i < NV; ++i) rem |= u[i];
  const bool hi = q[N + 1] != 0u;
  const uint32_t lz = hi ? clz32(q[N + 1]) : 0u;
  uint32_t t[N + 2];
  MPB_UNROLL
  for (int i = 0; i < N + 2; ++i) {
    const uint32_t lo = i > 0 ? q[i > 0 ? i - 1 : 0] : 0u;
    t[i] = hi ? fshl(lo, q[i], lz) : lo;
  }
  MPB_UNROLL
  for (int i = 0; i < N; ++i) r.m[i] = t[i + 2];
  const uint32_t rb = t[1] >> 31;
  const uint32_t st = (t[1] << 1) | t[0] | rem;
  int32_t e = a.e - (hi ? (int32_t)lz : 32) - 32 * (NV - 1);
  rndn<N>(r.m, e, rb, st);
  r.e = e;
  r.s = a.s;
}

/* r = round(a / d), d an unsigned 32-bit integer (d = 0 gives 0) */
template <int N>
MPB_HD void div_ui(fval<N> &r, const fval<N> &a, uint32_t d) {
  if (is_zero(a) || d == 0u) {
    set_zero(r);
    return;
  }
  const uint32_t dv[1] = {d};
  div_int<N, 1>(r, a, dv);
}

/* r = round(a / d), d an unsigned 64-bit integer (d = 0 gives 0) */
template <int N>
MPB_HD void div_u64(fval<N> &r, const fval<N> &a, uint64_t d) {
  if ((d >> 32) == 0u) {
    div_ui<N>(r, a, (uint32_t)d);
    return;
  }
  if (is_zero(a)) {
    set_zero(r);
    return;
  }
  const uint32_t dv[2] = {(uint32_t)d, (uint32_t)(d >> 32)};
  div_int<N, 2>(r, a, dv);
}

/* o[0 .. L] = a[0 .. L) * k exactly */
template <int L>
MPB_HD void mul_ui_exact(uint32_t *o, const uint32_t *a, uint32_t k) {
  uint32_t cf = 0;
  o[0] = a[0] * k;
  MPB_UNROLL
  for (int i = 1; i < L; ++i)
    o[i] = (i == 1) ? add_cc(a[i] * k, mulhi(a[i - 1], k), cf) : addc_cc(a[i] * k, mulhi(a[i - 1], k), cf);
  o[L] = addc(mulhi(a[L - 1], k), 0u, cf);
}

/* ------------------------------------------------------------------ *
 * out-of-line working-precision operations: one instance per NW in a
 * translation unit, called from the series loops (code size and compile
 * time stay linear in the number of functions)
 * ------------------------------------------------------------------ */
/* Up to kByValueLimbs limbs each operation is one out-of-line function taking
 * and returning values (passed in registers); wider operands go by reference
 * (passing them by value would spill). */
template <int N>
MPB_NOINLINE fval<N> w_op2_v(int op, fval<N> a, fval<N> b) {
  fval<N> r;
  switch (op) {
    case 0: mul<N>(r, a, b); break;
    case 1: add<N>(r, a, b); break;
    case 2: sub<N>(r, a, b); break;
    case 3: div<N>(r, a, b); break;
    default: sqrt_<N>(r, a);
  }
  return r;
}
template <int N>
MPB_NOINLINE void w_op2_r(int op, fval<N> &r, const fval<N> &a, const fval<N> &b) {
  switch (op) {
    case 0: mul<N>(r, a, b); break;
    case 1: add<N>(r, a, b); break;
    case 2: sub<N>(r, a, b); break;
    case 3: div<N>(r, a, b); break;
    default: sqrt_<N>(r, a);
  }
}
template <int N>
MPB_HD void w_op2(int op, fval<N> &r, const fval<N> &a, const fval<N> &b) {
  if constexpr (N <= kByValueLimbs)
    r = w_op2_v<N>(op, a, b);
  else
    w_op2_r<N>(op, r, a, b);
}
template <int N>
MPB_HD void w_mul(fval<N> &r, const fval<N> &a, const fval<N> &b) {
  w_op2<N>(0, r, a, b);
}
template <int N>
MPB_HD void w_add(fval<N> &r, const fval<N> &a, const fval<N> &b) {
  w_op2<N>(1, r, a, b);
}
template <int N>
MPB_HD void w_sub(fval<N> &r, const fval<N> &a, const fval<N> &b) {
  w_op2<N>(2, r, a, b);
}
template <int N>
MPB_HD void w_div(fval<N> &r, const fval<N> &a, const fval<N> &b) {
  w_op2<N>(3, r, a, b);
}
template <int N>
MPB_HD void w_sqrt(fval<N> &r, const fval<N> &a) {
  w_op2<N>(4, r, a, a);
}
template <int N>
MPB_NOINLINE fval<N> w_div_ui_v(fval<N> a, uint32_t d) {
  fval<N> r;
  div_ui<N>(r, a, d);
  return r;
}
template <int N>
MPB_NOINLINE void w_div_ui_r(fval<N> &r, const fval<N> &a, uint32_t d) {
  div_ui<N>(r, a, d);
}
template <int N>
MPB_HD void w_div_ui(fval<N> &r, const fval<N> &a, uint32_t d) {
  if constexpr (N <= kByValueLimbs)
    r = w_div_ui_v<N>(a, d);
  else
    w_div_ui_r<N>(r, a, d);
}
template <int N>
MPB_NOINLINE fval<N> w_fmmx_v(fval<N> a, fval<N> b, fval<N> c, fval<N> d, uint32_t negate_cd) {
  fval<N> r;
  fmms<N>(r, a, b, c, d, negate_cd);
  return r;
}
template <int N>
MPB_NOINLINE void w_fmmx_r(fval<N> &r, const fval<N> &a, const fval<N> &b, const fval<N> &c, const fval<N> &d,
                           uint32_t negate_cd) {
  fmms<N>(r, a, b, c, d, negate_cd);
}
template <int N>
MPB_HD void w_fmma(fval<N> &r, const fval<N> &a, const fval<N> &b, const fval<N> &c, const fval<N> &d) {
  if constexpr (N <= kByValueLimbs)
    r = w_fmmx_v<N>(a, b, c, d, 0u);
  else
    w_fmmx_r<N>(r, a, b, c, d, 0u);
}
template <int N>
MPB_HD void w_fmms(fval<N> &r, const fval<N> &a, const fval<N> &b, const fval<N> &c, const fval<N> &d) {
  if constexpr (N <= kByValueLimbs)
    r = w_fmmx_v<N>(a, b, c, d, 1u);
  else
    w_fmmx_r<N>(r, a, b, c, d, 1u);
}

/* ------------------------------------------------------------------ *
 * exponential family
 * ------------------------------------------------------------------ */
/* E = expm1(R) for |R| < 1 */
template <int NW>
MPB_NOINLINE void expm1_red(fval<NW> &E, const fval<NW> &R) {
  constexpr int kS = em1_halvings(NW), T = em1_terms(NW);
  if (is_zero(R)) {
    set_zero(E);
    return;
  }
  if (R.e < -(32 * NW + 8)) { /* expm1(R) = R (1 + R/2 + ...): R/2 is below the working precision */
    E = R;
    return;
  }
  int sh = R.e + kS;
  sh = sh < 0 ? 0 : (sh > kS ? kS : sh);
  fval<NW> r = R, one, h, e, two;
  r.e -= sh;
  one_w<NW>(one);
  h = one;
#pragma unroll 1
  for (int i = T; i >= 2; --i) { /* the hot loops inline their operations */
    fval<NW> t, u;
    mul<NW>(t, r, h);
    div_ui<NW>(u, t, (uint32_t)i);
    add<NW>(h, one, u);
  }
  w_mul<NW>(e, r, h);
  two = one;
  two.e += 1;
#pragma unroll 1
  for (int j = 0; j < sh; ++j) {
    fval<NW> t, u;
    add<NW>(t, e, two);
    mul<NW>(u, e, t);
    e = u;
  }
  E = e;
}

/* k = the integer nearest x / ln 2 (|x| < 2^29) */
template <int NW>
MPB_HD int32_t exp_k(const fval<NW> &x) {
  return (int32_t)nearbyint(to_dbl_approx<NW>(x) * 1.4426950408889634074);
}

/* R = x - k ln2 */
template <int NW>
MPB_HD void exp_reduce(fval<NW> &R, const fval<NW> &x, int32_t k) {
  if (k == 0) {
    R = x;
    return;
  }
  fval<NW> L, K, t;
  ln2_w<NW>(L);
  from_i32<NW>(K, k);
  w_mul<NW>(t, K, L);
  w_sub<NW>(R, x, t);
}

/* exp at the working precision; false when the result leaves the exponent
 * range (|x| >= 2^29) */
template <int NW>
MPB_NOINLINE bool exp_w(fval<NW> &r, const fval<NW> &x) {
  fval<NW> one;
  one_w<NW>(one);
  if (is_zero(x)) {
    r = one;
    return true;
  }
  if (x.e > 29) {
    set_zero(r);
    return false;
  }
  const int32_t k = exp_k<NW>(x);
  fval<NW> R, E, p;
  exp_reduce<NW>(R, x, k);
  expm1_red<NW>(E, R);
  w_add<NW>(p, E, one);
  p.e += k;
  r = p;
  return true;
}

/* expm1 at the working precision; false on overflow (x >= 2^29) */
template <int NW>
MPB_NOINLINE bool expm1_w(fval<NW> &r, const fval<NW> &x) {
  fval<NW> one;
  one_w<NW>(one);
  if (is_zero(x)) {
    set_zero(r);
    return true;
  }
  if (x.e > 29) { /* exp(x) - 1 rounds to -1 for x <= -2^29 */
    r = one;
    r.s = 1u;
    if (x.s) return true;
    set_zero(r);
    return false;
  }
  const int32_t k = exp_k<NW>(x);
  if (k == 0) { /* |x| < ln2 / 2 */
    expm1_red<NW>(r, x);
    return true;
  }
  fval<NW> p; /* |exp(x) - 1| > 0.29: at most two bits cancel */
  exp_w<NW>(p, x);
  w_sub<NW>(r, p, one);
  return true;
}

/* sh = sinh(x), ch = cosh(x) from E = expm1(|x|): sinh = (E + E/(E+1)) / 2,
 * cosh = ((E+1) + 1/(E+1)) / 2 (no cancellation); false on overflow */
template <int NW>
MPB_NOINLINE bool sinhcosh_w(fval<NW> &sh, fval<NW> &ch, const fval<NW> &x) {
  fval<NW> one, a = x, E, P, Q, iv;
  one_w<NW>(one);
  a.s = 0u;
  if (is_zero(a)) {
    set_zero(sh);
    ch = one;
    return true;
  }
  if (a.e > 29) {
    set_zero(sh);
    set_zero(ch);
    return false;
  }
  expm1_w<NW>(E, a);
  w_add<NW>(P, E, one);
  w_div<NW>(Q, E, P);
  w_add<NW>(sh, E, Q);
  sh.e -= 1;
  sh.s = x.s;
  w_div<NW>(iv, one, P);
  w_add<NW>(ch, P, iv);
  ch.e -= 1;
  return true;
}

/* ------------------------------------------------------------------ *
 * logarithm family
 * ------------------------------------------------------------------ */
/* r = z (1 + z^2/3 + z^4/5 + ...) (atanh), or with alternating signs (atan),
 * for |z| < 2^-ZB */
template <int NW, int ZB>
MPB_NOINLINE void odd_series(fval<NW> &r, const fval<NW> &z, bool alternate) {
  constexpr int T = odd_terms(NW, ZB);
  if (is_zero(z) || z.e < -(16 * NW + 8)) { /* z^2 / 3 is below the working precision */
    r = z;
    return;
  }
  fval<NW> one, z2, h;
  one_w<NW>(one);
  w_mul<NW>(z2, z, z);
  if (alternate) z2.s = 1u;
  w_div_ui<NW>(h, one, (uint32_t)(2 * T + 1));
#pragma unroll 1
  for (int i = T - 1; i >= 0; --i) {
    fval<NW> t, c;
    mul<NW>(t, z2, h);
    div_ui<NW>(c, one, (uint32_t)(2 * i + 1));
    add<NW>(h, c, t);
  }
  w_mul<NW>(r, z, h);
}

/* 2 atanh(D / (2 + D)) = log(1 + D) for |D| < 2^-(ZB) */
template <int NW, int ZB>
MPB_HD void log1p_small(fval<NW> &r, const fval<NW> &D) {
  fval<NW> two, S, z;
  one_w<NW>(two);
  two.e += 1;
  w_add<NW>(S, two, D);
  w_div<NW>(z, D, S);
  odd_series<NW, ZB>(r, z, false);
  if (!is_zero(r)) r.e += 1;
}

/* log at the working precision, x > 0: x = m 2^e, m in [1/sqrt2, sqrt2).
 * Near 1 (|m - 1| < 2^-12) log m = log1p_small(m - 1) directly; elsewhere
 * y0 = log m in double (|y0 - log m| < 2^-53), m' = m exp(-y0) = 1 + d with
 * |d| < 2^-50, and log m = y0 + log1p_small(d): one exponential and a few
 * series terms (d needs only absolute accuracy: |log m| > 2^-13). */
template <int NW>
MPB_NOINLINE void log_w(fval<NW> &r, const fval<NW> &x) {
  constexpr int ZB1 = kNearBits, ZB2 = 48;
  fval<NW> one, m = x, D, lm;
  one_w<NW>(one);
  int32_t e = x.e;
  m.s = 0u;
  if (top_fraction<NW>(x) < 0.70710678118654752440) {
    m.e = 1;
    e -= 1;
  } else {
    m.e = 0;
  }
  w_sub<NW>(D, m, one); /* exact */
  if (is_zero(D)) {
    set_zero(lm);
  } else if (D.e <= -ZB1) {
    log1p_small<NW, ZB1>(lm, D);
  } else {
    fval<NW> Y0, nY0, E, P, d, l1;
    from_dbl<NW>(Y0, log(ldexp(top_fraction<NW>(m), m.e)));
    nY0 = Y0;
    neg_w<NW>(nY0);
    exp_w<NW>(E, nY0);
    w_mul<NW>(P, m, E);
    w_sub<NW>(d, P, one);
    log1p_small<NW, ZB2>(l1, d);
    w_add<NW>(lm, Y0, l1);
  }
  if (e == 0) {
    r = lm;
    return;
  }
  fval<NW> L, E, t;
  ln2_w<NW>(L);
  from_i32<NW>(E, e);
  w_mul<NW>(t, E, L);
  w_add<NW>(r, t, lm);
}

/* log1p at the working precision; false for x <= -1 */
template <int NW>
MPB_NOINLINE bool log1p_w(fval<NW> &r, const fval<NW> &x) {
  constexpr int ZB = kNearBits;
  if (is_zero(x)) {
    set_zero(r);
    return true;
  }
  if (x.e <= -ZB) {
    log1p_small<NW, ZB>(r, x);
    return true;
  }
  fval<NW> one, t;
  one_w<NW>(one);
  w_add<NW>(t, one, x);
  if (is_zero(t) || t.s) {
    set_zero(r);
    return false;
  }
  log_w<NW>(r, t);
  return true;
}

/* ------------------------------------------------------------------ *
 * trigonometric family
 * ------------------------------------------------------------------ */
/* x = k pi/2 + R with k the integer nearest x 2/pi (|x| < 2^30): k pi/2 is
 * formed exactly from pi/4 at NR = 2N + 4 limbs and the difference rounded
 * once to NW limbs.  Returns k mod 4. */
template <int N, int NW>
MPB_HD uint32_t reduce_half_pi(fval<NW> &R, const fval<N> &x) {
  constexpr int NR = 2 * N + 4;
  static_assert(NR <= kPiWordCount, "precision above the pi table");
  const int32_t k = (int32_t)nearbyint(to_dbl_approx<N>(x) * 0.63661977236758134308);
  if (k == 0) {
    widen<N, NW>(R, x);
    return 0u;
  }
  const uint32_t ak = k < 0 ? 0u - (uint32_t)k : (uint32_t)k;
  uint32_t pw[NR], p[NR + 1], P[NR + 1], X[NR + 1];
  MPB_UNROLL
  for (int i = 0; i < NR; ++i) pw[i] = pi_word(kPiWordCount - NR + i);
  mul_ui_exact<NR>(p, pw, ak); /* |k| pi/4 2^(32 NR) */
  const bool z = p[NR] == 0u;  /* |k| pi/4 < 1: one limb down */
  MPB_UNROLL
  for (int i = 0; i < NR + 1; ++i) P[i] = z ? (i > 0 ? p[i > 0 ? i - 1 : 0] : 0u) : p[i];
  const uint32_t lz = clz32(P[NR]);
  MPB_UNROLL
  for (int i = NR; i > 0; --i) P[i] = fshl(P[i - 1], P[i], lz);
  P[0] <<= lz;
  /* |k| pi/2 = p 2^(1 - 32 NR) = P 2^(eP - 32 (NR + 1)) */
  const int32_t eP = 33 - (z ? 32 : 0) - (int32_t)lz;
  MPB_UNROLL
  for (int i = 0; i < NR + 1; ++i) X[i] = (i >= NR + 1 - N) ? x.m[i - (NR + 1 - N)] : 0u;
  add_round<NR + 1, NW>(R, X, x.e, x.s, P, eP, k > 0 ? 1u : 0u);
  return (uint32_t)k & 3u;
}

/* S = sin R, C = cos R for |R| <= pi/4 (slightly above) */
template <int NW>
MPB_NOINLINE void sincos_red(fval<NW> &S, fval<NW> &C, const fval<NW> &R) {
  constexpr int kS = sc_halvings(NW), T = sc_terms(NW);
  fval<NW> one;
  one_w<NW>(one);
  if (is_zero(R) || R.e < -(16 * NW + 8)) { /* R^2 / 6 is below the working precision */
    S = R;
    C = one;
    return;
  }
  int sh = R.e + kS;
  sh = sh < 0 ? 0 : (sh > kS ? kS : sh);
  fval<NW> r = R, r2, hs = one, hv = one, s, v;
  r.e -= sh;
  w_mul<NW>(r2, r, r);
#pragma unroll 1
  for (int i = T; i >= 1; --i) { /* the hot loops inline their operations */
    fval<NW> t, u;
    mul<NW>(t, r2, hs);
    div_ui<NW>(u, t, (uint32_t)((2 * i) * (2 * i + 1)));
    sub<NW>(hs, one, u);
    mul<NW>(t, r2, hv);
    div_ui<NW>(u, t, (uint32_t)((2 * i + 1) * (2 * i + 2)));
    sub<NW>(hv, one, u);
  }
  w_mul<NW>(s, r, hs);  /* sin r' */
  w_mul<NW>(v, r2, hv); /* 2 (1 - cos r') */
  v.e -= 1;
#pragma unroll 1
  for (int j = 0; j < sh; ++j) { /* v <- 2 s^2, s <- 2 s (1 - v) */
    fval<NW> c, s2, sc;
    sub<NW>(c, one, v);
    mul<NW>(s2, s, s);
    mul<NW>(sc, s, c);
    v = s2;
    v.e += 1;
    s = sc;
    s.e += 1;
  }
  S = s;
  w_sub<NW>(C, one, v);
}

/* sin and cos of an N-limb x at the working precision; false for |x| >= 2^30 */
template <int N, int NW>
MPB_NOINLINE bool sincos_w(fval<NW> &S, fval<NW> &C, const fval<N> &x) {
  if (is_zero(x)) {
    set_zero(S);
    one_w<NW>(C);
    return true;
  }
  if (x.e > 30) {
    set_zero(S);
    set_zero(C);
    return false;
  }
  fval<NW> R, s, c;
  const uint32_t q = reduce_half_pi<N, NW>(R, x);
  sincos_red<NW>(s, c, R);
  /* sin(R + q pi/2), cos(R + q pi/2) */
  if (q & 1u) {
    S = c;
    C = s;
    neg_w<NW>(C);
  } else {
    S = s;
    C = c;
  }
  if (q & 2u) {
    neg_w<NW>(S);
    neg_w<NW>(C);
  }
  return true;
}

/* atan at the working precision: a = |x|, 1/a above 1 (then pi/2 - .);
 * below 2^-12 the alternating odd series directly; otherwise y0 = atan a in
 * double, S = sin y0, C = cos y0 and atan a = y0 + atan w with
 * w = (a C - S) / (C + a S) = tan(atan a - y0), |w| < 2^-50: a few series
 * terms (w needs only absolute accuracy: atan a > 2^-13) */
template <int NW>
MPB_NOINLINE void atan_w(fval<NW> &r, const fval<NW> &x) {
  if (is_zero(x)) {
    set_zero(r);
    return;
  }
  fval<NW> one, a = x, res;
  one_w<NW>(one);
  a.s = 0u;
  const bool inv = cmpmag<NW>(a, one) > 0;
  if (inv) {
    fval<NW> t;
    w_div<NW>(t, one, a);
    a = t;
  }
  if (a.e <= -kNearBits) {
    odd_series<NW, kNearBits>(res, a, true);
  } else {
    fval<NW> Y0, S, C, aC, aS, num, den, w, l;
    from_dbl<NW>(Y0, atan(to_dbl_approx<NW>(a)));
    sincos_red<NW>(S, C, Y0);
    w_mul<NW>(aC, a, C);
    w_mul<NW>(aS, a, S);
    w_sub<NW>(num, aC, S);
    w_add<NW>(den, C, aS);
    w_div<NW>(w, num, den);
    odd_series<NW, 48>(l, w, true);
    w_add<NW>(res, Y0, l);
  }
  if (inv) {
    fval<NW> h, t;
    pi_w<NW>(h, 1);
    w_sub<NW>(t, h, res);
    res = t;
  }
  res.s = x.s;
  r = res;
}

/* atan2(y, x): the angle of (x, y) in (-pi, pi]; (0, 0) gives 0 */
template <int NW>
MPB_NOINLINE void atan2_w(fval<NW> &r, const fval<NW> &y, const fval<NW> &x) {
  if (is_zero(x)) {
    if (is_zero(y)) {
      set_zero(r);
      return;
    }
    pi_w<NW>(r, 1);
    r.s = y.s;
    return;
  }
  fval<NW> q, base;
  w_div<NW>(q, y, x);
  atan_w<NW>(base, q);
  if (!x.s) {
    r = base;
    return;
  }
  fval<NW> pi;
  pi_w<NW>(pi, 2);
  if (y.s) pi.s = 1u; /* y < 0: base - pi; y >= 0: base + pi */
  w_add<NW>(r, base, pi);
}

/* ------------------------------------------------------------------ *
 * the functions at N limbs (faithful)
 * ------------------------------------------------------------------ */
/* r = exp(x) */
template <int N>
MPB_NOINLINE void exp_(fval<N> &r, const fval<N> &x) {
  constexpr int NW = N + 4;
  fval<NW> X, Y;
  widen<N, NW>(X, x);
  if (!exp_w<NW>(Y, X)) {
    set_zero(r);
    return;
  }
  narrow<NW, N>(r, Y);
}

/* r = expm1(x) = exp(x) - 1 */
template <int N>
MPB_NOINLINE void expm1_(fval<N> &r, const fval<N> &x) {
  constexpr int NW = N + 4;
  fval<NW> X, Y;
  widen<N, NW>(X, x);
  if (!expm1_w<NW>(Y, X)) {
    set_zero(r);
    return;
  }
  narrow<NW, N>(r, Y);
}

/* r = log(x); x <= 0 gives 0 */
template <int N>
MPB_NOINLINE void log_(fval<N> &r, const fval<N> &x) {
  constexpr int NW = N + 4;
  if (is_zero(x) || x.s) {
    set_zero(r);
    return;
  }
  fval<NW> X, Y;
  widen<N, NW>(X, x);
  log_w<NW>(Y, X);
  narrow<NW, N>(r, Y);
}

/* r = log1p(x) = log(1 + x); x <= -1 gives 0 */
template <int N>
MPB_NOINLINE void log1p_(fval<N> &r, const fval<N> &x) {
  constexpr int NW = N + 4;
  fval<NW> X, Y;
  widen<N, NW>(X, x);
  if (!log1p_w<NW>(Y, X)) {
    set_zero(r);
    return;
  }
  narrow<NW, N>(r, Y);
}

/* sin, cos, tan (|x| < 2^30; larger |x| gives 0) */
template <int N>
MPB_NOINLINE void sin_(fval<N> &r, const fval<N> &x) {
  constexpr int NW = N + 4;
  fval<NW> S, C;
  if (!sincos_w<N, NW>(S, C, x)) {
    set_zero(r);
    return;
  }
  narrow<NW, N>(r, S);
}
template <int N>
MPB_NOINLINE void cos_(fval<N> &r, const fval<N> &x) {
  constexpr int NW = N + 4;
  fval<NW> S, C;
  if (!sincos_w<N, NW>(S, C, x)) {
    set_zero(r);
    return;
  }
  narrow<NW, N>(r, C);
}
template <int N>
MPB_NOINLINE void tan_(fval<N> &r, const fval<N> &x) {
  constexpr int NW = N + 4;
  fval<NW> S, C, T;
  if (!sincos_w<N, NW>(S, C, x)) {
    set_zero(r);
    return;
  }
  w_div<NW>(T, S, C);
  narrow<NW, N>(r, T);
}

/* atan, asin (|x| >= 1 gives +-pi/2), acos (x >= 1 gives 0, x <= -1 pi) */
template <int N>
MPB_NOINLINE void atan_(fval<N> &r, const fval<N> &x) {
  constexpr int NW = N + 4;
  fval<NW> X, Y;
  widen<N, NW>(X, x);
  atan_w<NW>(Y, X);
  narrow<NW, N>(r, Y);
}
template <int N>
MPB_NOINLINE void asin_(fval<N> &r, const fval<N> &x) {
  constexpr int NW = N + 4;
  if (is_zero(x)) {
    set_zero(r);
    return;
  }
  fval<NW> X, one, Y;
  widen<N, NW>(X, x);
  one_w<NW>(one);
  fval<NW> a = X;
  a.s = 0u;
  if (cmpmag<NW>(a, one) >= 0) {
    pi_w<NW>(Y, 1);
  } else { /* atan(x / sqrt((1 - x)(1 + x))) */
    fval<NW> u, v, w, s, t;
    w_sub<NW>(u, one, a);
    w_add<NW>(v, one, a);
    w_mul<NW>(w, u, v);
    w_sqrt<NW>(s, w);
    w_div<NW>(t, a, s);
    atan_w<NW>(Y, t);
  }
  Y.s = x.s;
  narrow<NW, N>(r, Y);
}
template <int N>
MPB_NOINLINE void acos_(fval<N> &r, const fval<N> &x) {
  constexpr int NW = N + 4;
  fval<NW> X, one, Y;
  widen<N, NW>(X, x);
  one_w<NW>(one);
  if (cmpmag<NW>(X, one) >= 0) { /* |x| >= 1 */
    if (x.s)
      pi_w<NW>(Y, 2);
    else
      set_zero(Y);
  } else { /* 2 atan(sqrt((1 - x) / (1 + x))) */
    fval<NW> u, v, q, s;
    w_sub<NW>(u, one, X);
    w_add<NW>(v, one, X);
    w_div<NW>(q, u, v);
    w_sqrt<NW>(s, q);
    atan_w<NW>(Y, s);
    Y.e += 1;
  }
  narrow<NW, N>(r, Y);
}

/* atanh (|x| >= 1 gives 0) = sign(x) log1p(2|x| / (1 - |x|)) / 2 (on |x|:
 * the argument of log1p stays positive, 1 + it never cancels) */
template <int N>
MPB_NOINLINE void atanh_(fval<N> &r, const fval<N> &x) {
  constexpr int NW = N + 4, ZB = kNearBits;
  fval<NW> X, one, Y;
  widen<N, NW>(X, x);
  X.s = 0u;
  one_w<NW>(one);
  if (is_zero(x) || cmpmag<NW>(X, one) >= 0) {
    set_zero(r);
    return;
  }
  if (X.e <= -ZB) {
    odd_series<NW, ZB>(Y, X, false);
  } else {
    fval<NW> u, q;
    w_sub<NW>(u, one, X); /* exact */
    w_div<NW>(q, X, u);
    q.e += 1;
    log1p_w<NW>(Y, q);
    Y.e -= 1;
  }
  Y.s = x.s;
  narrow<NW, N>(r, Y);
}

/* sinh, cosh (|x| >= 2^29 gives 0) */
template <int N>
MPB_NOINLINE void sinh_(fval<N> &r, const fval<N> &x) {
  constexpr int NW = N + 4;
  fval<NW> X, sh, ch;
  widen<N, NW>(X, x);
  if (!sinhcosh_w<NW>(sh, ch, X)) {
    set_zero(r);
    return;
  }
  narrow<NW, N>(r, sh);
}
template <int N>
MPB_NOINLINE void cosh_(fval<N> &r, const fval<N> &x) {
  constexpr int NW = N + 4;
  fval<NW> X, sh, ch;
  widen<N, NW>(X, x);
  if (!sinhcosh_w<NW>(sh, ch, X)) {
    set_zero(r);
    return;
  }
  narrow<NW, N>(r, ch);
}

/* cbrt (sign kept): x = f 2^(3q + rr), y ~ cbrt(f 2^rr) by Newton's
 * y <- y + (m / y^2 - y) / 3 from a double estimate, the count fixed by the
 * working precision (the error squares each step) */
template <int N>
MPB_NOINLINE void cbrt_(fval<N> &r, const fval<N> &x) {
  constexpr int NW = N + 4;
  if (is_zero(x)) {
    set_zero(r);
    return;
  }
  int32_t q = x.e / 3, rr = x.e - 3 * q;
  if (rr < 0) {
    rr += 3;
    q -= 1;
  }
  fval<NW> m, y;
  widen<N, NW>(m, x);
  m.s = 0u;
  m.e = rr;
  from_dbl<NW>(y, cbrt(ldexp(top_fraction<N>(x), rr)));
#pragma unroll 1
  for (int bits = 48; bits < 32 * NW + 8; bits *= 2) {
    fval<NW> y2, t, d, d3, yn;
    w_mul<NW>(y2, y, y);
    w_div<NW>(t, m, y2);
    w_sub<NW>(d, t, y);
    w_div_ui<NW>(d3, d, 3u);
    w_add<NW>(yn, y, d3);
    y = yn;
  }
  y.e += q;
  y.s = x.s;
  narrow<NW, N>(r, y);
}

/* y is an integer (odd: its parity) */
template <int N>
MPB_HD bool is_integer(const fval<N> &y, bool &odd) {
  odd = false;
  if (is_zero(y)) return true;
  if (y.e <= 0) return false;
  if (y.e > 32 * N) return true;
  const int f = 32 * N - y.e; /* mantissa bits [0, f) are below the binary point */
  for (int i = 0; i < N; ++i) {
    const int lo = 32 * i;
    uint32_t frac_mask;
    if (f >= lo + 32)
      frac_mask = 0xffffffffu;
    else if (f <= lo)
      frac_mask = 0u;
    else
      frac_mask = (1u << (f - lo)) - 1u;
    if (y.m[i] & frac_mask) return false;
    if (f >= lo && f < lo + 32) odd = (y.m[i] >> (f - lo)) & 1u;
  }
  return true;
}

/* pow(x, y) = exp(y log |x|): y = 0 gives 1, x = 0 gives 0, a negative x
 * needs an integer y (the sign by its parity), otherwise 0 */
template <int N>
MPB_NOINLINE void pow_(fval<N> &r, const fval<N> &x, const fval<N> &y) {
  constexpr int NW = N + 4;
  if (is_zero(y)) {
    fval<NW> one;
    one_w<NW>(one);
    narrow<NW, N>(r, one);
    return;
  }
  if (is_zero(x)) {
    set_zero(r);
    return;
  }
  bool odd = false;
  if (x.s && !is_integer<N>(y, odd)) {
    set_zero(r);
    return;
  }
  fval<NW> X, Y, L, Z, P;
  widen<N, NW>(X, x);
  X.s = 0u;
  widen<N, NW>(Y, y);
  log_w<NW>(L, X);
  w_mul<NW>(Z, Y, L);
  if (!exp_w<NW>(P, Z)) {
    set_zero(r);
    return;
  }
  P.s = (x.s && odd) ? 1u : 0u;
  narrow<NW, N>(r, P);
}

/* atan2(y, x) */
template <int N>
MPB_NOINLINE void atan2_(fval<N> &r, const fval<N> &y, const fval<N> &x) {
  constexpr int NW = N + 4;
  fval<NW> Y, X, A;
  widen<N, NW>(Y, y);
  widen<N, NW>(X, x);
  atan2_w<NW>(A, Y, X);
  narrow<NW, N>(r, A);
}

/* pi and ln 2 rounded to N limbs (correctly: the generator checks that the
 * 128 bits below never sit within one unit of halfway) */
template <int N>
MPB_HD void pi_(fval<N> &r) {
  fval<N + 4> p;
  pi_w<N + 4>(p, 2);
  narrow<N + 4, N>(r, p);
}
template <int N>
MPB_HD void ln2_(fval<N> &r) {
  fval<N + 4> p;
  ln2_w<N + 4>(p);
  narrow<N + 4, N>(r, p);
}

/* ------------------------------------------------------------------ *
 * complex functions (each component faithful)
 * ------------------------------------------------------------------ */
/* (ar + i ai) / (br + i bi) = ((ar br + ai bi) + i (ai br - ar bi)) / |b|^2,
 * each of the three sums with one rounding; b = 0 gives 0 */
template <int NW>
MPB_NOINLINE void cdiv_w(fval<NW> &rr, fval<NW> &ri, const fval<NW> &ar, const fval<NW> &ai,
                         const fval<NW> &br, const fval<NW> &bi) {
  fval<NW> den, nr, ni;
  w_fmma<NW>(den, br, br, bi, bi);
  if (is_zero(den)) {
    set_zero(rr);
    set_zero(ri);
    return;
  }
  w_fmma<NW>(nr, ar, br, ai, bi);
  w_fmms<NW>(ni, ai, br, ar, bi);
  w_div<NW>(rr, nr, den);
  w_div<NW>(ri, ni, den);
}

/* c = 0 (exp), 1 (log), 2 (sqrt), 3 (sin), 4 (cos), 5 (tan), 6 (sinh), 7 (cosh) */
template <int N>
MPB_NOINLINE void cfunc_(int c, fval<N> &rr, fval<N> &ri, const fval<N> &zr, const fval<N> &zi) {
  constexpr int NW = N + 4;
  fval<NW> X, Y, R, I;
  widen<N, NW>(X, zr);
  widen<N, NW>(Y, zi);
  set_zero(R);
  set_zero(I);
  switch (c) {
    case 0: { /* e^x (cos y, sin y) */
      fval<NW> ex, s, co;
      if (exp_w<NW>(ex, X) && sincos_w<N, NW>(s, co, zi)) {
        w_mul<NW>(R, ex, co);
        w_mul<NW>(I, ex, s);
      }
      break;
    }
    case 1: { /* (log |z|, atan2(y, x)); log |z| = log1p(|z|^2 - 1) / 2 near |z| = 1 */
      fval<NW> r2;
      w_fmma<NW>(r2, X, X, Y, Y);
      if (is_zero(r2)) break;
      if (r2.e == 0 || r2.e == 1) { /* |z|^2 in [1/2, 2): |z|^2 - 1 with one rounding */
        fval<NW> m1, t;
        one_w<NW>(m1);
        m1.s = 1u;
        fmma_add<NW>(t, X, X, Y, Y, m1, 0u);
        log1p_w<NW>(R, t);
      } else {
        log_w<NW>(R, r2);
      }
      if (!is_zero(R)) R.e -= 1;
      atan2_w<NW>(I, Y, X);
      break;
    }
    case 2: { /* principal root: x >= 0 (sqrt((|z| + x)/2), y / (2u)), else
                 (|y| / (2t), sign(y) t) with t = sqrt((|z| - x)/2) */
      if (is_zero(X) && is_zero(Y)) break;
      fval<NW> r2, mod, h, u, d;
      w_fmma<NW>(r2, X, X, Y, Y);
      w_sqrt<NW>(mod, r2);
      fval<NW> ax = X;
      ax.s = 0u;
      w_add<NW>(h, mod, ax); /* |z| + |x|: no cancellation */
      h.e -= 1;
      w_sqrt<NW>(u, h);
      fval<NW> two_u = u;
      two_u.e += 1;
      fval<NW> ay = Y;
      ay.s = 0u;
      w_div<NW>(d, ay, two_u);
      if (!X.s) {
        R = u;
        I = d;
        I.s = is_zero(d) ? 0u : Y.s;
      } else {
        R = d;
        I = u;
        I.s = Y.s;
      }
      break;
    }
    case 3:   /* sin: (sin x cosh y, cos x sinh y) */
    case 4:   /* cos: (cos x cosh y, -sin x sinh y) */
    case 6:   /* sinh: (sinh x cos y, cosh x sin y) */
    case 7: { /* cosh: (cosh x cos y, sinh x sin y) */
      const bool hyp = c >= 6;
      fval<NW> s, co, sh, ch;
      if (!sincos_w<N, NW>(s, co, hyp ? zi : zr)) break;
      if (!sinhcosh_w<NW>(sh, ch, hyp ? X : Y)) break;
      if (c == 3) {
        w_mul<NW>(R, s, ch);
        w_mul<NW>(I, co, sh);
      } else if (c == 4) {
        w_mul<NW>(R, co, ch);
        w_mul<NW>(I, s, sh);
        neg_w<NW>(I);
      } else if (c == 6) {
        w_mul<NW>(R, sh, co);
        w_mul<NW>(I, ch, s);
      } else {
        w_mul<NW>(R, ch, co);
        w_mul<NW>(I, sh, s);
      }
      break;
    }
    case 5: { /* tan: (sin x cos x, sinh y cosh y) / (cos^2 x + sinh^2 y) */
      fval<NW> s, co, sh, ch, den, a, b;
      if (!sincos_w<N, NW>(s, co, zr)) break;
      if (!sinhcosh_w<NW>(sh, ch, Y)) break;
      w_fmma<NW>(den, co, co, sh, sh);
      if (is_zero(den)) break;
      w_mul<NW>(a, s, co);
      w_mul<NW>(b, sh, ch);
      w_div<NW>(R, a, den);
      w_div<NW>(I, b, den);
      break;
    }
    default:
      break;
  }
  narrow<NW, N>(rr, R);
  narrow<NW, N>(ri, I);
}

/* complex division (each component faithful) */
template <int N>
MPB_NOINLINE void cdiv_(fval<N> &rr, fval<N> &ri, const fval<N> &ar, const fval<N> &ai, const fval<N> &br,
                        const fval<N> &bi) {
  constexpr int NW = N + 4;
  fval<NW> Ar, Ai, Br, Bi, R, I;
  widen<N, NW>(Ar, ar);
  widen<N, NW>(Ai, ai);
  widen<N, NW>(Br, br);
  widen<N, NW>(Bi, bi);
  cdiv_w<NW>(R, I, Ar, Ai, Br, Bi);
  narrow<NW, N>(rr, R);
  narrow<NW, N>(ri, I);
}

}  // namespace mpb

#endif /* MPB_ELEM_CUH */
