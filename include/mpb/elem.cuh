/* mpb/elem.cuh -- exponential and logarithm on the mpb core (host and device).
 *
 * Faithful (at most 1 ULP from the exact value; in practice almost always the
 * correctly rounded one), the contract of the reference's cu_exp / cu_log
 * (mpc_cuda include/mpc_cuda/cu_fmath.cuh:1-14, 197-218).  Both work at
 * NW = N + 4 limbs (128 guard bits) with the core's correctly rounded
 * operations and round once to N limbs at the end:
 *
 *   exp:  x = k ln2 + r (k from a double estimate, r computed at NW limbs),
 *         r' = r / 2^16, exp(r') by its Taylor series in Horner form
 *         (p = 1 + r' p / i, i = T .. 1, T ~ 32 NW / 17 + 3 terms), then 16
 *         squarings and the factor 2^k.  The reduction error grows with |k|
 *         (below 2^30) and the squarings multiply the relative error by 2^16;
 *         together they stay below 2^-80 of the PB-bit result's ULP.
 *   log:  near 1 (|x - 1| < 2^-8): 2 atanh(z), z = (x - 1) / (x + 1) (x - 1 is
 *         exact), by its series z (1 + z^2/3 + z^4/5 + ...).  Elsewhere Newton's
 *         iteration y <- y + x exp(-y) - 1 from a double estimate, the number of
 *         steps fixed by the working precision (the error squares each step).
 *
 * ln 2 comes from consts.cuh (generated by make_consts.py).  exp of an
 * argument of magnitude 2^29 or more, whose result leaves the exponent range,
 * and log of zero or a negative number have no value in this format: the
 * result is 0.
 */
#ifndef MPB_ELEM_CUH
#define MPB_ELEM_CUH

#include "core.cuh"
#include "consts.cuh"

namespace mpb {

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

/* the value of the top 64 bits, scaled by 2^-(64 - shift): m / 2^64 in [0.5, 1) */
template <int NW>
MPB_HD double top_fraction(const fval<NW> &x) {
  const uint64_t m = ((uint64_t)x.m[NW - 1] << 32) | (NW >= 2 ? x.m[NW >= 2 ? NW - 2 : 0] : 0u);
  return ldexp((double)m, -64);
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
  MPB_UNROLL
  for (int i = 0; i < NW; ++i) r.m[i] = ln2_word(kLn2WordCount - NW + i);
  r.e = 0;
  r.s = 0u;
}

template <int NW>
MPB_HD void one_w(fval<NW> &r) {
  from_i32<NW>(r, 1);
}

/* exp at the working precision: r = exp(x), both NW limbs; false when the
 * result leaves the exponent range */
template <int NW>
MPB_HD bool exp_w(fval<NW> &r, const fval<NW> &x) {
  fval<NW> one;
  one_w<NW>(one);
  if (is_zero(x)) {
    r = one;
    return true;
  }
  if (x.e > 29) { /* |x| >= 2^29: the result leaves the exponent range */
    set_zero(r);
    return false;
  }
  const double xd = ldexp(top_fraction<NW>(x), x.e) * (x.s ? -1.0 : 1.0);
  const int32_t k = (int32_t)nearbyint(xd * 1.4426950408889634074);
  fval<NW> L, K, t, R;
  ln2_w<NW>(L);
  from_i32<NW>(K, k);
  mul<NW>(t, K, L);
  sub<NW>(R, x, t);
  if (!is_zero(R)) R.e -= 16;
  const int T = 32 * NW / 17 + 3;
  fval<NW> p = one;
#pragma unroll 1
  for (int i = T; i >= 1; --i) {
    fval<NW> q, d, iw;
    mul<NW>(q, p, R);
    from_i32<NW>(iw, i);
    div<NW>(d, q, iw);
    add<NW>(p, d, one);
  }
#pragma unroll 1
  for (int j = 0; j < 16; ++j) {
    fval<NW> q;
    mul<NW>(q, p, p);
    p = q;
  }
  p.e += k;
  r = p;
  return true;
}

/* r = exp(x), faithful */
template <int N>
MPB_HD void exp_(fval<N> &r, const fval<N> &x) {
  constexpr int NW = N + 4;
  fval<NW> X, Y;
  widen<N, NW>(X, x);
  if (!exp_w<NW>(Y, X)) {
    set_zero(r);
    return;
  }
  narrow<NW, N>(r, Y);
}

/* r = log(x), faithful; x <= 0 gives 0 */
template <int N>
MPB_HD void log_(fval<N> &r, const fval<N> &x) {
  constexpr int NW = N + 4;
  if (is_zero(x) || x.s) {
    set_zero(r);
    return;
  }
  fval<NW> X, one, D, Y;
  widen<N, NW>(X, x);
  one_w<NW>(one);
  sub<NW>(D, X, one); /* exact: x has N limbs, the window NW */
  if (is_zero(D)) {
    set_zero(r);
    return;
  }
  if (D.e <= -8) { /* |x - 1| < 2^-8: 2 atanh((x-1)/(x+1)) */
    fval<NW> S, Z, Z2, s;
    add<NW>(S, X, one);
    div<NW>(Z, D, S);
    mul<NW>(Z2, Z, Z);
    const int T = 32 * NW / 16 + 2;
    set_zero(s);
#pragma unroll 1
    for (int i = T; i >= 0; --i) {
      fval<NW> c, q, t;
      from_i32<NW>(c, 2 * i + 1);
      div<NW>(q, one, c);
      mul<NW>(t, Z2, s);
      add<NW>(s, q, t);
    }
    mul<NW>(Y, Z, s);
    Y.e += 1;
  } else { /* Newton on exp from log(m) + e ln2 in double */
    const double y0 = log(top_fraction<NW>(X)) + (double)X.e * 0.69314718055994530942;
    from_dbl<NW>(Y, y0);
    /* absolute accuracy of the start in bits: the double's 52 bits less the
     * magnitude of y0 (up to 2^30 ln 2 for the largest exponents) */
    int bits = 48 - (int)(fabs(y0) < 1.0 ? 0.0 : log2(fabs(y0)) + 1.0);
#pragma unroll 1
    for (int it = 0; it < 12 && bits < 32 * NW + 8; ++it) {
      fval<NW> ny, E, XE, t;
      ny = Y;
      if (!is_zero(ny)) ny.s ^= 1u;
      exp_w<NW>(E, ny);
      mul<NW>(XE, X, E);
      sub<NW>(t, XE, one);
      fval<NW> y2;
      add<NW>(y2, Y, t);
      Y = y2;
      bits *= 2;
    }
  }
  narrow<NW, N>(r, Y);
}

}  // namespace mpb

#endif /* MPB_ELEM_CUH */
