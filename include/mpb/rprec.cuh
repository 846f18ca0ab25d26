/* mpb/rprec.cuh -- arithmetic at a runtime precision p on the fixed-precision
 * core (host and device).
 *
 * The reference's runtime-precision layer (its mpfr_t port, mpc_cuda
 * src/mpfr_cuda/mpfr.h:582-589, 804: cu_mpfr_add / sub / mul / div / sqrt /
 * fma, RNDN at the destination's precision) takes any precision per call.
 * Here a precision p is served by the smallest supported format of PB >= p + 2
 * bits: the operation is rounded to odd at PB bits by the core (kRnd = 1) and
 * the result then to nearest-even at p bits, which equals the correctly
 * rounded result at p bits (Boldo and Melquiond 2008: rounding to odd at 2 or
 * more extra bits makes the second rounding exact).  Operands may carry up to
 * PB bits; results carry p significant bits (the bits below are zero).
 */
#ifndef MPB_RPREC_CUH
#define MPB_RPREC_CUH

#include "core.cuh"

namespace mpb {

/* z = round-to-nearest-even of z at p bits (1 <= p < 32N; the low 32N - p
 * bits are cleared).  Every limb is visited with compile-time indices. */
template <int N>
MPB_HD void round_to_bits(fval<N> &z, int p) {
  if (is_zero(z) || p >= 32 * N || p < 1) return;
  const int cut = 32 * N - p;           /* bits dropped, >= 1 */
  const int rl = (cut - 1) >> 5, rbit = (cut - 1) & 31; /* the round bit */
  const int ll = cut >> 5, lbit = cut & 31;             /* the last kept bit */
  uint32_t rb = 0u, st = 0u, lsb = 0u;
  MPB_UNROLL
  for (int i = 0; i < N; ++i) {
    const uint32_t w = z.m[i];
    const uint32_t below = (i < rl) ? 0xffffffffu : (i == rl ? ((1u << rbit) - 1u) : 0u);
    st |= w & below;
    rb |= (i == rl) ? ((w >> rbit) & 1u) : 0u;
    lsb |= (i == ll) ? ((w >> lbit) & 1u) : 0u;
    z.m[i] = (i < ll) ? 0u : (i == ll ? (w & ~((1u << lbit) - 1u)) : w);
  }
  if (!(rb && (st || lsb))) return;
  uint32_t c = 0u;
  MPB_UNROLL
  for (int i = 0; i < N; ++i) {
    const uint32_t add = (i == ll) ? (1u << lbit) : 0u;
    const uint32_t s1 = z.m[i] + add;
    const uint32_t c1 = s1 < add ? 1u : 0u;
    const uint32_t s2 = s1 + c;
    const uint32_t c2 = s2 < c ? 1u : 0u;
    z.m[i] = s2;
    c = c1 | c2;
  }
  if (c) { /* 1111..1 + 1: the significand becomes 1000..0, one exponent up */
    z.m[N - 1] = 0x80000000u;
    z.e += 1;
  }
}

/* r = op(a, b, c) rounded to nearest at p bits (p <= 32N - 2): op 0 a*b,
 * 1 a+b, 2 a-b, 3 a*b+c, 4 a/b, 5 sqrt(a); a / 0 and sqrt of a negative give 0 */
template <int N>
MPB_HD void op_rp(int op, int p, fval<N> &r, const fval<N> &a, const fval<N> &b, const fval<N> &c) {
  switch (op) {
    case 0: mul<N, 1>(r, a, b); break;
    case 1: add<N, false, 1>(r, a, b); break;
    case 2: sub<N, false, 1>(r, a, b); break;
    case 3: fma<N, false, 1>(r, a, b, c); break;
    case 4: div<N, 1>(r, a, b); break;
    default: sqrt_<N, 1>(r, a);
  }
  round_to_bits<N>(r, p);
}

}  // namespace mpb

#endif /* MPB_RPREC_CUH */
