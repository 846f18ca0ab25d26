/* mpc_cuda/cu_fcomplex.cuh -- drop-in cu_fp::cu_fcomplex<PB> for the mpb engine.
 *
 * Same names, layout and semantics as the mpc_cuda header of the same path
 * (reference include/mpc_cuda/cu_fcomplex.cuh:22-133): { cu_freal<PB> re, im },
 * arithmetic bit-exact with MPC's per-component round-to-nearest (MPC_RNDNN).
 * The complex product rounds each component once from exact products:
 *   re = round(ar*br - ai*bi),  im = round(ar*bi + ai*br)
 * computed by the mpb core (mpb::fmms): two exact 2N-limb products and one
 * aligned sum in registers, no intermediate rounding.  Added over the
 * reference: cu_cfma (a*b + c, one rounding per component, MPC mpc_fma).
 */
#ifndef MPB_DROPIN_CU_FCOMPLEX_CUH
#define MPB_DROPIN_CU_FCOMPLEX_CUH

#include "cu_freal.cuh"

namespace cu_fp {

/* normalised exact wide product term: value = sign*M*2^(exp - 64*WN), MSB of M
 * set unless zero (reference cu_wterm, cu_fcomplex.cuh:24-28) */
template <int PB>
struct cu_wterm {
  static const int WN = 2 * cu_freal<PB>::N;
  int sign;
  long exp;
  bool zero;
  cu_limb M[WN];
};

/* exact a*b as a wide term (reference cu_mk_term, cu_fcomplex.cuh:30-42): the
 * core's exact normalised product of the two 32-bit-word significands, whose
 * 2 PB/32 words fill the term's 64-bit limbs from the top */
template <int PB>
__host__ __device__ static cu_wterm<PB> cu_mk_term(const cu_freal<PB> &a, const cu_freal<PB> &b) {
  typedef detail::core_of<PB> Cr;
  const int WN = cu_wterm<PB>::WN, NP = 2 * Cr::N32, OFF = 2 * WN - NP; /* zero low halves */
  typename Cr::type x, y;
  detail::to_core<PB>(x, a);
  detail::to_core<PB>(y, b);
  uint32_t p[NP];
  int32_t e;
  mpb::mul_exact_norm<Cr::N32>(p, e, x, y);
  cu_wterm<PB> t;
  t.zero = a.is_zero() || b.is_zero();
  t.sign = t.zero ? 1 : a.sign * b.sign;
  t.exp = t.zero ? 0 : (long)e;
  for (int k = 0; k < WN; k++) {
    const int lo = 2 * k - OFF, hi = lo + 1;
    const cu_limb l = (!t.zero && lo >= 0) ? p[lo] : 0u, h = (!t.zero && hi >= 0) ? p[hi] : 0u;
    t.M[k] = (h << 32) | l;
  }
  return t;
}

template <int PB>
__host__ __device__ static int cu_wcmp(const cu_wterm<PB> &a, const cu_wterm<PB> &b) {
  if (a.exp != b.exp) return a.exp > b.exp ? 1 : -1;
  for (int i = cu_wterm<PB>::WN - 1; i >= 0; i--)
    if (a.M[i] != b.M[i]) return a.M[i] > b.M[i] ? 1 : -1;
  return 0;
}

/* round(A + B), one rounding (reference cu_round_sum2, cu_fcomplex.cuh:52-88),
 * through the core's exact aligned sum on 32-bit limbs */
template <int PB>
__host__ __device__ static cu_freal<PB> cu_round_sum2(cu_wterm<PB> A, cu_wterm<PB> B) {
  constexpr int WN = cu_wterm<PB>::WN, NX = 2 * WN;
  uint32_t xa[NX], xb[NX];
  for (int k = 0; k < NX; k++) {
    xa[k] = A.zero ? 0u : detail::half32(A.M, WN, k);
    xb[k] = B.zero ? 0u : detail::half32(B.M, WN, k);
  }
  typename detail::core_of<PB>::type r;
  mpb::add_round<NX, PB / 32>(r, xa, A.zero ? mpb::kExpZero : (int32_t)A.exp, A.sign < 0 ? 1u : 0u, xb,
                              B.zero ? mpb::kExpZero : (int32_t)B.exp, B.sign < 0 ? 1u : 0u);
  return detail::from_core<PB>(r);
}

/* round(a*b - c*d), round(a*b + c*d) (reference cu_fmms/cu_fmma, cu_fcomplex.cuh:90-96) */
template <int PB>
__host__ __device__ static cu_freal<PB> cu_fmms(const cu_freal<PB> &a, const cu_freal<PB> &b,
                                                const cu_freal<PB> &c, const cu_freal<PB> &d) {
  typename detail::core_of<PB>::type x, y, z, w, r;
  detail::to_core<PB>(x, a);
  detail::to_core<PB>(y, b);
  detail::to_core<PB>(z, c);
  detail::to_core<PB>(w, d);
  mpb::fmms(r, x, y, z, w);
  return detail::from_core<PB>(r);
}
template <int PB>
__host__ __device__ static cu_freal<PB> cu_fmma(const cu_freal<PB> &a, const cu_freal<PB> &b,
                                                const cu_freal<PB> &c, const cu_freal<PB> &d) {
  typename detail::core_of<PB>::type x, y, z, w, r;
  detail::to_core<PB>(x, a);
  detail::to_core<PB>(y, b);
  detail::to_core<PB>(z, c);
  detail::to_core<PB>(w, d);
  mpb::fmma(r, x, y, z, w);
  return detail::from_core<PB>(r);
}

/* the complex type (reference cu_fcomplex.cuh:98-113) */
template <int PB>
struct cu_fcomplex {
  cu_freal<PB> re, im;

  __host__ __device__ cu_fcomplex() {}
  __host__ __device__ cu_fcomplex(const cu_freal<PB> &r, const cu_freal<PB> &i) : re(r), im(i) {}
  __host__ __device__ cu_fcomplex(double r, double i)
      : re(cu_freal<PB>::from_double(r)), im(cu_freal<PB>::from_double(i)) {}

  __host__ __device__ static cu_fcomplex from_doubles(double r, double i) { return cu_fcomplex(r, i); }
  __host__ __device__ double real_d() const { return re.to_double(); }
  __host__ __device__ double imag_d() const { return im.to_double(); }
};

/* reference cu_fcomplex.cuh:115-124 */
template <int PB>
__host__ __device__ static inline cu_fcomplex<PB> cu_cadd(const cu_fcomplex<PB> &a, const cu_fcomplex<PB> &b) {
  return cu_fcomplex<PB>(cu_fadd<PB>(a.re, b.re), cu_fadd<PB>(a.im, b.im));
}
template <int PB>
__host__ __device__ static inline cu_fcomplex<PB> cu_csub(const cu_fcomplex<PB> &a, const cu_fcomplex<PB> &b) {
  return cu_fcomplex<PB>(cu_fsub<PB>(a.re, b.re), cu_fsub<PB>(a.im, b.im));
}
template <int PB>
__host__ __device__ static inline cu_fcomplex<PB> cu_cmul(const cu_fcomplex<PB> &a, const cu_fcomplex<PB> &b) {
  typename detail::core_of<PB>::type ar, ai, br, bi, rr, ri;
  detail::to_core<PB>(ar, a.re);
  detail::to_core<PB>(ai, a.im);
  detail::to_core<PB>(br, b.re);
  detail::to_core<PB>(bi, b.im);
  mpb::cmul(rr, ri, ar, ai, br, bi);
  return cu_fcomplex<PB>(detail::from_core<PB>(rr), detail::from_core<PB>(ri));
}

template <int PB>
__host__ __device__ static inline cu_fcomplex<PB> operator+(const cu_fcomplex<PB> &a, const cu_fcomplex<PB> &b) {
  return cu_cadd<PB>(a, b);
}
template <int PB>
__host__ __device__ static inline cu_fcomplex<PB> operator-(const cu_fcomplex<PB> &a, const cu_fcomplex<PB> &b) {
  return cu_csub<PB>(a, b);
}
template <int PB>
__host__ __device__ static inline cu_fcomplex<PB> operator*(const cu_fcomplex<PB> &a, const cu_fcomplex<PB> &b) {
  return cu_cmul<PB>(a, b);
}
/* a*b + c with one rounding per component (MPC mpc_fma semantics; not in
 * the reference): re = round(ar*br - ai*bi + cr), im = round(ar*bi + ai*br + ci)
 * from exact products */
template <int PB>
__host__ __device__ static inline cu_fcomplex<PB> cu_cfma(const cu_fcomplex<PB> &a, const cu_fcomplex<PB> &b,
                                                          const cu_fcomplex<PB> &c) {
  typename detail::core_of<PB>::type ar, ai, br, bi, cr, ci, rr, ri;
  detail::to_core<PB>(ar, a.re);
  detail::to_core<PB>(ai, a.im);
  detail::to_core<PB>(br, b.re);
  detail::to_core<PB>(bi, b.im);
  detail::to_core<PB>(cr, c.re);
  detail::to_core<PB>(ci, c.im);
  mpb::cfma(rr, ri, ar, ai, br, bi, cr, ci);
  return cu_fcomplex<PB>(detail::from_core<PB>(rr), detail::from_core<PB>(ri));
}

} /* namespace cu_fp */

#endif /* MPB_DROPIN_CU_FCOMPLEX_CUH */
