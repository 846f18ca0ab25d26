/* mpc_cuda/cu_fmath.cuh -- drop-in division, square root and elementary
 * functions for cu_fp::cu_freal<PB>.
 *
 * The reference header of this name (mpc_cuda include/mpc_cuda/cu_fmath.cuh)
 * computes cu_fdiv (cu_fmath.cuh:67-75) and cu_sqrt (cu_fmath.cuh:92-100) by
 * Newton iteration at a guard precision: faithful, within about one ULP of
 * MPFR.  These have the same names and arguments and return the correctly
 * rounded result (MPFR mpfr_div / mpfr_sqrt, RNDN) instead: the mpb core
 * divides the significands exactly (long division with a remainder) and
 * takes an exact integer square root, so the round and sticky bits are
 * known.  A quotient by zero or the square root of a negative number has no
 * value in this format (no infinities or NaN): the result is 0.
 *
 * The elementary functions (reference cu_fmath.cuh:119-424: cu_exp, cu_log,
 * cu_expm1, cu_log1p, cu_sin, cu_cos, cu_tan, cu_atan, cu_sinh, cu_cosh,
 * cu_atanh, cu_asin, cu_acos, cu_cbrt, cu_pow, cu_div_ui, cu_pi, cu_ln2) keep
 * the reference's names, arguments and contract: faithful, within 1 ULP of
 * MPFR (mpb/elem.cuh: 128 guard bits); cu_div_ui, cu_pi and cu_ln2 are
 * correctly rounded.  The complex ones are in cu_fcmath.cuh.
 */
#ifndef MPB_DROPIN_CU_FMATH_CUH
#define MPB_DROPIN_CU_FMATH_CUH

#include "cu_freal.cuh"
#include "../mpb/elem.cuh"

namespace cu_fp {

/* round(a / b), one rounding (mpfr_div) */
template <int PB>
__host__ __device__ static inline cu_freal<PB> cu_fdiv(const cu_freal<PB> &a, const cu_freal<PB> &b) {
  typename detail::core_of<PB>::type x, y, r;
  detail::to_core<PB>(x, a);
  detail::to_core<PB>(y, b);
  mpb::div(r, x, y);
  return detail::from_core<PB>(r);
}

/* round(sqrt(x)), one rounding (mpfr_sqrt) */
template <int PB>
__host__ __device__ static inline cu_freal<PB> cu_sqrt(const cu_freal<PB> &x) {
  typename detail::core_of<PB>::type a, r;
  detail::to_core<PB>(a, x);
  mpb::sqrt_(r, a);
  return detail::from_core<PB>(r);
}

/* The elementary functions: faithful (at most 1 ULP; in practice almost
 * always correctly rounded), computed at PB + 128 bits and rounded once --
 * the reference's contract and guard width (cu_fmath.cuh:20-22).  Results
 * with no value in this format are 0: exp / sinh / cosh of |x| >= 2^29,
 * sin / cos / tan of |x| >= 2^30, log of x <= 0, log1p of x <= -1, atanh of
 * |x| >= 1, pow of a negative base and a non-integer exponent. */
#define MPB_DROPIN_UNARY(name, core)                                            \
  template <int PB>                                                            \
  __host__ __device__ static inline cu_freal<PB> name(const cu_freal<PB> &x) { \
    typename detail::core_of<PB>::type a, r;                                   \
    detail::to_core<PB>(a, x);                                                 \
    mpb::core(r, a);                                                           \
    return detail::from_core<PB>(r);                                           \
  }
MPB_DROPIN_UNARY(cu_exp, exp_)     /* reference cu_fmath.cuh:197-201 */
MPB_DROPIN_UNARY(cu_log, log_)     /* :214-218 */
MPB_DROPIN_UNARY(cu_expm1, expm1_) /* :234-237 */
MPB_DROPIN_UNARY(cu_log1p, log1p_) /* :247-250 */
MPB_DROPIN_UNARY(cu_sin, sin_)     /* :293-297 */
MPB_DROPIN_UNARY(cu_cos, cos_)     /* :299-303 */
MPB_DROPIN_UNARY(cu_tan, tan_)     /* :305-310 */
MPB_DROPIN_UNARY(cu_atan, atan_)   /* :329-332 (|x| >= 1 through pi/2 - atan(1/x)) */
MPB_DROPIN_UNARY(cu_sinh, sinh_)   /* :353-355 */
MPB_DROPIN_UNARY(cu_cosh, cosh_)   /* :356-358 */
MPB_DROPIN_UNARY(cu_atanh, atanh_) /* :373-375 */
MPB_DROPIN_UNARY(cu_asin, asin_)   /* :389-391 (|x| >= 1 gives +-pi/2) */
MPB_DROPIN_UNARY(cu_acos, acos_)   /* :401-403 (x >= 1 gives 0, x <= -1 pi) */
MPB_DROPIN_UNARY(cu_cbrt, cbrt_)   /* :119-127 (sign kept) */
#undef MPB_DROPIN_UNARY

/* x^y (reference cu_fmath.cuh:420-424): y = 0 gives 1, x = 0 gives 0, a
 * negative x needs an integer y */
template <int PB>
__host__ __device__ static inline cu_freal<PB> cu_pow(const cu_freal<PB> &x, const cu_freal<PB> &y) {
  typename detail::core_of<PB>::type a, b, r;
  detail::to_core<PB>(a, x);
  detail::to_core<PB>(b, y);
  mpb::pow_(r, a, b);
  return detail::from_core<PB>(r);
}

/* atan2(y, x) in (-pi, pi] ((0, 0) gives 0; the reference's cu_atan2_w,
 * cu_fcmath.cuh:18-29, at the type's precision) */
template <int PB>
__host__ __device__ static inline cu_freal<PB> cu_atan2(const cu_freal<PB> &y, const cu_freal<PB> &x) {
  typename detail::core_of<PB>::type a, b, r;
  detail::to_core<PB>(a, y);
  detail::to_core<PB>(b, x);
  mpb::atan2_(r, a, b);
  return detail::from_core<PB>(r);
}

/* round(x / u), one rounding (reference cu_div_ui, cu_fmath.cuh:32-50) */
template <int PB>
__host__ __device__ static inline cu_freal<PB> cu_div_ui(const cu_freal<PB> &x, unsigned long long u) {
  typename detail::core_of<PB>::type a, r;
  if (u == 1ull) return x;
  detail::to_core<PB>(a, x);
  mpb::div_u64(r, a, (uint64_t)u);
  return detail::from_core<PB>(r);
}

/* pi and ln 2, correctly rounded (reference cu_pi / cu_ln2, cu_fmath.cuh:174-175) */
template <int PB>
__host__ __device__ static inline cu_freal<PB> cu_pi() {
  typename detail::core_of<PB>::type r;
  mpb::pi_(r);
  return detail::from_core<PB>(r);
}
template <int PB>
__host__ __device__ static inline cu_freal<PB> cu_ln2() {
  typename detail::core_of<PB>::type r;
  mpb::ln2_(r);
  return detail::from_core<PB>(r);
}

} /* namespace cu_fp */

#endif /* MPB_DROPIN_CU_FMATH_CUH */
