/* mpc_cuda/cu_fmath.cuh -- drop-in division and square root for cu_fp::cu_freal<PB>.
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
 * cu_exp / cu_log (reference cu_fmath.cuh:197-218) keep the reference's
 * contract: faithful, within 1 ULP of MPFR (mpb/elem.cuh: 128 guard bits).
 * The reference's other elementary functions (expm1, log1p, trigonometric,
 * hyperbolic, pow, cbrt) are not part of this engine.
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

/* exp(x), faithful (at most 1 ULP; exp of |x| >= 2^29 gives 0) */
template <int PB>
__host__ __device__ static inline cu_freal<PB> cu_exp(const cu_freal<PB> &x) {
  typename detail::core_of<PB>::type a, r;
  detail::to_core<PB>(a, x);
  mpb::exp_(r, a);
  return detail::from_core<PB>(r);
}

/* log(x), faithful (at most 1 ULP; x <= 0 gives 0) */
template <int PB>
__host__ __device__ static inline cu_freal<PB> cu_log(const cu_freal<PB> &x) {
  typename detail::core_of<PB>::type a, r;
  detail::to_core<PB>(a, x);
  mpb::log_(r, a);
  return detail::from_core<PB>(r);
}

} /* namespace cu_fp */

#endif /* MPB_DROPIN_CU_FMATH_CUH */
