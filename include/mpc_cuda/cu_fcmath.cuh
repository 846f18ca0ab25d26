/* mpc_cuda/cu_fcmath.cuh -- drop-in complex elementary functions for
 * cu_fp::cu_fcomplex<PB>.
 *
 * Same names and arguments as the reference header of this name (mpc_cuda
 * include/mpc_cuda/cu_fcmath.cuh:13-113): cu_cconvert, cu_cdiv, cu_cexp,
 * cu_clog, cu_csqrt, cu_csin, cu_ccos, cu_ctan, cu_csinh, cu_ccosh.  The
 * reference computes them at PB + 128 bits from its real functions and
 * promises about 1 ULP per component against MPC (cu_fcmath.cuh:1-5); these
 * work at the same guard width on the mpb core (mpb/elem.cuh cfunc_ /
 * cdiv_) and are faithful per component, with these changes of formula
 * where the reference's loses accuracy:
 *   clog   log|z| = log1p(|z|^2 - 1) / 2 near |z| = 1, the three-term sum with
 *          one rounding (the reference takes log of a rounded |z|^2);
 *   ctan   (sin x cos x + i sinh y cosh y) / (cos^2 x + sinh^2 y), whose
 *          denominator never cancels (the reference divides csin by ccos);
 *   cdiv   numerators and |b|^2 each with one rounding (fmma / fmms).
 * Components with no value in this format are 0 (exp / sinh / cosh overflow,
 * sin / cos of |x| >= 2^30, division by zero, log of zero).
 */
#ifndef MPB_DROPIN_CU_FCMATH_CUH
#define MPB_DROPIN_CU_FCMATH_CUH

#include "cu_fcomplex.cuh"
#include "cu_fmath.cuh"

namespace cu_fp {

template <int TO, int FROM>
__host__ __device__ static inline cu_fcomplex<TO> cu_cconvert(const cu_fcomplex<FROM> &z) {
  return cu_fcomplex<TO>(cu_convert<TO>(z.re), cu_convert<TO>(z.im));
}

/* a / b (b = 0 gives 0) */
template <int PB>
__host__ __device__ static inline cu_fcomplex<PB> cu_cdiv(const cu_fcomplex<PB> &a, const cu_fcomplex<PB> &b) {
  typename detail::core_of<PB>::type ar, ai, br, bi, rr, ri;
  detail::to_core<PB>(ar, a.re);
  detail::to_core<PB>(ai, a.im);
  detail::to_core<PB>(br, b.re);
  detail::to_core<PB>(bi, b.im);
  mpb::cdiv_(rr, ri, ar, ai, br, bi);
  return cu_fcomplex<PB>(detail::from_core<PB>(rr), detail::from_core<PB>(ri));
}

namespace detail {
template <int PB>
__host__ __device__ inline cu_fcomplex<PB> cfunc(int c, const cu_fcomplex<PB> &z) {
  typename core_of<PB>::type zr, zi, rr, ri;
  to_core<PB>(zr, z.re);
  to_core<PB>(zi, z.im);
  mpb::cfunc_(c, rr, ri, zr, zi);
  return cu_fcomplex<PB>(from_core<PB>(rr), from_core<PB>(ri));
}
}  // namespace detail

#define MPB_DROPIN_CFUNC(name, c)                                                    \
  template <int PB>                                                                 \
  __host__ __device__ static inline cu_fcomplex<PB> name(const cu_fcomplex<PB> &z) { \
    return detail::cfunc<PB>(c, z);                                                 \
  }
MPB_DROPIN_CFUNC(cu_cexp, 0)  /* e^x (cos y + i sin y) */
MPB_DROPIN_CFUNC(cu_clog, 1)  /* log|z| + i atan2(y, x) */
MPB_DROPIN_CFUNC(cu_csqrt, 2) /* principal root */
MPB_DROPIN_CFUNC(cu_csin, 3)
MPB_DROPIN_CFUNC(cu_ccos, 4)
MPB_DROPIN_CFUNC(cu_ctan, 5)
MPB_DROPIN_CFUNC(cu_csinh, 6)
MPB_DROPIN_CFUNC(cu_ccosh, 7)
#undef MPB_DROPIN_CFUNC

} /* namespace cu_fp */

#endif /* MPB_DROPIN_CU_FCMATH_CUH */
