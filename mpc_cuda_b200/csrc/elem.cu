/* elem.cu -- real elementary functions over arrays, exponential and
 * logarithm family (the drop-in cu_exp, cu_log, cu_expm1, cu_log1p, cu_sinh,
 * cu_cosh, cu_atanh, cu_cbrt, cu_pow, mpb/elem.cuh), plus cu_div_ui and the
 * constants cu_pi / cu_ln2.  Faithful, the contract of the reference's
 * cu_fmath functions (mpc_cuda include/mpc_cuda/cu_fmath.cuh:1-14), computed
 * at 128 guard bits with the core's correctly rounded operations.
 *
 * mpb_fmath_r dispatches by function: this unit's family here, the
 * trigonometric one to elem_trig.cu.  One kernel per precision takes the
 * function as an argument (uniform across the grid); the functions are
 * out-of-line calls, so each precision's code holds one copy of every
 * building block.  Own translation units: the PB=2048 instances work at 68
 * limbs and are large.
 */
#include <initializer_list>

#include "common.cuh"
#include "mpb/elem.cuh"

namespace mpb {

constexpr int kBlock = 128;

int fmath_trig_launch(int fn, int prec, size_t n, const void *a, const void *b, void *r, void *stream);

template <int N>
__global__ void __launch_bounds__(kBlock) k_fmath_exp(int fn, size_t n, const uint8_t *a, const uint8_t *b,
                                                      uint8_t *r) {
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> x, y, z;
    load_elem<N, kStream>(x, a, i);
    switch (fn) {
      case MPB_FN_EXP: exp_<N>(z, x); break;
      case MPB_FN_LOG: log_<N>(z, x); break;
      case MPB_FN_EXPM1: expm1_<N>(z, x); break;
      case MPB_FN_LOG1P: log1p_<N>(z, x); break;
      case MPB_FN_SINH: sinh_<N>(z, x); break;
      case MPB_FN_COSH: cosh_<N>(z, x); break;
      case MPB_FN_ATANH: atanh_<N>(z, x); break;
      case MPB_FN_CBRT: cbrt_<N>(z, x); break;
      default: /* MPB_FN_POW */
        load_elem<N, kStream>(y, b, i);
        pow_<N>(z, x, y);
    }
    if (i < n) store_elem<N, kStream>(r, i, z);
  }
}

template <int N>
__global__ void __launch_bounds__(kBlock) k_div_ui(size_t n, const uint8_t *a, uint64_t u, uint8_t *r) {
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> x, z;
    load_elem<N, kStream>(x, a, i);
    if (u == 1u)
      z = x;
    else
      div_u64<N>(z, x, u);
    if (i < n) store_elem<N, kStream>(r, i, z);
  }
}

template <int N>
__global__ void __launch_bounds__(kBlock) k_const(int which, size_t n, uint8_t *r) {
  const size_t np = tiles_for(n) * 32u;
  fval<N> c;
  if (which == 0)
    pi_<N>(c);
  else
    ln2_<N>(c);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x)
    if (i < n) store_elem<N, kStream>(r, i, c);
}

static int check_args(int prec, size_t n, std::initializer_list<const void *> bufs) {
  if (!prec_ok(prec)) return MPB_ERR_PREC;
  if (n > kMaxElems) return MPB_ERR_SIZE;
  if (n == 0) return MPB_OK;
  for (const void *p : bufs) {
    const int rc = check_buf(p);
    if (rc != MPB_OK) return rc;
  }
  return MPB_OK;
}

static bool binary_fn(int fn) { return fn == MPB_FN_POW || fn == MPB_FN_ATAN2; }

} /* namespace mpb */

using namespace mpb;

extern "C" int mpb_fmath_r(int fn, int prec, size_t n, const void *a, const void *b, void *r, void *stream) {
  if (fn < MPB_FN_EXP || fn > MPB_FN_ATAN2) return MPB_ERR_ARG;
  const int rc = binary_fn(fn) ? check_args(prec, n, {a, b, (const void *)r}) : check_args(prec, n, {a, (const void *)r});
  if (rc != MPB_OK || n == 0) return rc;
  switch (fn) {
    case MPB_FN_SIN:
    case MPB_FN_COS:
    case MPB_FN_TAN:
    case MPB_FN_ATAN:
    case MPB_FN_ASIN:
    case MPB_FN_ACOS:
    case MPB_FN_ATAN2:
      return fmath_trig_launch(fn, prec, n, a, b, r, stream);
    default:
      break;
  }
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_fmath_exp<N>, kBlock, tiles_for(n) * 32u);
    k_fmath_exp<N><<<g, kBlock, 0, as_stream(stream)>>>(fn, n, (const uint8_t *)a, (const uint8_t *)b, (uint8_t *)r);
  });
  return launch_status();
}

extern "C" int mpb_exp_r(int prec, size_t n, const void *a, void *r, void *stream) {
  return mpb_fmath_r(MPB_FN_EXP, prec, n, a, nullptr, r, stream);
}
extern "C" int mpb_log_r(int prec, size_t n, const void *a, void *r, void *stream) {
  return mpb_fmath_r(MPB_FN_LOG, prec, n, a, nullptr, r, stream);
}

extern "C" int mpb_div_ui_r(int prec, size_t n, const void *a, uint64_t u, void *r, void *stream) {
  const int rc = check_args(prec, n, {a, (const void *)r});
  if (rc != MPB_OK || n == 0) return rc;
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_div_ui<N>, kBlock, tiles_for(n) * 32u);
    k_div_ui<N><<<g, kBlock, 0, as_stream(stream)>>>(n, (const uint8_t *)a, u, (uint8_t *)r);
  });
  return launch_status();
}

extern "C" int mpb_const_r(int which, int prec, size_t n, void *r, void *stream) {
  if (which != MPB_CONST_PI && which != MPB_CONST_LN2) return MPB_ERR_ARG;
  const int rc = check_args(prec, n, {(const void *)r});
  if (rc != MPB_OK || n == 0) return rc;
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_const<N>, kBlock, tiles_for(n) * 32u);
    k_const<N><<<g, kBlock, 0, as_stream(stream)>>>(which, n, (uint8_t *)r);
  });
  return launch_status();
}
