/* divsqrt.cu -- correctly rounded division and square root over arrays
 * (the drop-in cu_fdiv / cu_sqrt; MPFR mpfr_div / mpfr_sqrt semantics).
 *
 * The reference's cu_fdiv and cu_sqrt (mpc_cuda include/mpc_cuda/cu_fmath.cuh:
 * 67-75, 92-100) are Newton iterations at a guard precision, faithful only;
 * these round the exact quotient / square root once.  The core does an exact
 * long division of the significands (mpb::div) and an exact integer square
 * root (mpb::sqrt_: integer Newton with a long division per step).  Kept in
 * its own translation unit: the PB=2048 instances are large.
 */
#include <initializer_list>

#include "common.cuh"

namespace mpb {

constexpr int kBlock = 128;

template <int N>
__global__ void __launch_bounds__(kBlock) k_div_r(size_t n, const uint8_t *a, const uint8_t *b, uint8_t *r) {
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> x, y, z;
    load_elem<N, kStream>(x, a, i);
    load_elem<N, kStream>(y, b, i);
    div<N>(z, x, y);
    if (i < n) store_elem<N, kStream>(r, i, z);
  }
}
template <int N>
__global__ void __launch_bounds__(kBlock) k_sqrt_r(size_t n, const uint8_t *a, uint8_t *r) {
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> x, z;
    load_elem<N, kStream>(x, a, i);
    sqrt_<N>(z, x);
    if (i < n) store_elem<N, kStream>(r, i, z);
  }
}

static int args_ok(int prec, size_t n, std::initializer_list<const void *> bufs) {
  if (!prec_ok(prec)) return MPB_ERR_PREC;
  if (n > kMaxElems) return MPB_ERR_SIZE;
  if (n == 0) return 1;
  for (const void *p : bufs) {
    const int rc = check_buf(p);
    if (rc != MPB_OK) return rc;
  }
  return MPB_OK;
}

} /* namespace mpb */

using namespace mpb;

extern "C" int mpb_div_r(int prec, size_t n, const void *a, const void *b, void *r, void *stream) {
  const int rc = args_ok(prec, n, {a, b, r});
  if (rc != MPB_OK) return rc > 0 ? MPB_OK : rc;
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_div_r<N>, kBlock, tiles_for(n) * 32u);
    k_div_r<N><<<g, kBlock, 0, as_stream(stream)>>>(n, (const uint8_t *)a, (const uint8_t *)b, (uint8_t *)r);
  });
  return launch_status();
}
extern "C" int mpb_sqrt_r(int prec, size_t n, const void *a, void *r, void *stream) {
  const int rc = args_ok(prec, n, {a, r});
  if (rc != MPB_OK) return rc > 0 ? MPB_OK : rc;
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_sqrt_r<N>, kBlock, tiles_for(n) * 32u);
    k_sqrt_r<N><<<g, kBlock, 0, as_stream(stream)>>>(n, (const uint8_t *)a, (uint8_t *)r);
  });
  return launch_status();
}
