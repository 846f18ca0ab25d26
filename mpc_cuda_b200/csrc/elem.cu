/* elem.cu -- exponential and logarithm over arrays (the drop-in cu_exp /
 * cu_log, mpb/elem.cuh): faithful, the contract of the reference's cu_exp /
 * cu_log (mpc_cuda include/mpc_cuda/cu_fmath.cuh:197-218), computed at 128
 * guard bits with the core's correctly rounded operations.  Own translation
 * unit: the PB=2048 instances work at 68 limbs and are large.
 */
#include <initializer_list>

#include "common.cuh"
#include "mpb/elem.cuh"

namespace mpb {

constexpr int kBlock = 128;

template <int N, int OP>
__global__ void __launch_bounds__(kBlock) k_elem_r(size_t n, const uint8_t *a, uint8_t *r) {
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> x, z;
    load_elem<N, kStream>(x, a, i);
    if (OP == 0)
      exp_<N>(z, x);
    else
      log_<N>(z, x);
    if (i < n) store_elem<N, kStream>(r, i, z);
  }
}

template <int OP>
static int elem_entry(int prec, size_t n, const void *a, void *r, void *stream) {
  if (!prec_ok(prec)) return MPB_ERR_PREC;
  if (n > kMaxElems) return MPB_ERR_SIZE;
  if (n == 0) return MPB_OK;
  for (const void *p : {a, (const void *)r}) {
    const int rc = check_buf(p);
    if (rc != MPB_OK) return rc;
  }
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_elem_r<N, OP>, kBlock, tiles_for(n) * 32u);
    k_elem_r<N, OP><<<g, kBlock, 0, as_stream(stream)>>>(n, (const uint8_t *)a, (uint8_t *)r);
  });
  return launch_status();
}

} /* namespace mpb */

using namespace mpb;

extern "C" int mpb_exp_r(int prec, size_t n, const void *a, void *r, void *stream) {
  return elem_entry<0>(prec, n, a, r, stream);
}
extern "C" int mpb_log_r(int prec, size_t n, const void *a, void *r, void *stream) {
  return elem_entry<1>(prec, n, a, r, stream);
}
