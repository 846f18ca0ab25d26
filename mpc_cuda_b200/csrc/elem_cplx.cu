/* elem_cplx.cu -- complex elementary functions over arrays (the drop-in
 * cu_cexp, cu_clog, cu_csqrt, cu_csin, cu_ccos, cu_ctan, cu_csinh, cu_ccosh,
 * cu_cdiv; mpb/elem.cuh cfunc_ / cdiv_; reference mpc_cuda
 * include/mpc_cuda/cu_fcmath.cuh:31-113): each component faithful. */
#include <initializer_list>

#include "common.cuh"
#include "mpb/elem.cuh"

namespace mpb {

constexpr int kBlock = 128;

template <int N>
__global__ void __launch_bounds__(kBlock) k_fmath_c(int fn, size_t n, const uint8_t *a, const uint8_t *b,
                                                    uint8_t *r) {
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> zr, zi, wr, wi, rr, ri;
    load_celem<N, kStream>(zr, zi, a, i);
    if (fn == MPB_CFN_DIV) {
      load_celem<N, kStream>(wr, wi, b, i);
      cdiv_<N>(rr, ri, zr, zi, wr, wi);
    } else {
      cfunc_<N>(fn, rr, ri, zr, zi);
    }
    if (i < n) store_celem<N, kStream>(r, i, rr, ri);
  }
}

} /* namespace mpb */

using namespace mpb;

extern "C" int mpb_fmath_c(int fn, int prec, size_t n, const void *a, const void *b, void *r, void *stream) {
  if (fn < MPB_CFN_EXP || fn > MPB_CFN_DIV) return MPB_ERR_ARG;
  if (!prec_ok(prec)) return MPB_ERR_PREC;
  if (n > kMaxElems) return MPB_ERR_SIZE;
  if (n == 0) return MPB_OK;
  for (const void *p : {a, fn == MPB_CFN_DIV ? b : a, (const void *)r}) {
    const int rc = check_buf(p);
    if (rc != MPB_OK) return rc;
  }
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_fmath_c<N>, kBlock, tiles_for(n) * 32u);
    k_fmath_c<N><<<g, kBlock, 0, as_stream(stream)>>>(fn, n, (const uint8_t *)a, (const uint8_t *)b, (uint8_t *)r);
  });
  return launch_status();
}
