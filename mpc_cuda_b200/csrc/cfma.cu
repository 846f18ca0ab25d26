/* cfma.cu -- complex fused multiply-add over arrays, r = a*b + c with one
 * rounding per component (the drop-in cu_cfma, MPC mpc_fma semantics).
 *
 * Each component is the correctly rounded sum of three exact terms (two
 * 2N-limb products and c), mpb::sum3_round in the core.  It lives in its own
 * translation unit because its PB=2048 instance is large and compiles slowly;
 * the rest of the library builds in parallel with it.  No counterpart in the
 * reference (its complex type has no fused multiply-add).
 */
#include <initializer_list>

#include "common.cuh"

namespace mpb {

constexpr int kBlock = 128;

template <int N>
__global__ void __launch_bounds__(kBlock) k_fma_c(size_t n, const uint8_t *a, const uint8_t *b, const uint8_t *c,
                                                  uint8_t *r) {
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> ar, ai, br, bi, cr, ci, zr, zi;
    load_celem<N, kStream>(ar, ai, a, i);
    load_celem<N, kStream>(br, bi, b, i);
    load_celem<N, kStream>(cr, ci, c, i);
    cfma<N, true>(zr, zi, ar, ai, br, bi, cr, ci);
    if (i < n) store_celem<N, kStream>(r, i, zr, zi);
  }
}
} /* namespace mpb */

using namespace mpb;

extern "C" int mpb_fma_c(int prec, size_t n, const void *a, const void *b, const void *c, void *r, void *stream) {
  if (!prec_ok(prec)) return MPB_ERR_PREC;
  if (n > kMaxElems) return MPB_ERR_SIZE;
  if (n == 0) return MPB_OK;
  for (const void *p : {a, b, c, (const void *)r}) {
    const int rc = check_buf(p);
    if (rc != MPB_OK) return rc;
  }
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_fma_c<N>, kBlock, tiles_for(n) * 32u);
    k_fma_c<N><<<g, kBlock, 0, as_stream(stream)>>>(n, (const uint8_t *)a, (const uint8_t *)b, (const uint8_t *)c,
                                                  (uint8_t *)r);
  });
  return launch_status();
}
