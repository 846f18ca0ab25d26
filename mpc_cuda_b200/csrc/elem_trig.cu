/* elem_trig.cu -- real elementary functions over arrays, trigonometric family
 * (the drop-in cu_sin, cu_cos, cu_tan, cu_atan, cu_asin, cu_acos and atan2,
 * mpb/elem.cuh; reference mpc_cuda include/mpc_cuda/cu_fmath.cuh:254-403,
 * cu_fcmath.cuh:20-29).  Launched through mpb_fmath_r (elem.cu). */
#include "common.cuh"
#include "mpb/elem.cuh"

namespace mpb {

constexpr int kBlock = 128;

template <int N>
__global__ void __launch_bounds__(kBlock) k_fmath_trig(int fn, size_t n, const uint8_t *a, const uint8_t *b,
                                                       uint8_t *r) {
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> x, y, z;
    load_elem<N, kStream>(x, a, i);
    switch (fn) {
      case MPB_FN_SIN: sin_<N>(z, x); break;
      case MPB_FN_COS: cos_<N>(z, x); break;
      case MPB_FN_TAN: tan_<N>(z, x); break;
      case MPB_FN_ATAN: atan_<N>(z, x); break;
      case MPB_FN_ASIN: asin_<N>(z, x); break;
      case MPB_FN_ACOS: acos_<N>(z, x); break;
      default: /* MPB_FN_ATAN2: atan2(a, b) */
        load_elem<N, kStream>(y, b, i);
        atan2_<N>(z, x, y);
    }
    if (i < n) store_elem<N, kStream>(r, i, z);
  }
}

/* arguments checked by mpb_fmath_r */
int fmath_trig_launch(int fn, int prec, size_t n, const void *a, const void *b, void *r, void *stream) {
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_fmath_trig<N>, kBlock, tiles_for(n) * 32u);
    k_fmath_trig<N><<<g, kBlock, 0, as_stream(stream)>>>(fn, n, (const uint8_t *)a, (const uint8_t *)b,
                                                         (uint8_t *)r);
  });
  return launch_status();
}

} /* namespace mpb */
