/* rprec.cu -- element-wise arithmetic at a runtime precision (mpb/rprec.cuh):
 * round to odd at the storage format's PB bits, then to nearest at p bits. */
#include <initializer_list>

#include "common.cuh"
#include "mpb/rprec.cuh"

namespace mpb {

constexpr int kBlock = 128;

template <int N>
__global__ void __launch_bounds__(kBlock) k_op_rp(int op, int p, size_t n, const uint8_t *a, const uint8_t *b,
                                                  const uint8_t *c, uint8_t *r) {
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> x, y, z, o;
    load_elem<N, kStream>(x, a, i);
    if (op != MPB_RP_SQRT) load_elem<N, kStream>(y, b, i);
    if (op == MPB_RP_FMA) load_elem<N, kStream>(z, c, i);
    op_rp<N>(op, p, o, x, y, z);
    if (i < n) store_elem<N, kStream>(r, i, o);
  }
}

} /* namespace mpb */

using namespace mpb;

extern "C" int mpb_storage_prec(int prec) {
  if (prec < 1) return MPB_ERR_PREC;
  for (int pb : {64, 128, 256, 512, 1024, 2048})
    if (pb >= prec + 2) return pb;
  return MPB_ERR_PREC;
}

extern "C" int mpb_op_rp(int op, int prec, size_t n, const void *a, const void *b, const void *c, void *r,
                         void *stream) {
  if (op < MPB_RP_MUL || op > MPB_RP_SQRT) return MPB_ERR_ARG;
  const int pb = mpb_storage_prec(prec);
  if (pb < 0) return MPB_ERR_PREC;
  if (n > kMaxElems) return MPB_ERR_SIZE;
  if (n == 0) return MPB_OK;
  for (const void *q : {a, op == MPB_RP_SQRT ? a : b, op == MPB_RP_FMA ? c : a, (const void *)r}) {
    const int rc = check_buf(q);
    if (rc != MPB_OK) return rc;
  }
  MPB_DISPATCH_PREC(pb, {
    const int g = grid_for(k_op_rp<N>, kBlock, tiles_for(n) * 32u);
    k_op_rp<N><<<g, kBlock, 0, as_stream(stream)>>>(op, prec, n, (const uint8_t *)a, (const uint8_t *)b,
                                                   (const uint8_t *)c, (uint8_t *)r);
  });
  return launch_status();
}
