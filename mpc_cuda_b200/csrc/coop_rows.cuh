/* coop_rows.cuh -- warp-cooperative row kernels shared by the plain and the
 * batched GEMV: one row of y_out = A.x + y per group of G lanes (mpb/coop.cuh),
 * in the per-operation-rounded, sequential-k order of mpb_gemv_r
 * (acc = +0; acc = round(acc + round(A[i,k] x[k])); y_out[i] = round(acc + y[i])).
 * x[k] is the same element for every group of the warp, so its limbs are
 * uniform loads (one broadcast transaction), the uniform operand of the
 * cooperative product. */
#ifndef MPB_COOP_ROWS_CUH
#define MPB_COOP_ROWS_CUH

#include "common.cuh"
#include "mpb/coop.cuh"

namespace mpb {

/* words of shared memory one group needs for the row (coop::add) */
template <int N>
struct coop_row_smem {
  static constexpr int words = 3 * N + 3;
};

/* acc = row ir of A (starting at element arow) dotted with x, plus y[ir] */
template <int L, int G>
__device__ __forceinline__ void coop_gemv_row(coop::cv<L> &acc, const uint8_t *A, size_t arow, size_t n,
                                              const uint8_t *x, const uint8_t *y, size_t ir, uint32_t *sm) {
  constexpr int N = G * L;
  coop::set_zero(acc);
  for (size_t k = 0; k < n; ++k) { /* n is the same for the whole warp */
    coop::cv<L> a, t;
    coop::load<L, G>(a, A, arow + k);
    const coop::uref u = coop::uniform_ref<N>(x, k);
    int32_t ue;
    uint32_t us;
    coop::uniform_head<N>(u, ue, us);
    coop::mul_round_u<L, G>(t, a, u, ue, us);
    coop::add<L, G>(acc, acc, t, sm);
  }
  coop::cv<L> yv;
  coop::load<L, G>(yv, y, ir);
  coop::add<L, G>(acc, acc, yv, sm);
}

}  // namespace mpb

#endif /* MPB_COOP_ROWS_CUH */
