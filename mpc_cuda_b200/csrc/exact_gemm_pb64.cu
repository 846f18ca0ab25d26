/* exact_gemm_pb64.cu -- the exact GEMM's kernels instantiated for PB = 64
 * (N = 2 limbs); one translation unit per precision keeps the build parallel. */
#include "exact_gemm.cuh"

namespace mpb {
namespace exact {
template int run_exact_n<2>(const Plan &, const uint8_t *, size_t, const uint8_t *, size_t, uint8_t *, size_t,
                             uint8_t *, int *, cudaStream_t);
} /* namespace exact */
} /* namespace mpb */
