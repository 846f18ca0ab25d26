/* exact_gemm_pb1024.cu -- the exact GEMM's kernels instantiated for PB = 1024
 * (N = 32 limbs); one translation unit per precision keeps the build parallel. */
#include "exact_gemm.cuh"

namespace mpb {
namespace exact {
template int run_exact_n<32>(const Plan &, const uint8_t *, size_t, const uint8_t *, size_t, uint8_t *, size_t,
                             uint8_t *, int *, cudaStream_t);
} /* namespace exact */
} /* namespace mpb */
