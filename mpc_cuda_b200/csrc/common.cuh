/* common.cuh -- shared host-side plumbing of the mpb C ABI: precision dispatch,
 * argument validation, grid sizing.  Internal header (not installed). */
#ifndef MPB_COMMON_CUH
#define MPB_COMMON_CUH

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <utility>

#include "mpb.h"
#include "mpb/layout.cuh"

namespace mpb {

/* largest element count any entry point accepts (2^40) */
constexpr size_t kMaxElems = (size_t)1 << 40;

inline bool prec_ok(int prec) {
  return prec == 64 || prec == 128 || prec == 256 || prec == 512 || prec == 1024 || prec == 2048;
}
inline bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }
inline cudaStream_t as_stream(void *s) { return (cudaStream_t)s; }

/* a device buffer argument: required when count > 0 */
inline int check_buf(const void *p) {
  if (!p) return MPB_ERR_NULL;
  if (!aligned16(p)) return MPB_ERR_ALIGN;
  return MPB_OK;
}

inline int launch_status() {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MPB_OK : MPB_ERR_CUDA;
}

/* SM count of the current device (cached per device) */
int sm_count();

/* Programmatic dependent launch: a kernel launched with launch_pdl may start
 * (be scheduled, run its prologue) while the kernel before it on the stream
 * is finishing; it must call pdl_wait() before it touches memory that kernel
 * writes.  pdl_wait() waits for the whole previous grid and the visibility of
 * its writes; in a kernel launched normally it returns at once.  Used along
 * the chains of small dependent launches, where it hides the launch latency
 * between them. */
__device__ __forceinline__ void pdl_wait() {
#if defined(__CUDA_ARCH__)
  asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

/* thread-vs-warp split (mpb_set_split): lanes per element for a kind and
 * precision, 1 = one thread per element */
constexpr int kSplitKinds = 2;
constexpr int kDefaultSplit1024 = 8;      /* GEMV rows at 1024 bits */
constexpr int kDefaultSplit2048 = 8;      /* GEMV rows at 2048 bits */
constexpr int kDefaultSplitAxpyC1024 = 1; /* complex AXPY elements at 1024 bits */
int split_lanes(int kind, int prec);
bool split_supported(int kind, int prec, int lanes);

/* plain GEMM warps per block (mpb_set_gemm_warps): 4, 8 or 16 */
constexpr int kDefaultGemmWarps = 8;
int gemm_warps(int cplx, int prec);

/* Opt-in phase timing (mpb_profile_enable): entry points that run several
 * kernels record a CUDA event pair around each phase on the caller's stream. */
enum {
  kPhaseStats = 0,
  kPhaseSlice = 1,
  kPhaseTensor = 2,
  kPhaseRound = 3,
  kPhaseFallback = 4,
  kPhaseTensorLow = 5, /* recomputation of the low diagonals of marked tiles */
  kPhases = 6
};
void profile_mark(int phase, bool begin, cudaStream_t st);

/* Grid for a grid-stride kernel over `work` warp-sized units of 32 threads
 * each: enough blocks to fill every SM at the kernel's occupancy, never more
 * than the work needs. */
template <typename K>
inline int grid_for(K kernel, int block, size_t threads_needed) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const size_t full = (size_t)sm_count() * (size_t)per_sm;
  const size_t need = (threads_needed + (size_t)block - 1) / (size_t)block;
  size_t g = need < full ? need : full;
  if (g < 1) g = 1;
  return (int)g;
}

} /* namespace mpb */

/* runtime precision -> compile-time limb count N (32-bit limbs) */
#define MPB_DISPATCH_PREC(prec, ...)            \
  switch (prec) {                               \
    case 64: {                                  \
      constexpr int N = 2;                      \
      __VA_ARGS__;                              \
    } break;                                    \
    case 128: {                                 \
      constexpr int N = 4;                      \
      __VA_ARGS__;                              \
    } break;                                    \
    case 256: {                                 \
      constexpr int N = 8;                      \
      __VA_ARGS__;                              \
    } break;                                    \
    case 512: {                                 \
      constexpr int N = 16;                     \
      __VA_ARGS__;                              \
    } break;                                    \
    case 1024: {                                \
      constexpr int N = 32;                     \
      __VA_ARGS__;                              \
    } break;                                    \
    case 2048: {                                \
      constexpr int N = 64;                     \
      __VA_ARGS__;                              \
    } break;                                    \
    default:                                    \
      return MPB_ERR_PREC;                      \
  }

#endif /* MPB_COMMON_CUH */
