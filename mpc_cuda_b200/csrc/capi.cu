/* capi.cu -- library information and layout queries of the mpb C ABI. */
#include <mutex>

#include "common.cuh"

namespace mpb {

int sm_count() {
  static int cached[64];
  static std::once_flag once[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  std::call_once(once[dev], [dev] {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v < 1) v = 148;
    cached[dev] = v;
  });
  return cached[dev];
}

} /* namespace mpb */

extern "C" int mpb_version(void) { return 100; }

extern "C" const char *mpb_status_string(int status) {
  switch (status) {
    case MPB_OK:
      return "ok";
    case MPB_ERR_PREC:
      return "unsupported precision (use 64, 128, 256, 512, 1024 or 2048)";
    case MPB_ERR_SIZE:
      return "size out of range";
    case MPB_ERR_NULL:
      return "null pointer";
    case MPB_ERR_ALIGN:
      return "device buffer not 16-byte aligned";
    case MPB_ERR_LD:
      return "leading dimension not a multiple of 32 or smaller than the row length";
    case MPB_ERR_CUDA:
      return "CUDA error";
    case MPB_ERR_ARG:
      return "invalid argument";
    case MPB_ERR_WORKSPACE:
      return "workspace missing or too small";
    default:
      return "unknown status";
  }
}

extern "C" int mpb_prec_supported(int prec) { return mpb::prec_ok(prec) ? 1 : 0; }

extern "C" size_t mpb_vec_bytes(int prec, size_t n) {
  if (!mpb::prec_ok(prec) || n > mpb::kMaxElems) return 0;
  return mpb::tiles_for(n) * mpb::tile_bytes_for(prec / 32);
}
extern "C" size_t mpb_cvec_bytes(int prec, size_t n) { return 2u * mpb_vec_bytes(prec, n); }
extern "C" size_t mpb_aos_bytes(int prec) {
  if (!mpb::prec_ok(prec)) return 0;
  return 16u + 8u * (size_t)((prec + 63) / 64);
}
