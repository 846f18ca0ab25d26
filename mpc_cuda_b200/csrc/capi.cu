/* capi.cu -- library information and layout queries of the mpb C ABI. */
#include <atomic>
#include <mutex>
#include <utility>
#include <vector>

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

/* ---------------- opt-in phase timing ---------------- */
/* Each recorded interval is an event pair taken from a growing pool; the
 * intervals of every call since mpb_profile_enable(1) are kept and summed. */
static std::atomic<int> g_profile{0};
static std::atomic<unsigned> g_profile_mask{~0u}; /* phases that record events */
static std::mutex g_prof_mu;
static std::vector<cudaEvent_t> g_pool;
static size_t g_pool_used = 0;
static std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_iv[kPhases];
static cudaEvent_t g_open[kPhases];

static cudaEvent_t next_event() {
  if (g_pool_used == g_pool.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    g_pool.push_back(e);
  }
  return g_pool[g_pool_used++];
}

void profile_mark(int phase, bool begin, cudaStream_t st) {
  if (!g_profile.load(std::memory_order_relaxed) || phase < 0 || phase >= kPhases) return;
  if (!((g_profile_mask.load(std::memory_order_relaxed) >> phase) & 1u)) return;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  cudaEvent_t e = next_event();
  if (!e) return;
  /* inside a stream capture a plain record only orders the capture; an
   * external record becomes a node that records the event at every replay */
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusActive)
    cudaEventRecordWithFlags(e, st, cudaEventRecordExternal);
  else
    cudaEventRecord(e, st);
  if (begin)
    g_open[phase] = e;
  else if (g_open[phase])
    g_iv[phase].emplace_back(g_open[phase], e), g_open[phase] = nullptr;
}

/* ---------------- thread-vs-warp split ---------------- */
/* lanes per element of the kernels that have a warp-cooperative form, per
 * kind and precision group (64 .. 2048); 1 = one thread per element */
static std::atomic<int> g_split[kSplitKinds][6];
static std::once_flag g_split_once;

static int prec_group(int prec) {
  switch (prec) {
    case 64: return 0;
    case 128: return 1;
    case 256: return 2;
    case 512: return 3;
    case 1024: return 4;
    case 2048: return 5;
    default: return -1;
  }
}

bool split_supported(int kind, int prec, int lanes) {
  if (kind < 0 || kind >= kSplitKinds || prec_group(prec) < 0) return false;
  if (lanes == 1) return true;
  if (kind == MPB_SPLIT_AXPY_C) return prec == 1024 && (lanes == 4 || lanes == 8);
  if (prec == 1024) return lanes == 4 || lanes == 8;
  if (prec == 2048) return lanes == 8 || lanes == 16;
  return false;
}

static void split_defaults() {
  for (int k = 0; k < kSplitKinds; ++k)
    for (int g = 0; g < 6; ++g) g_split[k][g].store(1, std::memory_order_relaxed);
  /* measured on B200: the cooperative forms win from 1024 bits on */
  g_split[MPB_SPLIT_GEMV_R][4].store(kDefaultSplit1024, std::memory_order_relaxed);
  g_split[MPB_SPLIT_GEMV_R][5].store(kDefaultSplit2048, std::memory_order_relaxed);
  g_split[MPB_SPLIT_AXPY_C][4].store(kDefaultSplitAxpyC1024, std::memory_order_relaxed);
}

int split_lanes(int kind, int prec) {
  std::call_once(g_split_once, split_defaults);
  const int g = prec_group(prec);
  if (kind < 0 || kind >= kSplitKinds || g < 0) return 1;
  return g_split[kind][g].load(std::memory_order_relaxed);
}

/* ---------------- plain GEMM block shape ---------------- */
static std::atomic<int> g_gemm_warps[2][6] = {{{kDefaultGemmWarps}, {kDefaultGemmWarps}, {kDefaultGemmWarps},
                                               {kDefaultGemmWarps}, {kDefaultGemmWarps}, {kDefaultGemmWarps}},
                                              {{kDefaultGemmWarps}, {kDefaultGemmWarps}, {kDefaultGemmWarps},
                                               {kDefaultGemmWarps}, {kDefaultGemmWarps}, {kDefaultGemmWarps}}};

int gemm_warps(int cplx, int prec) {
  const int g = prec_group(prec);
  if (g < 0) return kDefaultGemmWarps;
  return g_gemm_warps[cplx ? 1 : 0][g].load(std::memory_order_relaxed);
}

} /* namespace mpb */

extern "C" int mpb_set_split(int kind, int prec, int lanes) {
  using namespace mpb;
  if (kind < 0 || kind >= kSplitKinds) return MPB_ERR_ARG;
  if (prec_group(prec) < 0) return MPB_ERR_PREC;
  if (!split_supported(kind, prec, lanes)) return MPB_ERR_ARG;
  std::call_once(g_split_once, split_defaults);
  g_split[kind][prec_group(prec)].store(lanes, std::memory_order_relaxed);
  return MPB_OK;
}

extern "C" int mpb_get_split(int kind, int prec, int *lanes) {
  using namespace mpb;
  if (!lanes) return MPB_ERR_NULL;
  if (kind < 0 || kind >= kSplitKinds) return MPB_ERR_ARG;
  if (prec_group(prec) < 0) return MPB_ERR_PREC;
  *lanes = split_lanes(kind, prec);
  return MPB_OK;
}

extern "C" int mpb_set_gemm_warps(int cplx, int prec, int warps) {
  using namespace mpb;
  if (prec_group(prec) < 0) return MPB_ERR_PREC;
  if (warps != 4 && warps != 8 && warps != 16) return MPB_ERR_ARG;
  g_gemm_warps[cplx ? 1 : 0][prec_group(prec)].store(warps, std::memory_order_relaxed);
  return MPB_OK;
}

extern "C" int mpb_get_gemm_warps(int cplx, int prec, int *warps) {
  using namespace mpb;
  if (!warps) return MPB_ERR_NULL;
  if (prec_group(prec) < 0) return MPB_ERR_PREC;
  *warps = gemm_warps(cplx, prec);
  return MPB_OK;
}

extern "C" void mpb_profile_enable(int on) {
  using namespace mpb;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  for (int p = 0; p < kPhases; ++p) {
    g_iv[p].clear();
    g_open[p] = nullptr;
  }
  g_pool_used = 0;
  g_profile.store(on ? 1 : 0);
}

extern "C" void mpb_profile_phases(unsigned mask) {
  using namespace mpb;
  g_profile_mask.store(mask);
}

extern "C" float mpb_profile_phase_ms(int phase) {
  using namespace mpb;
  if (phase < 0 || phase >= kPhases) return -1.0f;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (g_iv[phase].empty()) return -1.0f;
  double total = 0.0;
  for (auto &iv : g_iv[phase]) {
    float ms = 0.0f;
    if (cudaEventSynchronize(iv.second) != cudaSuccess || cudaEventElapsedTime(&ms, iv.first, iv.second) != cudaSuccess) {
      cudaGetLastError(); /* a failed query is this call's answer, not a later launch's error */
      return -1.0f;
    }
    total += ms;
  }
  return (float)total;
}

extern "C" int mpb_profile_phase_count(int phase) {
  using namespace mpb;
  if (phase < 0 || phase >= kPhases) return 0;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  return (int)g_iv[phase].size();
}

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
