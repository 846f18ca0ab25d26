/* batch.cu -- thousands of independent GEMV problems y_out = A.x + y of uneven
 * sizes and mixed precisions in one launch sequence.
 *
 * Every problem keeps the per-operation-rounded, sequential-k order of
 * mpb_gemv_r (acc = +0; acc = round(acc + round(A[i,k] x[k])); y_out[i] =
 * round(acc + y[i])), so each result is bit-exact with MPFR at its own
 * precision.
 *
 * plan (host, once): validate every descriptor, group the problems by
 * precision, order each group by decreasing cost (n per row), split them
 * into 32-row units (one warp each) and upload the descriptors, the problem
 * order and each group's unit prefix sums into the caller's workspace.
 * run (device, any number of times): reset the queue counters and launch one
 * persistent kernel per precision present, largest precision first, each on
 * the whole GPU.  Warps claim units from the group's atomic queue, longest
 * problems first, so the uneven batch balances itself.  The groups run one
 * after the other rather than side by side: a PB=2048 block needs a whole
 * SM's register file, so concurrent groups fragment the SMs and the largest
 * group ends up on a fraction of the GPU (measured 2x slower than serial).
 * run allocates nothing and never synchronises the host, so the caller can
 * capture it into a CUDA graph.  autotune times each group with every
 * candidate (block size, blocks per SM) on the planned batch and keeps the
 * fastest; set_tuning installs a cached choice.
 */
#include <algorithm>
#include <mutex>
#include <new>
#include <vector>

#include "common.cuh"
#include "coop_rows.cuh"

namespace mpb {
namespace batch {

constexpr int kGroups = 6; /* 64, 128, 256, 512, 1024, 2048 */
inline int group_of(int prec) {
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

struct DevProb { /* device copy of one problem */
  const uint8_t *A, *x, *y;
  uint8_t *yo;
  int m, n;
  long long lda;
};

struct Tuning {
  int block;        /* threads per block (multiple of 32) */
  int blocks_per_sm; /* persistent grid: SMs x this (capped by occupancy) */
  int lanes;        /* lanes per row: 1, or a warp-cooperative group (coop_rows.cuh) */
};

/* launch shapes tried by the autotuner, each with every split the precision offers */
static const Tuning kCandidates[] = {{64, 2, 1}, {64, 4, 1}, {128, 1, 1}, {128, 2, 1},
                                     {128, 4, 1}, {256, 1, 1}, {256, 2, 1}};
static const Tuning kCoopCandidates[] = {{64, 0, 1}, {128, 0, 1}, {128, 4, 1}, {256, 0, 1}, {256, 2, 1}};

template <int N>
__global__ void __launch_bounds__(256) k_batch_gemv(const DevProb *probs, const int *order, const long long *prefix,
                                                    int nprob, long long nunits, unsigned long long *counter) {
  const int lane = threadIdx.x & 31;
  while (true) {
    long long u = 0;
    if (lane == 0) u = (long long)atomicAdd(counter, 1ull);
    u = __shfl_sync(0xffffffffu, u, 0);
    if (u >= nunits) break;
    /* problem owning unit u: last p with prefix[p] <= u */
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (prefix[mid] <= u)
        lo = mid;
      else
        hi = mid - 1;
    }
    const DevProb pr = probs[order[lo]];
    const long long blk = u - prefix[lo];
    const int i = (int)(blk * 32) + lane;
    const int ir = i < pr.m ? i : pr.m - 1; /* padding lanes recompute the last row */
    fval<N> acc, yv;
    set_zero(acc);
    const uint8_t *arow = pr.A;
    for (int k = 0; k < pr.n; ++k) {
      fval<N> a, xv, t;
      load_elem<N>(a, arow, (size_t)ir * pr.lda + k);
      load_elem<N>(xv, pr.x, k);
      mul<N>(t, a, xv);
      add<N, true>(acc, acc, t);
    }
    load_elem<N>(yv, pr.y, ir);
    add<N, true>(acc, acc, yv);
    if (i < pr.m) store_elem<N>(pr.yo, i, acc);
  }
}

/* the same with G lanes per row.  A 32-row unit is split into G work items
 * of 32/G rows (nunits counts the items: G per unit), each taken by one warp:
 * the rows of a long problem then run on G times as many warps at once, and
 * the batch's critical path -- the longest row's sequential k loop -- is the
 * cooperative row's, a fraction of one thread's (items past a problem's last
 * row return at once) */
template <int L, int G>
__global__ void __launch_bounds__(256) k_batch_gemv_coop(const DevProb *probs, const int *order,
                                                         const long long *prefix, int nprob, long long nunits,
                                                         unsigned long long *counter) {
  constexpr int N = G * L, RPW = 32 / G, SMW = coop_row_smem<N>::words;
  extern __shared__ uint32_t sm_dyn[];
  const int lane = threadIdx.x & 31;
  const uint32_t warp = threadIdx.x >> 5, gw = (uint32_t)lane / G;
  uint32_t *sm = sm_dyn + (warp * RPW + gw) * SMW;
  while (true) {
    long long u = 0;
    if (lane == 0) u = (long long)atomicAdd(counter, 1ull);
    u = __shfl_sync(0xffffffffu, u, 0);
    if (u >= nunits) break;
    const long long unit = u / G;
    const int pass = (int)(u % G);
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (prefix[mid] <= unit)
        lo = mid;
      else
        hi = mid - 1;
    }
    const DevProb pr = probs[order[lo]];
    const long long blk = unit - prefix[lo];
    {
      const int r0 = (int)(blk * 32) + pass * RPW;
      if (r0 >= pr.m) continue; /* warp-uniform: an item past the last row */
      const int i = r0 + (int)gw;
      const int ir = i < pr.m ? i : pr.m - 1;
      coop::cv<L> acc;
      coop_gemv_row<L, G>(acc, pr.A, (size_t)ir * pr.lda, (size_t)pr.n, pr.x, pr.y, (size_t)ir, sm);
      if (i < pr.m) coop::store<L, G>(pr.yo, (size_t)i, acc);
    }
  }
}
template <int N>
constexpr size_t coop_smem_bytes(int block, int G) {
  return (size_t)(block / 32) * (size_t)(32 / G) * (size_t)coop_row_smem<N>::words * 4u;
}

using KernelFn = void (*)(const DevProb *, const int *, const long long *, int, long long, unsigned long long *);
/* the kernel of group g at `lanes` lanes per row, and its dynamic shared memory per block */
static KernelFn coop_kernel_of(int g, int lanes, int block, size_t *smem) {
  if (g == 4) {
    *smem = coop_smem_bytes<32>(block, lanes);
    return lanes == 4 ? k_batch_gemv_coop<8, 4> : k_batch_gemv_coop<4, 8>;
  }
  *smem = coop_smem_bytes<64>(block, lanes);
  return lanes == 8 ? k_batch_gemv_coop<8, 8> : k_batch_gemv_coop<4, 16>;
}
static bool lanes_ok(int g, int lanes) {
  if (lanes == 1) return true;
  if (g == 4) return lanes == 4 || lanes == 8;
  if (g == 5) return lanes == 8 || lanes == 16;
  return false;
}
static KernelFn kernel_of(int g) {
  switch (g) {
    case 0: return k_batch_gemv<2>;
    case 1: return k_batch_gemv<4>;
    case 2: return k_batch_gemv<8>;
    case 3: return k_batch_gemv<16>;
    case 4: return k_batch_gemv<32>;
    default: return k_batch_gemv<64>;
  }
}

} /* namespace batch */
} /* namespace mpb */

using namespace mpb;
using namespace mpb::batch;

/* opaque host-side plan */
struct mpb_batch_plan {
  int device;
  int count;
  uint8_t *ws;
  DevProb *probs;   /* device */
  int *order;       /* device: problem indices, grouped, longest first */
  long long *prefix; /* device: per-group unit prefix sums */
  int *counters;    /* device: one queue counter per group */
  int gstart[kGroups], gcount[kGroups];
  long long gunits[kGroups];
  Tuning tune[kGroups];
  float tuned_ms[kGroups]; /* autotune: best solo time of the group, -1 before */
};

static size_t up256b(size_t x) { return (x + 255) & ~(size_t)255; }

static void layout_ws(int count, size_t *o_probs, size_t *o_order, size_t *o_prefix, size_t *o_cnt, size_t *total) {
  size_t o = 0;
  *o_probs = o;
  o = up256b(o + sizeof(DevProb) * (size_t)count);
  *o_order = o;
  o = up256b(o + sizeof(int) * (size_t)count);
  *o_prefix = o;
  o = up256b(o + sizeof(long long) * (size_t)(count + kGroups));
  *o_cnt = o;
  o = up256b(o + 64 * kGroups);
  *total = o;
}

extern "C" size_t mpb_batch_gemv_workspace(int count) {
  if (count <= 0 || count > (1 << 24)) return 0;
  size_t a, b, c, d, t;
  layout_ws(count, &a, &b, &c, &d, &t);
  return t;
}

static int check_prob(const mpb_gemv_problem &p) {
  const int g = group_of(p.prec);
  if (g < 0) return MPB_ERR_PREC;
  if (p.m < 0 || p.n < 0 || p.m > (1 << 24) || p.n > (1 << 24)) return MPB_ERR_SIZE;
  if (p.m == 0) return MPB_OK;
  if (p.n > 0 && (p.lda % 32 != 0 || p.lda < (size_t)p.n)) return MPB_ERR_LD;
  if (!p.y || !p.y_out || (p.n > 0 && (!p.A || !p.x))) return MPB_ERR_NULL;
  if (!aligned16(p.y) || !aligned16(p.y_out) || (p.n > 0 && (!aligned16(p.A) || !aligned16(p.x))))
    return MPB_ERR_ALIGN;
  return MPB_OK;
}

extern "C" int mpb_batch_gemv_plan(int count, const mpb_gemv_problem *problems, void *workspace, size_t ws_bytes,
                                   mpb_batch_plan **plan_out) {
  if (!plan_out) return MPB_ERR_NULL;
  *plan_out = nullptr;
  if (count <= 0 || count > (1 << 24)) return MPB_ERR_SIZE;
  if (!problems) return MPB_ERR_NULL;
  size_t o_probs, o_order, o_prefix, o_cnt, total;
  layout_ws(count, &o_probs, &o_order, &o_prefix, &o_cnt, &total);
  if (!workspace || ws_bytes < total) return MPB_ERR_WORKSPACE;
  if (((uintptr_t)workspace & 255u) != 0) return MPB_ERR_ALIGN;
  for (int i = 0; i < count; ++i) {
    const int rc = check_prob(problems[i]);
    if (rc != MPB_OK) return rc;
  }
  /* group by precision, longest (per-row cost) first */
  std::vector<int> idx(count);
  for (int i = 0; i < count; ++i) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
    const int ga = group_of(problems[a].prec), gb = group_of(problems[b].prec);
    if (ga != gb) return ga < gb;
    return problems[a].n > problems[b].n;
  });
  mpb_batch_plan *pl = new (std::nothrow) mpb_batch_plan();
  if (!pl) return MPB_ERR_ARG;
  if (cudaGetDevice(&pl->device) != cudaSuccess) {
    delete pl;
    return MPB_ERR_CUDA;
  }
  pl->count = count;
  pl->ws = (uint8_t *)workspace;
  pl->probs = (DevProb *)(pl->ws + o_probs);
  pl->order = (int *)(pl->ws + o_order);
  pl->prefix = (long long *)(pl->ws + o_prefix);
  pl->counters = (int *)(pl->ws + o_cnt);
  std::vector<DevProb> hp(count);
  std::vector<long long> pre(count + kGroups, 0);
  for (int g = 0; g < kGroups; ++g) {
    pl->gstart[g] = 0;
    pl->gcount[g] = 0;
    pl->gunits[g] = 0;
    pl->tune[g] = Tuning{128, 0, 1}; /* 0: full occupancy */
    pl->tuned_ms[g] = -1.0f;
  }
  for (int g = 4; g < kGroups; ++g) pl->tune[g].lanes = split_lanes(MPB_SPLIT_GEMV_R, 64 << g);
  for (int i = 0; i < count; ++i) {
    const mpb_gemv_problem &p = problems[i];
    hp[i] = DevProb{(const uint8_t *)p.A, (const uint8_t *)p.x, (const uint8_t *)p.y, (uint8_t *)p.y_out,
                    p.m, p.n, (long long)p.lda};
  }
  /* per group: order slice and unit prefix sums (prefix array holds, for each
   * group, its problems' prefixes contiguously at [gstart, gstart+gcount)) */
  int pos = 0;
  for (int g = 0; g < kGroups; ++g) {
    pl->gstart[g] = pos;
    long long units = 0;
    while (pos < count && group_of(problems[idx[pos]].prec) == g) {
      const mpb_gemv_problem &p = problems[idx[pos]];
      pre[pos] = units;
      units += (p.m + 31) / 32;
      ++pos;
    }
    pl->gcount[g] = pos - pl->gstart[g];
    pl->gunits[g] = units;
  }
  bool ok = cudaMemcpy(pl->probs, hp.data(), sizeof(DevProb) * count, cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(pl->order, idx.data(), sizeof(int) * count, cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(pl->prefix, pre.data(), sizeof(long long) * count, cudaMemcpyHostToDevice) == cudaSuccess;
  if (!ok) {
    mpb_batch_gemv_destroy(pl);
    return MPB_ERR_CUDA;
  }
  *plan_out = pl;
  return MPB_OK;
}

static int launch_group(mpb_batch_plan *pl, int g, cudaStream_t st) {
  if (pl->gcount[g] == 0 || pl->gunits[g] == 0) return MPB_OK;
  const Tuning t = pl->tune[g];
  size_t smem = 0;
  KernelFn fn = t.lanes > 1 ? coop_kernel_of(g, t.lanes, t.block, &smem) : kernel_of(g);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, t.block, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const int bps = t.blocks_per_sm > 0 ? std::min(t.blocks_per_sm, per_sm) : per_sm;
  long long grid = (long long)sm_count() * bps;
  const long long items = pl->gunits[g] * (t.lanes > 1 ? t.lanes : 1); /* one warp per item */
  const long long max_grid = (items * 32 + t.block - 1) / t.block;
  grid = std::min(grid, std::max(1LL, max_grid));
  fn<<<(int)grid, t.block, smem, st>>>(pl->probs, pl->order + pl->gstart[g], pl->prefix + pl->gstart[g],
                                       pl->gcount[g], items,
                                       (unsigned long long *)((uint8_t *)pl->counters + 64 * g));
  return launch_status();
}

extern "C" int mpb_batch_gemv_run(mpb_batch_plan *pl, void *stream) {
  if (!pl) return MPB_ERR_NULL;
  cudaStream_t st = as_stream(stream);
  if (cudaMemsetAsync(pl->counters, 0, 64 * kGroups, st) != cudaSuccess) return MPB_ERR_CUDA;
  for (int g = kGroups - 1; g >= 0; --g) {
    const int rc = launch_group(pl, g, st);
    if (rc != MPB_OK) return rc;
  }
  return MPB_OK;
}

extern "C" int mpb_batch_gemv_autotune(mpb_batch_plan *pl, void *stream) {
  if (!pl) return MPB_ERR_NULL;
  cudaStream_t st = as_stream(stream);
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return MPB_ERR_CUDA;
  int rc = MPB_OK;
  for (int g = 0; g < kGroups && rc == MPB_OK; ++g) {
    if (pl->gcount[g] == 0) continue;
    float best = 1e30f;
    Tuning bestt = pl->tune[g];
    std::vector<Tuning> cands(std::begin(kCandidates), std::end(kCandidates));
    for (int lanes : {4, 8, 16})
      if (lanes_ok(g, lanes))
        for (Tuning c : kCoopCandidates) {
          c.lanes = lanes;
          cands.push_back(c);
        }
    for (const Tuning &c : cands) {
      pl->tune[g] = c;
      float ms_sum = 0.0f;
      for (int rep = 0; rep < 3 && rc == MPB_OK; ++rep) {
        if (cudaMemsetAsync((uint8_t *)pl->counters + 64 * g, 0, 64, st) != cudaSuccess) rc = MPB_ERR_CUDA;
        cudaEventRecord(e0, st);
        const int r = launch_group(pl, g, st);
        cudaEventRecord(e1, st);
        if (r != MPB_OK || cudaEventSynchronize(e1) != cudaSuccess) rc = MPB_ERR_CUDA;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) ms_sum += ms; /* first run warms up */
      }
      if (rc == MPB_OK && ms_sum < best) {
        best = ms_sum;
        bestt = c;
      }
    }
    pl->tune[g] = bestt;
    pl->tuned_ms[g] = best / 2.0f;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

extern "C" int mpb_batch_gemv_get_tuning(const mpb_batch_plan *pl, int prec, int *block, int *blocks_per_sm) {
  if (!pl || !block || !blocks_per_sm) return MPB_ERR_NULL;
  const int g = group_of(prec);
  if (g < 0) return MPB_ERR_PREC;
  *block = pl->tune[g].block;
  *blocks_per_sm = pl->tune[g].blocks_per_sm;
  return MPB_OK;
}

extern "C" int mpb_batch_gemv_tuned_ms(const mpb_batch_plan *pl, int prec, float *ms) {
  if (!pl || !ms) return MPB_ERR_NULL;
  const int g = group_of(prec);
  if (g < 0) return MPB_ERR_PREC;
  *ms = pl->gcount[g] > 0 ? pl->tuned_ms[g] : 0.0f;
  return MPB_OK;
}

extern "C" int mpb_batch_gemv_set_tuning(mpb_batch_plan *pl, int prec, int block, int blocks_per_sm) {
  if (!pl) return MPB_ERR_NULL;
  const int g = group_of(prec);
  if (g < 0) return MPB_ERR_PREC;
  if (block < 32 || block > 256 || block % 32 != 0 || blocks_per_sm < 0 || blocks_per_sm > 64) return MPB_ERR_ARG;
  pl->tune[g].block = block;
  pl->tune[g].blocks_per_sm = blocks_per_sm;
  return MPB_OK;
}

extern "C" int mpb_batch_gemv_get_split(const mpb_batch_plan *pl, int prec, int *lanes) {
  if (!pl || !lanes) return MPB_ERR_NULL;
  const int g = group_of(prec);
  if (g < 0) return MPB_ERR_PREC;
  *lanes = pl->tune[g].lanes;
  return MPB_OK;
}

extern "C" int mpb_batch_gemv_set_split(mpb_batch_plan *pl, int prec, int lanes) {
  if (!pl) return MPB_ERR_NULL;
  const int g = group_of(prec);
  if (g < 0) return MPB_ERR_PREC;
  if (!lanes_ok(g, lanes)) return MPB_ERR_ARG;
  pl->tune[g].lanes = lanes;
  return MPB_OK;
}

extern "C" void mpb_batch_gemv_destroy(mpb_batch_plan *pl) {
  if (!pl) return;
  delete pl;
}
