/* mpb/layout.cuh -- the engine's HBM layout ("SoL tiles") and its device
 * load/store helpers.
 *
 * A real vector of n elements at precision PB = 32*N is a sequence of
 * ceil(n/32) tiles; tile t holds elements 32t .. 32t+31:
 *
 *   [G vector groups][32 elements][V limbs]   limbs  (V = min(4, N), G = N/V)
 *   [32 elements] uint32                      heads
 *
 * so a tile is 32*(4N+4) = 128*(N+1) bytes (1152 B at PB=256) and starts on a
 * 128-byte boundary.  A warp that handles the 32 elements of one tile reads
 * each vector group as one 512-byte contiguous span of 16-byte loads (V=4),
 * and the heads as one 128-byte span: every access is coalesced and 128-bit
 * vectorised.  Whole tiles are contiguous, so a tile is also a single bulk
 * copy into shared memory.
 *
 * Limb k of an element is bits [32k, 32k+32) of its left-justified
 * significand M (mpb/core.cuh).  The head word is (e << 1) | sign, with
 * 0x80000000 for zero (whose limbs are all zero).  This 32-bit head covers
 * MPFR's default exponent range [1-2^30, 2^30-1].
 *
 * A complex vector is a sequence of complex tiles: [re tile][im tile].
 * A matrix is row-major with a leading dimension ld (elements, a multiple of
 * 32): element (i, j) is vector element i*ld + j, so every row is whole tiles.
 */
#ifndef MPB_LAYOUT_CUH
#define MPB_LAYOUT_CUH

#include <stddef.h>
#include <stdint.h>

#include "core.cuh"

namespace mpb {

template <int N>
struct sol {
  static constexpr int V = (N >= 4) ? 4 : N;
  static constexpr int G = N / V;
  static constexpr size_t kTileBytes = 128u * (size_t)(N + 1);
  static constexpr size_t kHeadOff = 128u * (size_t)N;
};

MPB_HDI size_t tile_bytes_for(int nlimbs) { return 128u * (size_t)(nlimbs + 1); }
MPB_HDI size_t tiles_for(size_t n) { return (n + 31u) / 32u; }

#if defined(__CUDACC__)

template <int V>
struct vec_t;
template <>
struct vec_t<4> {
  typedef uint4 type;
};
template <>
struct vec_t<2> {
  typedef uint2 type;
};
template <>
struct vec_t<1> {
  typedef uint32_t type;
};

template <int V>
__device__ __forceinline__ void put_vec(uint32_t *m, const typename vec_t<V>::type &v);
template <>
__device__ __forceinline__ void put_vec<4>(uint32_t *m, const uint4 &v) {
  m[0] = v.x;
  m[1] = v.y;
  m[2] = v.z;
  m[3] = v.w;
}
template <>
__device__ __forceinline__ void put_vec<2>(uint32_t *m, const uint2 &v) {
  m[0] = v.x;
  m[1] = v.y;
}
template <>
__device__ __forceinline__ void put_vec<1>(uint32_t *m, const uint32_t &v) {
  m[0] = v;
}
template <int V>
__device__ __forceinline__ typename vec_t<V>::type get_vec(const uint32_t *m);
template <>
__device__ __forceinline__ uint4 get_vec<4>(const uint32_t *m) {
  return make_uint4(m[0], m[1], m[2], m[3]);
}
template <>
__device__ __forceinline__ uint2 get_vec<2>(const uint32_t *m) {
  return make_uint2(m[0], m[1]);
}
template <>
__device__ __forceinline__ uint32_t get_vec<1>(const uint32_t *m) {
  return m[0];
}

/* Load modes: kCached (plain global load, reused data), kStream (read-once
 * streaming data: evict-first, keeps L2 for reused operands). */
enum { kCached = 0, kStream = 1 };

template <int V, int MODE>
__device__ __forceinline__ typename vec_t<V>::type ld_vec(const void *p) {
  typedef typename vec_t<V>::type T;
  if (MODE == kStream) return __ldcs((const T *)p);
  return __ldg((const T *)p);
}
template <int V, int MODE>
__device__ __forceinline__ void st_vec(void *p, const typename vec_t<V>::type &v) {
  typedef typename vec_t<V>::type T;
  if (MODE == kStream)
    __stcs((T *)p, v);
  else
    *(T *)p = v;
}

/* element i of the tiled vector at base (tile-local addressing) */
template <int N, int MODE = kCached>
__device__ __forceinline__ void load_elem(fval<N> &x, const uint8_t *base, size_t i) {
  typedef sol<N> L;
  const uint8_t *t = base + (i >> 5) * L::kTileBytes;
  const uint32_t lane = (uint32_t)(i & 31u);
#pragma unroll
  for (int g = 0; g < L::G; ++g)
    put_vec<L::V>(x.m + g * L::V, ld_vec<L::V, MODE>(t + (size_t)g * 128u * L::V + lane * 4u * L::V));
  const uint32_t h = (MODE == kStream) ? __ldcs((const uint32_t *)(t + L::kHeadOff) + lane)
                                       : __ldg((const uint32_t *)(t + L::kHeadOff) + lane);
  /* canonical zero: a zero head forces zero limbs */
  const uint32_t keep = (h == kHeadZero) ? 0u : 0xffffffffu;
#pragma unroll
  for (int k = 0; k < N; ++k) x.m[k] &= keep;
  x.e = head_exp(h);
  x.s = head_sign(h);
}

template <int N, int MODE = kCached>
__device__ __forceinline__ void store_elem(uint8_t *base, size_t i, const fval<N> &x) {
  typedef sol<N> L;
  uint8_t *t = base + (i >> 5) * L::kTileBytes;
  const uint32_t lane = (uint32_t)(i & 31u);
#pragma unroll
  for (int g = 0; g < L::G; ++g)
    st_vec<L::V, MODE>(t + (size_t)g * 128u * L::V + lane * 4u * L::V, get_vec<L::V>(x.m + g * L::V));
  const uint32_t h = pack_head(x.e, x.s);
  if (MODE == kStream)
    __stcs((uint32_t *)(t + L::kHeadOff) + lane, h);
  else
    ((uint32_t *)(t + L::kHeadOff))[lane] = h;
}

/* complex element i: re in the first tile of the complex tile, im in the second */
template <int N, int MODE = kCached>
__device__ __forceinline__ void load_celem(fval<N> &re, fval<N> &im, const uint8_t *base, size_t i) {
  const uint8_t *ct = base + (i >> 5) * 2u * sol<N>::kTileBytes;
  load_elem<N, MODE>(re, ct, i & 31u);
  load_elem<N, MODE>(im, ct + sol<N>::kTileBytes, i & 31u);
}
template <int N, int MODE = kCached>
__device__ __forceinline__ void store_celem(uint8_t *base, size_t i, const fval<N> &re,
                                            const fval<N> &im) {
  uint8_t *ct = base + (i >> 5) * 2u * sol<N>::kTileBytes;
  store_elem<N, MODE>(ct, i & 31u, re);
  store_elem<N, MODE>(ct + sol<N>::kTileBytes, i & 31u, im);
}

#endif /* __CUDACC__ */

} /* namespace mpb */

#endif /* MPB_LAYOUT_CUH */
