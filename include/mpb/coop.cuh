/* mpb/coop.cuh -- warp-cooperative fixed-precision arithmetic for wide operands
 * (sm_100a, device only).
 *
 * Above 512 bits one thread cannot hold an operand, a product window and an
 * accumulator in registers: the thread-per-element kernels then run at the
 * 255-register ceiling with a warp or two per scheduler, or spill.  Here a
 * value of N = G*L 32-bit limbs is spread over an aligned group of G lanes
 * (G a power of two, 2..32): lane t of the group holds limbs [tL, tL + L),
 * every lane of the group the exponent and the sign, with the value
 * convention of mpb::fval (value = (-1)^s M 2^(e - 32N), M left-justified;
 * zero: e == kExpZero and zero limbs).  A warp holds 32/G values.
 *
 *  - Products (mul_u) multiply a group value by a UNIFORM significand (the
 *    AXPY scalar, GEMV's x[k], the A[i,k] a GEMM row shares): row by row,
 *    limb j of the uniform operand times every lane's L limbs, added into a
 *    window of N words spread like the value; after each row the window
 *    moves down one word (one __shfl_down per row), the word that leaves it
 *    at lane 0 is a finished low word of the product, and the word a lane's
 *    row pushes past its top is kept in a per-lane overflow carried into
 *    the lane above at the next move.  With L limbs a lane does 2L
 *    multiply-adds per row against two shuffles, so the IMAD pipe, not the
 *    shuffle unit, bounds the product.
 *  - Carries across lanes (sums, increments, negation) are resolved at once
 *    with a carry-lookahead on ballots: each lane adds its words with carry-in
 *    0 and reports "generates a carry" / "all ones" (propagates); the carries
 *    into all lanes are then the bits of (g|p) + g + cin (carry_into).
 *  - Aligned sums with one rounding (add_round_sm) take their operands from
 *    this group's shared-memory buffers, so the alignment shift by any
 *    number of words is an indexed shared load (no shift networks); the
 *    normalisation reads the result back at the leading-word offset found by
 *    a ballot.  The rounding rule is the core's (round to nearest even, the
 *    sticky-borrow rule for opposite signs).
 *
 * Every function here must be called by all 32 lanes of the warp (the
 * shuffles and ballots use the full mask); group-dependent decisions are data,
 * never branches around a shuffle.  Blocks are whole warps (blockDim.x a
 * multiple of 32).
 */
#ifndef MPB_COOP_CUH
#define MPB_COOP_CUH

#include "layout.cuh"

#if defined(__CUDACC__)

namespace mpb {
namespace coop {

constexpr uint32_t kFull = 0xffffffffu;

template <int G>
struct grp {
  static_assert(G >= 2 && G <= 32 && (G & (G - 1)) == 0, "group size: a power of two from 2 to 32");
  __device__ __forceinline__ static uint32_t t() { return threadIdx.x & (uint32_t)(G - 1); }
  __device__ __forceinline__ static uint32_t base() { return threadIdx.x & 31u & ~(uint32_t)(G - 1); }
  /* the group's votes, bit t = lane t of the group */
  __device__ __forceinline__ static uint32_t ballot(bool p) {
    const uint32_t b = __ballot_sync(kFull, p) >> base();
    return G == 32 ? b : (b & ((1u << G) - 1u));
  }
  __device__ __forceinline__ static uint32_t bcast(uint32_t v, int src) { return __shfl_sync(kFull, v, src, G); }
};

/* this lane's part of a group value */
template <int L>
struct cv {
  uint32_t m[L];
  int32_t e;
  uint32_t s;
};
template <int L>
__device__ __forceinline__ void set_zero(cv<L> &x) {
#pragma unroll
  for (int k = 0; k < L; ++k) x.m[k] = 0u;
  x.e = kExpZero;
  x.s = 0u;
}

/* carry into this lane of a chain through the group's lanes, lane 0 taking
 * cin: gen = this lane's words overflow on their own, prop = they are all
 * ones (an incoming carry passes through); never both.  cout: the carry out
 * of the top lane. */
template <int G>
__device__ __forceinline__ uint32_t carry_into(bool gen, bool prop, uint32_t cin, uint32_t &cout) {
  const uint64_t gm = grp<G>::ballot(gen), pm = grp<G>::ballot(prop);
  const uint64_t a = gm | pm, sum = a + gm + (uint64_t)cin;
  cout = (uint32_t)(sum >> G) & 1u;
  return (uint32_t)((sum ^ a ^ gm) >> grp<G>::t()) & 1u;
}

/* d = x + y over L words with carry-in 0; gen = carry out, prop = d is all ones */
template <int L>
__device__ __forceinline__ void add_local(uint32_t (&d)[L], const uint32_t (&x)[L], const uint32_t (&y)[L],
                                          bool &gen, bool &prop) {
  uint32_t cf = 0;
  d[0] = add_cc(x[0], y[0], cf);
#pragma unroll
  for (int k = 1; k < L; ++k) d[k] = addc_cc(x[k], y[k], cf);
  gen = addc(0u, 0u, cf) != 0u;
  uint32_t all = d[0];
#pragma unroll
  for (int k = 1; k < L; ++k) all &= d[k];
  prop = all == 0xffffffffu;
}
/* d += c (c in {0, 1}) over L words */
template <int L>
__device__ __forceinline__ void inc_local(uint32_t (&d)[L], uint32_t c) {
  uint32_t cf = 0;
  d[0] = add_cc(d[0], c, cf);
#pragma unroll
  for (int k = 1; k < L; ++k) d[k] = addc_cc(d[k], 0u, cf);
}
template <int L>
__device__ __forceinline__ bool all_ones(const uint32_t (&d)[L]) {
  uint32_t all = d[0];
#pragma unroll
  for (int k = 1; k < L; ++k) all &= d[k];
  return all == 0xffffffffu;
}

/* round the group significand m (N words) to nearest-even given the round bit
 * rb and the sticky word stk (both uniform in the group); a carry out of the
 * top gives 1000...0 and e + 1 */
template <int L, int G>
__device__ __forceinline__ void round_nearest(uint32_t (&m)[L], int32_t &e, uint32_t rb, uint32_t stk) {
  const uint32_t lsb = grp<G>::bcast(m[0], 0) & 1u;
  const uint32_t inc = rb & ((stk != 0u ? 1u : 0u) | lsb);
  uint32_t cout;
  const uint32_t cin = carry_into<G>(false, all_ones(m), inc, cout);
  inc_local(m, cin);
  if (cout) { /* every word wrapped to zero */
    if (grp<G>::t() == (uint32_t)(G - 1)) m[L - 1] = 0x80000000u;
    e += 1;
  }
}

/* ---- the tiled layout: this lane's L limbs of element i ---- */
template <int L, int G, int MODE = kCached>
__device__ __forceinline__ void load(cv<L> &x, const uint8_t *base, size_t i) {
  constexpr int N = G * L;
  static_assert(L % 4 == 0 && N >= 4, "four limbs per 128-bit load");
  typedef sol<N> S;
  const uint8_t *tile = base + (i >> 5) * S::kTileBytes;
  const uint32_t slot = (uint32_t)(i & 31u), t = grp<G>::t();
#pragma unroll
  for (int v = 0; v < L / 4; ++v) {
    const uint4 w = ld_vec<4, MODE>(tile + (size_t)(t * (L / 4) + v) * 512u + slot * 16u);
    x.m[4 * v] = w.x;
    x.m[4 * v + 1] = w.y;
    x.m[4 * v + 2] = w.z;
    x.m[4 * v + 3] = w.w;
  }
  const uint32_t h = (MODE == kStream) ? __ldcs((const uint32_t *)(tile + S::kHeadOff) + slot)
                                       : __ldg((const uint32_t *)(tile + S::kHeadOff) + slot);
  const uint32_t keep = (h == kHeadZero) ? 0u : 0xffffffffu;
#pragma unroll
  for (int k = 0; k < L; ++k) x.m[k] &= keep;
  x.e = head_exp(h);
  x.s = head_sign(h);
}
template <int L, int G, int MODE = kCached>
__device__ __forceinline__ void store(uint8_t *base, size_t i, const cv<L> &x) {
  constexpr int N = G * L;
  typedef sol<N> S;
  uint8_t *tile = base + (i >> 5) * S::kTileBytes;
  const uint32_t slot = (uint32_t)(i & 31u), t = grp<G>::t();
  const bool z = x.e == kExpZero;
#pragma unroll
  for (int v = 0; v < L / 4; ++v) {
    uint4 w;
    w.x = z ? 0u : x.m[4 * v];
    w.y = z ? 0u : x.m[4 * v + 1];
    w.z = z ? 0u : x.m[4 * v + 2];
    w.w = z ? 0u : x.m[4 * v + 3];
    st_vec<4, MODE>(tile + (size_t)(t * (L / 4) + v) * 512u + slot * 16u, w);
  }
  if (t == 0) {
    const uint32_t h = z ? kHeadZero : pack_head(x.e, x.s);
    if (MODE == kStream)
      __stcs((uint32_t *)(tile + S::kHeadOff) + slot, h);
    else
      ((uint32_t *)(tile + S::kHeadOff))[slot] = h;
  }
}

/* a uniform operand: element slot of the tile at tile (every lane of the warp
 * reads the same addresses, one broadcast transaction per load) */
struct uref {
  const uint8_t *tile;
  uint32_t slot;
};
template <int N>
__device__ __forceinline__ uref uniform_ref(const uint8_t *base, size_t i) {
  return uref{base + (i >> 5) * sol<N>::kTileBytes, (uint32_t)(i & 31u)};
}
/* head of a uniform operand: exponent and sign, kExpZero for zero */
template <int N>
__device__ __forceinline__ void uniform_head(const uref &u, int32_t &e, uint32_t &s) {
  const uint32_t h = __ldg((const uint32_t *)(u.tile + sol<N>::kHeadOff) + u.slot);
  e = head_exp(h);
  s = head_sign(h);
}

/* ---- the exact product of a group value and a uniform significand ---- */
/* x (this lane's L limbs) times the N limbs of u: the upper N words of the 2N
 * word product land in hi (lane t: words N + tL + k).  The lower N words are
 * stored to lo[0..N) in shared memory by lane 0 (kStoreLow), or summarised
 * for a rounding: w1 = word N-1, w2 = word N-2, st = OR of words 0..N-3,
 * uniform in the group. */
template <int L, int G, bool kStoreLow>
__device__ __forceinline__ void mul_u(uint32_t (&hi)[L], uint32_t *lo, uint32_t &w1, uint32_t &w2, uint32_t &st,
                                      const uint32_t (&x)[L], const uref &u) {
  constexpr int N = G * L;
  static_assert(L % 4 == 0 && L >= 4, "L: a multiple of 4");
  const uint32_t t = grp<G>::t();
  uint32_t acc[L];
#pragma unroll
  for (int k = 0; k < L; ++k) acc[k] = 0u;
  uint32_t ovl = 0u, ovh = 0u, q1 = 0u, q2 = 0u, qs = 0u;
#pragma unroll 1
  for (int jb = 0; jb < N; jb += L) {
    uint32_t b[L];
#pragma unroll
    for (int v = 0; v < L / 4; ++v) {
      const uint4 w = __ldg((const uint4 *)(u.tile + (size_t)(jb / 4 + v) * 512u + u.slot * 16u));
      b[4 * v] = w.x;
      b[4 * v + 1] = w.y;
      b[4 * v + 2] = w.z;
      b[4 * v + 3] = w.w;
    }
#pragma unroll
    for (int s = 0; s < L; ++s) {
      /* logical window word k sits in acc[(k + s) % L]: the move of the window
       * after each row is a renaming */
#define MPB_W(k) acc[((k) + s) % L]
      uint32_t cf = 0;
      MPB_W(0) = madlo_cc(b[s], x[0], MPB_W(0), cf);
#pragma unroll
      for (int k = 1; k < L; ++k) MPB_W(k) = madclo_cc(b[s], x[k], MPB_W(k), cf);
      uint32_t top = addc(0u, 0u, cf);
      MPB_W(1) = madhi_cc(b[s], x[0], MPB_W(1), cf);
#pragma unroll
      for (int k = 1; k < L - 1; ++k) MPB_W(k + 1) = madchi_cc(b[s], x[k], MPB_W(k + 1), cf);
      top = madchi(b[s], x[L - 1], top, cf); /* the row's word above the lane: < 2^32 */
      ovl = add_cc(ovl, top, cf);
      ovh = addc(ovh, 0u, cf);
      const uint32_t out = MPB_W(0);
      if (kStoreLow) {
        if (t == 0) lo[jb + s] = out;
      } else {
        qs |= q2;
        q2 = q1;
        q1 = out;
      }
      uint32_t in = __shfl_down_sync(kFull, out, 1, G);
      if (t == (uint32_t)(G - 1)) in = 0u;
      /* the word from the lane above and this lane's overflow meet at the new top word */
      MPB_W(0) = add_cc(in, ovl, cf);
      ovl = addc(ovh, 0u, cf);
      ovh = 0u;
#undef MPB_W
    }
  }
  /* the overflow of lane t belongs to word 0 of lane t + 1 */
  uint32_t inl = __shfl_up_sync(kFull, ovl, 1, G);
  if (t == 0) inl = 0u;
  uint32_t add[L];
#pragma unroll
  for (int k = 0; k < L; ++k) add[k] = k == 0 ? inl : 0u;
  bool gen, prop;
  add_local(hi, acc, add, gen, prop);
  uint32_t cout;
  const uint32_t cin = carry_into<G>(gen, prop, 0u, cout);
  inc_local(hi, cin);
  if (!kStoreLow) {
    w1 = grp<G>::bcast(q1, 0);
    w2 = grp<G>::bcast(q2, 0);
    st = grp<G>::bcast(qs, 0);
  }
}

/* r = round(x * u) (RNDN), u a uniform operand with exponent ue, sign us */
template <int L, int G>
__device__ __forceinline__ void mul_round_u(cv<L> &r, const cv<L> &x, const uref &u, int32_t ue, uint32_t us) {
  uint32_t hi[L], w1, w2, st;
  const bool zero = x.e == kExpZero || ue == kExpZero;
  uint32_t xm[L];
#pragma unroll
  for (int k = 0; k < L; ++k) xm[k] = zero ? 0u : x.m[k]; /* a zero u may carry stale limbs */
  mul_u<L, G, false>(hi, nullptr, w1, w2, st, xm, u);
  const uint32_t t = grp<G>::t();
  /* the product's leading bit is its top bit or the one below: shift by sh */
  const uint32_t sh = (grp<G>::bcast(hi[L - 1], G - 1) >> 31) ^ 1u;
  uint32_t below = __shfl_up_sync(kFull, hi[L - 1], 1, G);
  if (t == 0) below = w1;
  r.m[0] = fshl(below, hi[0], sh);
#pragma unroll
  for (int k = 1; k < L; ++k) r.m[k] = fshl(hi[k - 1], hi[k], sh);
  const uint32_t low = fshl(w2, w1, sh);
  int32_t e = x.e + ue - (int32_t)sh;
  round_nearest<L, G>(r.m, e, low >> 31, (low << 1) | (w2 << sh) | st);
  r.e = e;
  r.s = x.s ^ us;
  if (zero) set_zero(r);
}

/* ---- aligned sum with one rounding, operands in shared memory ---- */
/* r = round(X + Y) at N = G*L limbs.  X and Y: exact magnitudes of NX = G*LX
 * words in this group's shared memory (little-endian), value M 2^(e - 32 NX)
 * with the window-top exponents ex, ey (zero: kExpZero and zero words), signs
 * sx, sy.  E: NX + 3 words of scratch.  The caller synchronises the warp
 * after writing X and Y; E may be reused after the call returns. */
template <int L, int G, int LX>
__device__ __forceinline__ void add_round_sm(cv<L> &r, const uint32_t *X, int32_t ex, uint32_t sx, const uint32_t *Y,
                                             int32_t ey, uint32_t sy, uint32_t *E) {
  constexpr int N = G * L, NX = G * LX, W = NX + 3;
  const int t = (int)grp<G>::t();
  const bool sw = ey > ex;
  const uint32_t *A = sw ? Y : X;
  const uint32_t *B = sw ? X : Y;
  const int32_t ea = sw ? ey : ex, eb = sw ? ex : ey;
  const uint32_t sa = sw ? sy : sx, sb = sw ? sx : sy;
  const int64_t dd = (int64_t)ea - (int64_t)eb;
  const uint32_t d = dd > (int64_t)(32 * W) ? (uint32_t)(32 * W) : (uint32_t)dd;
  const int q = (int)(d >> 5);
  const uint32_t rs = d & 31u;
  auto bw = [&](int j) -> uint32_t { return (j >= 0 && j < NX) ? B[j] : 0u; };
  /* the window: A in words [0, NX), B shifted right by d; two guard words under it */
  uint32_t a[LX], bs[LX];
  uint32_t stl = 0u;
#pragma unroll
  for (int k = 0; k < LX; ++k) {
    const int w = t * LX + k;
    a[k] = A[w];
    bs[k] = fshr(bw(w + q), bw(w + q + 1), rs);
    const uint32_t own = B[w]; /* B's bits under the guard words: sticky */
    stl |= (w < q - 2) ? own : ((w == q - 2) ? (own & ((1u << rs) - 1u)) : 0u);
  }
  const uint32_t g1 = fshr(bw(q - 1), bw(q), rs), g0 = fshr(bw(q - 2), bw(q - 1), rs);
  const uint32_t st = grp<G>::ballot(stl != 0u) != 0u ? 1u : 0u;
  const uint32_t sub = sa ^ sb, msk = 0u - sub;
  /* opposite signs: A - B - sticky in two's complement, the guard words first */
  const uint64_t gv = ((uint64_t)g1 << 32) | g0;
  const uint64_t gs = sub ? 0ull - gv - (uint64_t)st : gv;
  const uint32_t borrow = sub & ((gv != 0ull || st) ? 1u : 0u);
#pragma unroll
  for (int k = 0; k < LX; ++k) bs[k] ^= msk;
  uint32_t D[LX];
  bool gen, prop;
  add_local(D, a, bs, gen, prop);
  uint32_t cout;
  uint32_t cin = carry_into<G>(gen, prop, sub & (borrow ^ 1u), cout);
  inc_local(D, cin);
  /* a negative difference (possible only when d = 0: nothing under the
   * window) is negated exactly */
  const uint32_t neg = sub & (cout ^ 1u);
#pragma unroll
  for (int k = 0; k < LX; ++k) D[k] ^= 0u - neg;
  uint32_t c2;
  cin = carry_into<G>(false, all_ones(D), neg, c2);
  inc_local(D, cin);
  const uint32_t cs = (sub ^ 1u) & cout; /* same-sign carry out: one word above the window */
  /* E = [guard 0, guard 1, D..., carry word] */
  if (t == 0) {
    E[0] = (uint32_t)gs;
    E[1] = (uint32_t)(gs >> 32);
    E[W - 1] = cs;
  }
#pragma unroll
  for (int k = 0; k < LX; ++k) E[2 + t * LX + k] = D[k];
  __syncwarp();
  /* leading word: the highest nonzero word of E */
  int hp = -1;
  if (t == 0) {
    hp = E[0] ? 0 : hp;
    hp = E[1] ? 1 : hp;
  }
#pragma unroll
  for (int k = 0; k < LX; ++k) hp = D[k] ? 2 + t * LX + k : hp;
  if (t == G - 1 && cs) hp = W - 1;
  const uint32_t has = grp<G>::ballot(hp >= 0);
  const int top_lane = has ? 31 - __clz((int)has) : 0;
  const int top = __shfl_sync(kFull, hp, top_lane, G);
  const bool zero = has == 0u || ea == kExpZero;
  const int tw = top >= 0 ? (int)E[top] : 1;
  const int msb = 32 * (top >= 0 ? top : 0) + 31 - (int)clz32((uint32_t)tw);
  auto ew = [&](int j) -> uint32_t { return (j >= 0 && j < W) ? E[j] : 0u; };
  /* the result's N words end at bit b0 of E */
  const int b0 = msb - 32 * N + 1;
#pragma unroll
  for (int k = 0; k < L; ++k) {
    const int pos = b0 + 32 * (t * L + k);
    const int wi = pos >> 5; /* floor: pos may be negative */
    r.m[k] = fshr(ew(wi), ew(wi + 1), (uint32_t)(pos & 31));
  }
  const int rp = b0 - 1; /* the round bit's position */
  const uint32_t rb = rp >= 0 ? (ew(rp >> 5) >> (rp & 31)) & 1u : 0u;
  uint32_t s2 = 0u;
#pragma unroll
  for (int j = 0; j < (W + G - 1) / G; ++j) {
    const int w = t + G * j;
    if (w < W) {
      const int below = rp - 32 * w; /* bits of word w under the round bit */
      const uint32_t v = E[w];
      s2 |= below >= 32 ? v : (below > 0 ? (v & ((1u << below) - 1u)) : 0u);
    }
  }
  const uint32_t stk = (grp<G>::ballot(s2 != 0u) != 0u ? 1u : 0u) | st;
  int32_t e = (int32_t)((int64_t)ea + (msb + 1 - 64 - 32 * NX));
  round_nearest<L, G>(r.m, e, rb, stk);
  r.e = e;
  r.s = sa ^ neg;
  if (zero) set_zero(r);
  __syncwarp();
}

/* r = round(x + y) of two group values; sm: 3N + 3 words of this group's
 * shared memory */
template <int L, int G>
__device__ __forceinline__ void add(cv<L> &r, const cv<L> &x, const cv<L> &y, uint32_t *sm) {
  constexpr int N = G * L;
  const uint32_t t = grp<G>::t();
#pragma unroll
  for (int k = 0; k < L; ++k) {
    sm[t * L + k] = x.m[k];
    sm[N + t * L + k] = y.m[k];
  }
  __syncwarp();
  add_round_sm<L, G, L>(r, sm, x.e, x.s, sm + N, y.e, y.s, sm + 2 * N);
}

/* r = round(x1 u1 - x2 u2) (negate = 1) or round(x1 u1 + x2 u2) (negate = 0)
 * from the exact products, one rounding: the complex product's components
 * (MPC_RNDNN).  sm: 6N + 3 words of this group's shared memory. */
template <int L, int G>
__device__ __forceinline__ void fmms_u(cv<L> &r, const cv<L> &x1, const uref &u1, int32_t e1, uint32_t s1,
                                       const cv<L> &x2, const uref &u2, int32_t e2, uint32_t s2, uint32_t negate,
                                       uint32_t *sm) {
  constexpr int N = G * L;
  const uint32_t t = grp<G>::t();
  uint32_t *P1 = sm, *P2 = sm + 2 * N, *E = sm + 4 * N;
  const bool z1 = x1.e == kExpZero || e1 == kExpZero, z2 = x2.e == kExpZero || e2 == kExpZero;
  uint32_t xm[L], hi[L], w1, w2, st;
#pragma unroll
  for (int k = 0; k < L; ++k) xm[k] = z1 ? 0u : x1.m[k];
  mul_u<L, G, true>(hi, P1, w1, w2, st, xm, u1);
#pragma unroll
  for (int k = 0; k < L; ++k) P1[N + t * L + k] = hi[k];
#pragma unroll
  for (int k = 0; k < L; ++k) xm[k] = z2 ? 0u : x2.m[k];
  mul_u<L, G, true>(hi, P2, w1, w2, st, xm, u2);
#pragma unroll
  for (int k = 0; k < L; ++k) P2[N + t * L + k] = hi[k];
  __syncwarp();
  add_round_sm<L, G, 2 * L>(r, P1, z1 ? kExpZero : x1.e + e1, x1.s ^ s1, P2, z2 ? kExpZero : x2.e + e2,
                            x2.s ^ s2 ^ negate, E);
}

}  // namespace coop
}  // namespace mpb

#endif /* __CUDACC__ */
#endif /* MPB_COOP_CUH */
