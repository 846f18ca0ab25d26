/* elementwise.cu -- conversions, element-wise operators and AXPY (real and
 * complex) over the tiled layout.
 *
 * Thread per element; every grid-stride loop walks whole 32-element tiles so
 * warps stay converged (the core's warp votes and the coalesced tile loads
 * depend on it).  Streamed operands use evict-first loads/stores so the
 * read-once AXPY traffic does not displace reused data in L2.
 */
#include <math.h>

#include <initializer_list>

#include "common.cuh"
#include "mpb/coop.cuh"

namespace mpb {

constexpr int kBlock = 128;

/* ---- AoS cu_freal<32N> <-> tiles ---- */
constexpr long long kAosZeroExp = -0x7fffffffffffffLL; /* CU_FREAL_ZERO_EXP */

template <int N>
__device__ __forceinline__ void aos_read(fval<N> &x, const uint8_t *e) {
  const int32_t sign = *(const int32_t *)e;
  const long long ex = *(const long long *)(e + 8);
  const uint32_t *m = (const uint32_t *)(e + 16);
#pragma unroll
  for (int k = 0; k < N; ++k) x.m[k] = m[k];
  if (ex == kAosZeroExp) {
    set_zero(x);
  } else {
    x.e = (int32_t)ex;
    x.s = sign < 0 ? 1u : 0u;
  }
}
template <int N>
__device__ __forceinline__ void aos_write(uint8_t *e, const fval<N> &x) {
  const bool z = is_zero(x);
  *(int32_t *)e = (z || !x.s) ? 1 : -1;
  *(int32_t *)(e + 4) = 0;
  *(long long *)(e + 8) = z ? kAosZeroExp : (long long)x.e;
  uint32_t *m = (uint32_t *)(e + 16);
#pragma unroll
  for (int k = 0; k < N; ++k) m[k] = z ? 0u : x.m[k];
}

template <int N>
__global__ void __launch_bounds__(kBlock) k_pack_aos(size_t n, int cplx, const uint8_t *aos, uint8_t *vec) {
  const size_t es = 16u + 4u * N;
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> re, im;
    if (i >= n) { /* padding lanes of the last tile hold canonical zeros */
      set_zero(re);
      if (cplx)
        store_celem<N>(vec, i, re, re);
      else
        store_elem<N>(vec, i, re);
      continue;
    }
    if (cplx) {
      aos_read<N>(re, aos + i * 2u * es);
      aos_read<N>(im, aos + i * 2u * es + es);
      store_celem<N>(vec, i, re, im);
    } else {
      aos_read<N>(re, aos + i * es);
      store_elem<N>(vec, i, re);
    }
  }
}
template <int N>
__global__ void __launch_bounds__(kBlock) k_unpack_aos(size_t n, int cplx, const uint8_t *vec, uint8_t *aos) {
  const size_t es = 16u + 4u * N;
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    if (i >= n) continue;
    fval<N> re, im;
    if (cplx) {
      load_celem<N>(re, im, vec, i);
      aos_write<N>(aos + i * 2u * es, re);
      aos_write<N>(aos + i * 2u * es + es, im);
    } else {
      load_elem<N>(re, vec, i);
      aos_write<N>(aos + i * es, re);
    }
  }
}

/* ---- double <-> tiles ---- */
/* exact: d = f * 2^k, f in [1/2, 1), F = f * 2^53 a 53-bit integer; all
 * supported precisions hold >= 64 bits (reference from_double semantics) */
template <int N>
__global__ void __launch_bounds__(kBlock) k_from_double(size_t n, const double *d, uint8_t *vec) {
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    if (i >= n) continue;
    const double v = d[i];
    fval<N> x;
#pragma unroll
    for (int k = 0; k < N; ++k) x.m[k] = 0u;
    if (v == 0.0) {
      set_zero(x);
    } else {
      int ex;
      const double f = frexp(fabs(v), &ex);
      const unsigned long long F = (unsigned long long)ldexp(f, 53);
      x.m[N - 1] = (uint32_t)(F >> 21);
      x.m[N - 2] = (uint32_t)(F << 11);
      x.e = ex;
      x.s = v < 0 ? 1u : 0u;
    }
    store_elem<N>(vec, i, x);
  }
}
/* RNDN to 53 bits, then ldexp (reference to_double semantics) */
template <int N>
__global__ void __launch_bounds__(kBlock) k_to_double(size_t n, const uint8_t *vec, double *d) {
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    if (i >= n) continue;
    fval<N> x;
    load_elem<N>(x, vec, i);
    if (is_zero(x)) {
      d[i] = 0.0;
      continue;
    }
    unsigned long long F = ((unsigned long long)x.m[N - 1] << 21) | (x.m[N - 2] >> 11);
    const uint32_t rb = (x.m[N - 2] >> 10) & 1u;
    uint32_t st = x.m[N - 2] & 0x3ffu;
#pragma unroll
    for (int k = 0; k < N - 2; ++k) st |= x.m[k];
    int e = x.e;
    if (rb && (st || (F & 1ull))) {
      F++;
      if (F == (1ull << 53)) {
        F >>= 1;
        e++;
      }
    }
    const double r = ldexp((double)F, e - 53);
    d[i] = x.s ? -r : r;
  }
}

/* ---- element-wise operators ---- */
template <int N>
__global__ void __launch_bounds__(kBlock) k_binop_r(size_t n, int op, const uint8_t *a, const uint8_t *b,
                                                    uint8_t *r) {
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> x, y, z;
    load_elem<N, kStream>(x, a, i);
    load_elem<N, kStream>(y, b, i);
    if (op == MPB_OP_MUL)
      mul<N>(z, x, y);
    else if (op == MPB_OP_ADD)
      add<N, true>(z, x, y);
    else
      sub<N, true>(z, x, y);
    if (i < n) store_elem<N, kStream>(r, i, z);
  }
}
template <int N>
__global__ void __launch_bounds__(kBlock) k_fma_r(size_t n, const uint8_t *a, const uint8_t *b, const uint8_t *c,
                                                  uint8_t *r) {
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> x, y, w, z;
    load_elem<N, kStream>(x, a, i);
    load_elem<N, kStream>(y, b, i);
    load_elem<N, kStream>(w, c, i);
    fma<N, true>(z, x, y, w);
    if (i < n) store_elem<N, kStream>(r, i, z);
  }
}
template <int N>
__global__ void __launch_bounds__(kBlock) k_binop_c(size_t n, int op, const uint8_t *a, const uint8_t *b,
                                                    uint8_t *r) {
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> ar, ai, br, bi, zr, zi;
    load_celem<N, kStream>(ar, ai, a, i);
    load_celem<N, kStream>(br, bi, b, i);
    if (op == MPB_OP_MUL) {
      cmul<N, true>(zr, zi, ar, ai, br, bi);
    } else if (op == MPB_OP_ADD) {
      add<N, true>(zr, ar, br);
      add<N, true>(zi, ai, bi);
    } else {
      sub<N, true>(zr, ar, br);
      sub<N, true>(zi, ai, bi);
    }
    if (i < n) store_celem<N, kStream>(r, i, zr, zi);
  }
}

/* ---- AXPY ---- */
/* z = round(round(a*x) + y): the scalar a lives in shared memory (warp-
 * uniform broadcast reads, no registers held), and it is the row multiplier
 * of the schoolbook product, so each of its limbs is read once per product.
 * A scalar whose limbs below the top one or two are zero (one converted from
 * a double, a small integer: 1.5, 2, -0.25 ...) takes the exact short product
 * (mul_short: N or 2N partial products instead of the ~N^2/2 upper columns);
 * the branch is uniform over the grid and the result is the same. */
template <int N>
__global__ void __launch_bounds__(kBlock) k_axpy_r(size_t n, const uint8_t *a, const uint8_t *x, const uint8_t *y,
                                                   uint8_t *z) {
  __shared__ fval<N> sa;
  __shared__ int klen;
  if (threadIdx.x == 0) {
    fval<N> t;
    load_elem<N>(t, a, 0);
    sa = t;
    klen = limb_length<N>(t.m);
  }
  __syncthreads();
  const int kl = N > 2 ? klen : N;
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> xv, yv, t, r;
    load_elem<N, kStream>(xv, x, i);
    load_elem<N, kStream>(yv, y, i);
    if constexpr (N > 2) {
      if (kl == 1)
        mul_short<N, 1>(t, xv, sa.m, sa.e, sa.s);
      else if (kl == 2)
        mul_short<N, 2>(t, xv, sa.m, sa.e, sa.s);
      else
        mul<N>(t, xv, sa);
    } else {
      mul<N>(t, xv, sa);
    }
    add<N, true>(r, t, yv);
    if (i < n) store_elem<N, kStream>(z, i, r);
  }
}
/* complex z = a*x + y: re = round(xr*ar - xi*ai), im = round(xr*ai + xi*ar)
 * from exact products (the scalar as row multiplier again), then the
 * component-wise rounded add of y.  Both components share the x operands and
 * differ only in which part of a multiplies them, so the body runs as a
 * two-trip loop over the component with the a parts picked by pointer: one
 * copy of the product/rounding code instead of two keeps the loop inside the
 * instruction cache at high precision. */
template <int N>
__global__ void __launch_bounds__(kBlock) k_axpy_c(size_t n, const uint8_t *a, const uint8_t *x, const uint8_t *y,
                                                   uint8_t *z) {
  __shared__ fval<N> sa[2];
  if (threadIdx.x == 0) {
    fval<N> tr, ti;
    load_celem<N>(tr, ti, a, 0);
    sa[0] = tr;
    sa[1] = ti;
  }
  __syncthreads();
  const size_t np = tiles_for(n) * 32u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    fval<N> xr, xi;
    load_celem<N, kStream>(xr, xi, x, i);
    const size_t ct = (i >> 5) * 2u * sol<N>::kTileBytes;
#pragma unroll 1
    for (int comp = 0; comp < 2; ++comp) {
      /* re: xr*ar - xi*ai ; im: xr*ai + xi*ar */
      const fval<N> &a1 = sa[comp];
      const fval<N> &a2 = sa[comp ^ 1];
      fval<N> t, yv, r;
      fmms<N, true>(t, xr, a1, xi, a2, comp == 0 ? 1u : 0u);
      load_elem<N, kStream>(yv, y + ct + comp * sol<N>::kTileBytes, i & 31u);
      add<N, true>(r, t, yv);
      if (i < n) store_elem<N, kStream>(z + ct + comp * sol<N>::kTileBytes, i & 31u, r);
    }
  }
}

/* complex AXPY with a group of G lanes per element (the warp-cooperative form
 * for wide operands): both components of a*x from the exact products, one
 * rounding each (coop::fmms_u, the scalar's parts as the uniform operands),
 * then the rounded adds of y, as k_axpy_c */
template <int L, int G>
__global__ void __launch_bounds__(kBlock) k_axpy_c_coop(size_t n, const uint8_t *a, const uint8_t *x, const uint8_t *y,
                                                        uint8_t *z) {
  constexpr int N = G * L, EPW = 32 / G, SMW = 6 * N + 3;
  constexpr size_t TB = sol<N>::kTileBytes;
  __shared__ uint32_t sm_all[(kBlock / 32) * EPW * SMW];
  const uint32_t warp = threadIdx.x >> 5, gw = (threadIdx.x & 31u) / G;
  uint32_t *sm = sm_all + (warp * EPW + gw) * SMW;
  const coop::uref ar{a, 0u}, ai{a + TB, 0u}; /* element 0: re tile, then im tile */
  int32_t are, aie;
  uint32_t ars, ais;
  coop::uniform_head<N>(ar, are, ars);
  coop::uniform_head<N>(ai, aie, ais);
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  const size_t egroups = (n + EPW - 1) / EPW;
  for (size_t eg = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; eg < egroups; eg += nw) {
    const size_t i = eg * EPW + gw;
    const size_t ic = i < n ? i : n - 1; /* lanes past the end recompute the last element */
    const uint8_t *xt = x + (ic >> 5) * 2u * TB;
    const uint8_t *yt = y + (ic >> 5) * 2u * TB;
    const uint32_t slot = (uint32_t)(ic & 31u);
    coop::cv<L> xr, xi, yv, re, im;
    coop::load<L, G, kStream>(xr, xt, slot);
    coop::load<L, G, kStream>(xi, xt + TB, slot);
    coop::fmms_u<L, G>(re, xr, ar, are, ars, xi, ai, aie, ais, 1u, sm); /* xr ar - xi ai */
    coop::fmms_u<L, G>(im, xr, ai, aie, ais, xi, ar, are, ars, 0u, sm); /* xr ai + xi ar */
    coop::load<L, G, kStream>(yv, yt, slot);
    coop::add<L, G>(re, re, yv, sm);
    coop::load<L, G, kStream>(yv, yt + TB, slot);
    coop::add<L, G>(im, im, yv, sm);
    if (i < n) {
      uint8_t *zt = z + (i >> 5) * 2u * TB;
      coop::store<L, G, kStream>(zt, slot, re);
      coop::store<L, G, kStream>(zt + TB, slot, im);
    }
  }
}

} /* namespace mpb */

using namespace mpb;

/* ------------------------------------------------------------------ *
 * C ABI
 * ------------------------------------------------------------------ */
#define MPB_CHECK(x)            \
  do {                          \
    const int _rc = (x);        \
    if (_rc != MPB_OK) return _rc; \
  } while (0)

static int conv_common(int prec, size_t n, const void *p, const void *q) {
  if (!prec_ok(prec)) return MPB_ERR_PREC;
  if (n > kMaxElems) return MPB_ERR_SIZE;
  if (n == 0) return 1; /* no-op */
  if (!p || !q) return MPB_ERR_NULL;
  return MPB_OK;
}

extern "C" int mpb_pack_aos(int prec, size_t n, const void *aos, void *vec, void *stream) {
  const int rc = conv_common(prec, n, aos, vec);
  if (rc != MPB_OK) return rc > 0 ? MPB_OK : rc;
  if (!aligned16(vec) || ((uintptr_t)aos & 7u)) return MPB_ERR_ALIGN;
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_pack_aos<N>, kBlock, tiles_for(n) * 32u);
    k_pack_aos<N><<<g, kBlock, 0, as_stream(stream)>>>(n, 0, (const uint8_t *)aos, (uint8_t *)vec);
  });
  return launch_status();
}
extern "C" int mpb_unpack_aos(int prec, size_t n, const void *vec, void *aos, void *stream) {
  const int rc = conv_common(prec, n, aos, vec);
  if (rc != MPB_OK) return rc > 0 ? MPB_OK : rc;
  if (!aligned16(vec) || ((uintptr_t)aos & 7u)) return MPB_ERR_ALIGN;
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_unpack_aos<N>, kBlock, tiles_for(n) * 32u);
    k_unpack_aos<N><<<g, kBlock, 0, as_stream(stream)>>>(n, 0, (const uint8_t *)vec, (uint8_t *)aos);
  });
  return launch_status();
}
extern "C" int mpb_cpack_aos(int prec, size_t n, const void *aos, void *cvec, void *stream) {
  const int rc = conv_common(prec, n, aos, cvec);
  if (rc != MPB_OK) return rc > 0 ? MPB_OK : rc;
  if (!aligned16(cvec) || ((uintptr_t)aos & 7u)) return MPB_ERR_ALIGN;
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_pack_aos<N>, kBlock, tiles_for(n) * 32u);
    k_pack_aos<N><<<g, kBlock, 0, as_stream(stream)>>>(n, 1, (const uint8_t *)aos, (uint8_t *)cvec);
  });
  return launch_status();
}
extern "C" int mpb_cunpack_aos(int prec, size_t n, const void *cvec, void *aos, void *stream) {
  const int rc = conv_common(prec, n, aos, cvec);
  if (rc != MPB_OK) return rc > 0 ? MPB_OK : rc;
  if (!aligned16(cvec) || ((uintptr_t)aos & 7u)) return MPB_ERR_ALIGN;
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_unpack_aos<N>, kBlock, tiles_for(n) * 32u);
    k_unpack_aos<N><<<g, kBlock, 0, as_stream(stream)>>>(n, 1, (const uint8_t *)cvec, (uint8_t *)aos);
  });
  return launch_status();
}
extern "C" int mpb_from_double(int prec, size_t n, const double *d, void *vec, void *stream) {
  const int rc = conv_common(prec, n, d, vec);
  if (rc != MPB_OK) return rc > 0 ? MPB_OK : rc;
  if (!aligned16(vec) || ((uintptr_t)d & 7u)) return MPB_ERR_ALIGN;
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_from_double<N>, kBlock, tiles_for(n) * 32u);
    k_from_double<N><<<g, kBlock, 0, as_stream(stream)>>>(n, d, (uint8_t *)vec);
  });
  return launch_status();
}
extern "C" int mpb_to_double(int prec, size_t n, const void *vec, double *d, void *stream) {
  const int rc = conv_common(prec, n, d, vec);
  if (rc != MPB_OK) return rc > 0 ? MPB_OK : rc;
  if (!aligned16(vec) || ((uintptr_t)d & 7u)) return MPB_ERR_ALIGN;
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_to_double<N>, kBlock, tiles_for(n) * 32u);
    k_to_double<N><<<g, kBlock, 0, as_stream(stream)>>>(n, (const uint8_t *)vec, d);
  });
  return launch_status();
}


static int vec_args(int prec, size_t n, std::initializer_list<const void *> bufs) {
  if (!prec_ok(prec)) return MPB_ERR_PREC;
  if (n > kMaxElems) return MPB_ERR_SIZE;
  if (n == 0) return 1;
  for (const void *p : bufs) MPB_CHECK(check_buf(p));
  return MPB_OK;
}

extern "C" int mpb_binop_r(int prec, int op, size_t n, const void *a, const void *b, void *r, void *stream) {
  if (op != MPB_OP_MUL && op != MPB_OP_ADD && op != MPB_OP_SUB) return MPB_ERR_ARG;
  const int rc = vec_args(prec, n, {a, b, r});
  if (rc != MPB_OK) return rc > 0 ? MPB_OK : rc;
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_binop_r<N>, kBlock, tiles_for(n) * 32u);
    k_binop_r<N><<<g, kBlock, 0, as_stream(stream)>>>(n, op, (const uint8_t *)a, (const uint8_t *)b, (uint8_t *)r);
  });
  return launch_status();
}
extern "C" int mpb_fma_r(int prec, size_t n, const void *a, const void *b, const void *c, void *r, void *stream) {
  const int rc = vec_args(prec, n, {a, b, c, r});
  if (rc != MPB_OK) return rc > 0 ? MPB_OK : rc;
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_fma_r<N>, kBlock, tiles_for(n) * 32u);
    k_fma_r<N><<<g, kBlock, 0, as_stream(stream)>>>(n, (const uint8_t *)a, (const uint8_t *)b, (const uint8_t *)c,
                                                  (uint8_t *)r);
  });
  return launch_status();
}
extern "C" int mpb_binop_c(int prec, int op, size_t n, const void *a, const void *b, void *r, void *stream) {
  if (op != MPB_OP_MUL && op != MPB_OP_ADD && op != MPB_OP_SUB) return MPB_ERR_ARG;
  const int rc = vec_args(prec, n, {a, b, r});
  if (rc != MPB_OK) return rc > 0 ? MPB_OK : rc;
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_binop_c<N>, kBlock, tiles_for(n) * 32u);
    k_binop_c<N><<<g, kBlock, 0, as_stream(stream)>>>(n, op, (const uint8_t *)a, (const uint8_t *)b, (uint8_t *)r);
  });
  return launch_status();
}
extern "C" int mpb_axpy_r(int prec, size_t n, const void *a, const void *x, const void *y, void *z, void *stream) {
  const int rc = vec_args(prec, n, {a, x, y, z});
  if (rc != MPB_OK) return rc > 0 ? MPB_OK : rc;
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_axpy_r<N>, kBlock, tiles_for(n) * 32u);
    k_axpy_r<N><<<g, kBlock, 0, as_stream(stream)>>>(n, (const uint8_t *)a, (const uint8_t *)x, (const uint8_t *)y,
                                                   (uint8_t *)z);
  });
  return launch_status();
}
extern "C" int mpb_axpy_c(int prec, size_t n, const void *a, const void *x, const void *y, void *z, void *stream) {
  const int rc = vec_args(prec, n, {a, x, y, z});
  if (rc != MPB_OK) return rc > 0 ? MPB_OK : rc;
  const int lanes = split_lanes(MPB_SPLIT_AXPY_C, prec);
  if (prec == 1024 && lanes > 1) {
    const size_t warps = (n + 32 / lanes - 1) / (32 / lanes);
    if (lanes == 4) {
      const int g = grid_for(k_axpy_c_coop<8, 4>, kBlock, warps * 32u);
      k_axpy_c_coop<8, 4><<<g, kBlock, 0, as_stream(stream)>>>(n, (const uint8_t *)a, (const uint8_t *)x,
                                                              (const uint8_t *)y, (uint8_t *)z);
    } else {
      const int g = grid_for(k_axpy_c_coop<4, 8>, kBlock, warps * 32u);
      k_axpy_c_coop<4, 8><<<g, kBlock, 0, as_stream(stream)>>>(n, (const uint8_t *)a, (const uint8_t *)x,
                                                              (const uint8_t *)y, (uint8_t *)z);
    }
    return launch_status();
  }
  MPB_DISPATCH_PREC(prec, {
    const int g = grid_for(k_axpy_c<N>, kBlock, tiles_for(n) * 32u);
    k_axpy_c<N><<<g, kBlock, 0, as_stream(stream)>>>(n, (const uint8_t *)a, (const uint8_t *)x, (const uint8_t *)y,
                                                   (uint8_t *)z);
  });
  return launch_status();
}
