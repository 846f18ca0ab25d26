/* mpfr_interop.cu -- host-side conversion between AoS cu_freal / cu_fcomplex
 * arrays and MPFR's mpfr_t / MPC's mpc_t objects, without linking MPFR.
 *
 * The reference converts with mpz_import + mpfr_set_z (RNDN) + mpfr_mul_2si
 * (tools/test_freal.cu:28-39): the value rounded to nearest-even at the
 * destination's precision, exact when that precision is large enough.  These
 * helpers give the same results by writing and reading the mpfr_t fields
 * directly, using MPFR's public struct layout (mpfr.h, MPFR >= 3):
 *   { long prec; int sign; long exp; uint64_t *d }   (64-bit limbs)
 * value = sign * 0.d * 2^exp, the top limb's top bit set, the bits below prec
 * zero; exp = -LONG_MAX marks zero, 1 - LONG_MAX NaN, 2 - LONG_MAX infinity.
 * cu_freal uses the same significand / exponent convention, so a conversion
 * is a copy of limbs plus, when the precisions differ, one rounding.  The
 * destination mpfr_t must be initialised (mpfr_init2) by the caller; its
 * precision is kept.  Exponents must lie within the mpfr_t's current range
 * (MPFR's default +-(2^30 - 1) covers the engine's).
 */
#include <climits>
#include <cstdint>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace {

struct mpfr_view {
  long prec;
  int sign;
  long exp;
  uint64_t *d;
};

constexpr long kExpZeroMpfr = -LONG_MAX;
constexpr long kExpNanMpfr = 1 - LONG_MAX;
constexpr long kExpInfMpfr = 2 - LONG_MAX;
constexpr int64_t kAosZeroExp = -0x7fffffffffffffLL; /* CU_FREAL_ZERO_EXP, reference cu_freal.cuh:37 */

/* dst (nd limbs, q significant bits) = src (ns limbs, MSB set) rounded to
 * nearest-even at q bits; returns 1 when the rounding carried out of the top
 * (dst is then 1000...0 and the exponent grows by one) */
int round_limbs(uint64_t *dst, int nd, long q, const uint64_t *src, int ns) {
  /* align: dst[nd-1] <- src[ns-1], ... */
  for (int i = 0; i < nd; ++i) {
    const int j = ns - nd + i;
    dst[i] = (j >= 0) ? src[j] : 0u;
  }
  const long lowbits = 64L * nd - q; /* bits of dst[0] below precision */
  /* round bit and sticky: from dst's discarded low bits and src limbs below dst */
  uint64_t rb = 0, st = 0;
  if (lowbits > 0) {
    const uint64_t mask = (lowbits >= 64) ? ~0ull : ((1ull << lowbits) - 1u);
    const uint64_t half = 1ull << (lowbits - 1);
    rb = (dst[0] & half) ? 1u : 0u;
    st = (dst[0] & (mask >> 1)) ? 1u : 0u;
    dst[0] &= ~mask;
  }
  for (int j = 0; j < ns - nd; ++j) {
    if (j == ns - nd - 1 && lowbits == 0) {
      rb = src[j] >> 63;
      st |= (src[j] << 1) ? 1u : 0u;
    } else {
      st |= src[j] ? 1u : 0u;
    }
  }
  const uint64_t ulp = (lowbits > 0) ? (1ull << lowbits) : 1u;
  const uint64_t lsb = (dst[0] & ulp) ? 1u : 0u;
  if (!(rb && (st || lsb))) return 0;
  uint64_t c = ulp;
  for (int i = 0; i < nd && c; ++i) {
    const uint64_t s = dst[i] + c;
    c = (s < dst[i]) ? 1u : 0u;
    dst[i] = s;
  }
  if (c) { /* carried out: the significand becomes 0.1000...0 */
    for (int i = 0; i < nd; ++i) dst[i] = 0u;
    dst[nd - 1] = 1ull << 63;
    return 1;
  }
  return 0;
}

struct aos_view { /* cu_freal<PB>: { int sign; long exp; uint64_t m[N] } */
  int32_t sign;
  int32_t pad;
  int64_t exp;
};

int to_mpfr_one(int prec, const uint8_t *e, mpfr_view *z) {
  const int n64 = (prec + 63) / 64;
  const aos_view *h = (const aos_view *)e;
  const uint64_t *m = (const uint64_t *)(e + 16);
  if (!z || z->prec < 1 || !z->d) return MPB_ERR_ARG;
  if (h->exp == kAosZeroExp) {
    z->sign = 1;
    z->exp = kExpZeroMpfr;
    return MPB_OK;
  }
  const int nd = (int)((z->prec + 63) / 64);
  std::vector<uint64_t> d((size_t)nd);
  const long e2 = (long)h->exp + round_limbs(d.data(), nd, z->prec, m, n64);
  /* MPFR's default exponent range is [1 - 2^30, 2^30 - 1]; a value outside it
   * (possible after a carry at the top, or from a head at the range's edge)
   * would make an invalid mpfr_t, so it is refused and z is left unchanged */
  if (e2 > (1L << 30) - 1 || e2 < 1 - (1L << 30)) return MPB_ERR_ARG;
  std::memcpy(z->d, d.data(), 8u * (size_t)nd);
  z->exp = e2;
  z->sign = h->sign < 0 ? -1 : 1;
  return MPB_OK;
}

int from_mpfr_one(int prec, const mpfr_view *z, uint8_t *e) {
  const int n64 = (prec + 63) / 64;
  aos_view *h = (aos_view *)e;
  uint64_t *m = (uint64_t *)(e + 16);
  if (!z) return MPB_ERR_NULL;
  if (z->exp == kExpNanMpfr || z->exp == kExpInfMpfr) return MPB_ERR_ARG; /* no NaN or infinity here */
  if (z->exp == kExpZeroMpfr) {
    h->pad = 0;
    h->sign = 1;
    h->exp = kAosZeroExp;
    std::memset(m, 0, 8u * (size_t)n64);
    return MPB_OK;
  }
  const int ns = (int)((z->prec + 63) / 64);
  uint64_t d[32]; /* n64 <= 32 (PB <= 2048) */
  const long e2 = z->exp + round_limbs(d, n64, prec, z->d, ns);
  /* outside the engine's exponent range: refused before anything is written,
   * so the element keeps its old value */
  if (e2 >= (1L << 30) || e2 <= -(1L << 30)) return MPB_ERR_ARG;
  std::memcpy(m, d, 8u * (size_t)n64);
  h->pad = 0;
  h->exp = e2;
  h->sign = z->sign < 0 ? -1 : 1;
  return MPB_OK;
}

}  // namespace

extern "C" int mpb_aos_to_mpfr(int prec, size_t n, const void *aos, void *const *dst) {
  if (!mpb::prec_ok(prec)) return MPB_ERR_PREC;
  if (n == 0) return MPB_OK;
  if (!aos || !dst) return MPB_ERR_NULL;
  const size_t es = 16u + 8u * (size_t)((prec + 63) / 64);
  for (size_t i = 0; i < n; ++i) {
    const int rc = to_mpfr_one(prec, (const uint8_t *)aos + i * es, (mpfr_view *)dst[i]);
    if (rc != MPB_OK) return rc;
  }
  return MPB_OK;
}

extern "C" int mpb_aos_from_mpfr(int prec, size_t n, const void *const *src, void *aos) {
  if (!mpb::prec_ok(prec)) return MPB_ERR_PREC;
  if (n == 0) return MPB_OK;
  if (!aos || !src) return MPB_ERR_NULL;
  const size_t es = 16u + 8u * (size_t)((prec + 63) / 64);
  for (size_t i = 0; i < n; ++i) {
    const int rc = from_mpfr_one(prec, (const mpfr_view *)src[i], (uint8_t *)aos + i * es);
    if (rc != MPB_OK) return rc;
  }
  return MPB_OK;
}

/* mpc_t = { mpfr re; mpfr im } (mpc.h); complex AoS = { cu_freal re; cu_freal im } */
extern "C" int mpb_caos_to_mpc(int prec, size_t n, const void *caos, void *const *dst) {
  if (!mpb::prec_ok(prec)) return MPB_ERR_PREC;
  if (n == 0) return MPB_OK;
  if (!caos || !dst) return MPB_ERR_NULL;
  const size_t es = 16u + 8u * (size_t)((prec + 63) / 64);
  for (size_t i = 0; i < n; ++i) {
    mpfr_view *z = (mpfr_view *)dst[i];
    if (!z) return MPB_ERR_NULL;
    for (int c = 0; c < 2; ++c) {
      const int rc = to_mpfr_one(prec, (const uint8_t *)caos + (2 * i + c) * es, z + c);
      if (rc != MPB_OK) return rc;
    }
  }
  return MPB_OK;
}

extern "C" int mpb_caos_from_mpc(int prec, size_t n, const void *const *src, void *caos) {
  if (!mpb::prec_ok(prec)) return MPB_ERR_PREC;
  if (n == 0) return MPB_OK;
  if (!caos || !src) return MPB_ERR_NULL;
  const size_t es = 16u + 8u * (size_t)((prec + 63) / 64);
  for (size_t i = 0; i < n; ++i) {
    const mpfr_view *z = (const mpfr_view *)src[i];
    if (!z) return MPB_ERR_NULL;
    for (int c = 0; c < 2; ++c) {
      const int rc = from_mpfr_one(prec, z + c, (uint8_t *)caos + (2 * i + c) * es);
      if (rc != MPB_OK) return rc;
    }
  }
  return MPB_OK;
}
