/* mpb_oracle.c -- CPU ORACLE.  TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library, and only as the checker or as the timed CPU baseline.  The
 * product (libmpb.so) never links, loads or calls it.
 *
 * Two independent halves:
 *
 *  (1) A plain-C restatement of the reference's fixed-precision arithmetic
 *      (mpc_cuda include/mpc_cuda/cu_freal.cuh, include/mpc_cuda/cu_fcomplex.cuh)
 *      and of the loops its kernels run (demos/bench_3way.cu, tools/linalg_fast.cu,
 *      tools/axpy_fast_complex.cu, demos/matmul_mpc.cu).  Each function names
 *      the reference lines whose behaviour it restates.  It works on 64-bit
 *      limbs exactly like the reference so that SB=32 precisions (96, 160, ...)
 *      are covered too.
 *
 *  (2) The same operations computed by the system MPFR 4.2.1 / MPC 1.3.1
 *      libraries (through mpfr_shim.h), which is the correctness oracle the
 *      reference itself is tested against (tools/test_freal.cu:69-76,
 *      tools/test_fcomplex.cu:71-78, tools/linalg_fast.cu:71-83).
 *
 * Element format (both halves): the reference's AoS struct cu_freal<PB>
 *   { int32 sign; int32 pad; int64 exp; uint64 m[N64]; }   N64 = ceil(PB/64)
 * value = sign * M * 2^(exp - 64*N64), M = sum m[i] 2^(64 i), m[N64-1] MSB set,
 * low SB = 64*N64 - PB bits zero; zero is exp == ORC_ZERO_EXP
 * (cu_freal.cuh:12-16,37,67-81).  A complex element is {re, im}.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "mpfr_shim.h"

typedef uint64_t u64;
typedef unsigned __int128 u128;

#define ORC_ZERO_EXP (-0x7fffffffffffffLL) /* cu_freal.cuh:37 */
#define ORC_MAXN64 64                      /* PB <= 4096 */
#define ORC_WBUF (2 * ORC_MAXN64 + 4)

typedef struct {
  int32_t sign;
  int32_t pad;
  int64_t exp;
  u64 m[];
} elem_t;

static inline int n64_of(int P) { return (P + 63) / 64; }
static inline size_t esz_of(int P) { return 16 + 8 * (size_t)n64_of(P); }
static inline elem_t *at(void *base, size_t esz, long i) {
  return (elem_t *)((char *)base + (size_t)i * esz);
}
static inline const elem_t *cat(const void *base, size_t esz, long i) {
  return (const elem_t *)((const char *)base + (size_t)i * esz);
}
static inline int is_zero(const elem_t *x) { return x->exp == ORC_ZERO_EXP; }
static inline void set_zero(int P, elem_t *r) {
  r->sign = 1;
  r->pad = 0;
  r->exp = ORC_ZERO_EXP;
  memset(r->m, 0, 8 * (size_t)n64_of(P));
}
static inline void copy_elem(int P, elem_t *r, const elem_t *x) {
  memcpy(r, x, esz_of(P));
}

/* floor division helpers for signed bit positions */
static inline long fdiv64(long x) { return x >= 0 ? x / 64 : -((-x + 63) / 64); }

/* 64 bits of the little-endian integer D[len] starting at signed bit
 * position pos (bits outside [0, 64*len) read as zero). */
static u64 bits64_at(const u64 *D, int len, long pos) {
  long w = fdiv64(pos);
  int b = (int)(pos - 64 * w);
  u64 lo = (w >= 0 && w < len) ? D[w] : 0;
  u64 hi = (w + 1 >= 0 && w + 1 < len) ? D[w + 1] : 0;
  return b ? (lo >> b) | (hi << (64 - b)) : lo;
}
/* single bit i of D (cu_freal.cuh:52-54) */
static u64 bit_at(const u64 *D, int len, long i) {
  if (i < 0 || i >= 64L * len) return 0;
  return (D[i >> 6] >> (i & 63)) & 1;
}
/* 1 if any of bits [0, i) of D is set (cu_freal.cuh:56-64) */
static u64 any_below(const u64 *D, int len, long i) {
  if (i <= 0) return 0;
  long full = i >> 6;
  for (long j = 0; j < full && j < len; j++)
    if (D[j]) return 1;
  int rem = (int)(i & 63);
  if (rem && full < len && (D[full] & ((((u64)1) << rem) - 1))) return 1;
  return 0;
}
/* index of the highest set bit of D, -1 if D == 0 */
static long top_bit(const u64 *D, int len) {
  for (int i = len - 1; i >= 0; i--)
    if (D[i]) return 64L * i + 63 - __builtin_clzll(D[i]);
  return -1;
}

/* Round the exact magnitude D[len] to P bits, round-to-nearest-even, and store
 * into r.  Bit `msb` of D is the leading one and has weight 2^Ehi; rnd/sti are
 * round/sticky material lying strictly below bit 0 of D.
 * Restates the single rounding point cu_freal<PB>::finalize
 * (cu_freal.cuh:89-138): keep bits [msb-P+1, msb], round on the next bit with
 * the OR of everything below as sticky, renormalise on carry-out, then
 * left-justify the P-bit result in N64 limbs (low SB bits zero). */
static void round_into(int P, elem_t *r, const u64 *D, int len, long msb, long Ehi,
                       u64 rnd, u64 sti, int sgn) {
  const int N = n64_of(P), SB = 64 * N - P;
  if (msb < 0) {
    set_zero(P, r);
    return;
  }
  long lo = msb - P + 1; /* weight-0 bit of the kept P-bit window */
  u64 V[ORC_MAXN64 + 1];
  for (int i = 0; i < N; i++) V[i] = bits64_at(D, len, lo + 64L * i);
  /* bits of V above P-1 belong to nothing (window is exactly P bits) */
  if (SB) V[N - 1] &= (((u64)1) << (64 - SB)) - 1;
  u64 rb, st;
  if (lo > 0) {
    rb = bit_at(D, len, lo - 1);
    st = rnd | sti | any_below(D, len, lo - 1);
  } else if (lo == 0) {
    rb = rnd;
    st = sti;
  } else { /* fewer than P significant bits: the value is exact */
    rb = 0;
    st = 0;
  }
  long E = Ehi;
  if (rb && (st || (V[0] & 1))) {
    u64 c = 1;
    for (int i = 0; i < N && c; i++) {
      V[i] += c;
      c = (V[i] == 0);
    }
    int carried = SB ? (int)((V[N - 1] >> (64 - SB)) & 1) : (int)c;
    if (carried) { /* P-bit window overflowed to 2^P: becomes 2^(P-1), E+1 */
      memset(V, 0, sizeof(u64) * N);
      V[(P - 1) >> 6] = ((u64)1) << ((P - 1) & 63);
      E++;
    }
  }
  /* left-justify: M = V << SB */
  for (int i = N - 1; i >= 0; i--) {
    u64 hi = V[i], lo2 = (i > 0) ? V[i - 1] : 0;
    r->m[i] = SB ? (hi << SB) | (lo2 >> (64 - SB)) : hi;
  }
  r->sign = sgn;
  r->pad = 0;
  r->exp = E + 1;
}

/* ---------------- exact products ---------------- */
/* N x N -> 2N limb schoolbook product (cu_freal.cuh:174-200) */
static void mul_exact(int N, u64 *R, const u64 *a, const u64 *b) {
  memset(R, 0, sizeof(u64) * 2 * N);
  for (int j = 0; j < N; j++) {
    u64 carry = 0;
    for (int i = 0; i < N; i++) {
      u128 t = (u128)a[i] * b[j] + R[i + j] + carry;
      R[i + j] = (u64)t;
      carry = (u64)(t >> 64);
    }
    R[N + j] = carry;
  }
}

/* r = round(a * b)  (cu_fmul, cu_freal.cuh:203-213) */
static void o_mul(int P, elem_t *r, const elem_t *a, const elem_t *b) {
  const int N = n64_of(P);
  if (is_zero(a) || is_zero(b)) {
    set_zero(P, r);
    return;
  }
  u64 W[ORC_WBUF];
  mul_exact(N, W, a->m, b->m);
  long msb = (W[2 * N - 1] >> 63) ? 128L * N - 1 : 128L * N - 2;
  long Ehi = a->exp + b->exp - 128L * N + msb;
  round_into(P, r, W, 2 * N, msb, Ehi, 0, 0, a->sign * b->sign);
}

/* magnitude order by (exp, limbs)  (cu_freal.cuh:216-222) */
static int mag_cmp(int N, const elem_t *a, const elem_t *b) {
  if (a->exp != b->exp) return a->exp > b->exp ? 1 : -1;
  for (int i = N - 1; i >= 0; i--)
    if (a->m[i] != b->m[i]) return a->m[i] > b->m[i] ? 1 : -1;
  return 0;
}

/* r = round(|a| + |b|) with sign sgn  (cu_addmag, cu_freal.cuh:225-245):
 * align the smaller operand into N limbs, its lost bits feed round/sticky. */
static void o_addmag(int P, elem_t *r, const elem_t *a, const elem_t *b, int sgn) {
  const int N = n64_of(P);
  if (b->exp > a->exp) {
    const elem_t *t = a;
    a = b;
    b = t;
  }
  long d = a->exp - b->exp;
  u64 Bs[ORC_MAXN64], D[ORC_MAXN64 + 1];
  for (int i = 0; i < N; i++) Bs[i] = (d >= 64L * N) ? 0 : bits64_at(b->m, N, d + 64L * i);
  u64 rb = bit_at(b->m, N, d - 1), st = any_below(b->m, N, d - 1);
  u64 c = 0;
  for (int i = 0; i < N; i++) {
    u128 s = (u128)a->m[i] + Bs[i] + c;
    D[i] = (u64)s;
    c = (u64)(s >> 64);
  }
  D[N] = c;
  long msb = c ? 64L * N : 64L * N - 1;
  round_into(P, r, D, N + 1, msb, a->exp - 64L * N + msb, rb, st, sgn);
}

/* r = round(|a| - |b|), |a| > |b|, sign sgn  (cu_submag, cu_freal.cuh:248-277):
 * a 2-limb (128-bit) guard window below a; any bit of b shifted below the
 * window makes the window difference one unit too large, so subtract one unit
 * and carry the fact as sticky. */
static void o_submag(int P, elem_t *r, const elem_t *a, const elem_t *b, int sgn) {
  const int N = n64_of(P), W = N + 2;
  long d = a->exp - b->exp;
  u64 A[ORC_MAXN64 + 2], Bw[ORC_MAXN64 + 2], T[ORC_MAXN64 + 2], D[ORC_MAXN64 + 2];
  memset(A, 0, sizeof(u64) * W);
  memset(T, 0, sizeof(u64) * W);
  for (int i = 0; i < N; i++) {
    A[i + 2] = a->m[i];
    T[i + 2] = b->m[i];
  }
  u64 ext;
  if (d < 64L * W) {
    ext = any_below(T, W, d);
    for (int i = 0; i < W; i++) Bw[i] = bits64_at(T, W, d + 64L * i);
  } else {
    ext = 1;
    memset(Bw, 0, sizeof(u64) * W);
  }
  u64 br = 0;
  for (int i = 0; i < W; i++) {
    u128 s = (u128)A[i] - Bw[i] - br;
    D[i] = (u64)s;
    br = (u64)(s >> 64) & 1;
  }
  if (ext) {
    for (int i = 0; i < W; i++) {
      u64 old = D[i];
      D[i] = old - 1;
      if (old != 0) break;
    }
  }
  long msb = top_bit(D, W);
  if (msb < 0) {
    set_zero(P, r);
    return;
  }
  round_into(P, r, D, W, msb, a->exp - 64L * W + msb, 0, ext, sgn);
}

/* r = round(a + b)  (cu_fadd, cu_freal.cuh:280-289) */
static void o_add(int P, elem_t *r, const elem_t *a, const elem_t *b) {
  const int N = n64_of(P);
  if (is_zero(a)) {
    copy_elem(P, r, b);
    return;
  }
  if (is_zero(b)) {
    copy_elem(P, r, a);
    return;
  }
  if (a->sign == b->sign) {
    o_addmag(P, r, a, b, a->sign);
    return;
  }
  int c = mag_cmp(N, a, b);
  if (c == 0) {
    set_zero(P, r);
    return;
  }
  if (c > 0)
    o_submag(P, r, a, b, a->sign);
  else
    o_submag(P, r, b, a, b->sign);
}
/* r = round(a - b)  (cu_fsub, cu_freal.cuh:290-292) */
static void o_sub(int P, elem_t *r, const elem_t *a, const elem_t *b) {
  u64 buf[2 + ORC_MAXN64 + 2];
  elem_t *nb = (elem_t *)buf;
  copy_elem(P, nb, b);
  nb->sign = -nb->sign;
  o_add(P, r, a, nb);
}

/* ---------------- wide (exact-product) terms ---------------- */
/* A normalised exact term: value = sign * M * 2^(exp - 64*WN), MSB of M set
 * (cu_wterm, cu_fcomplex.cuh:25-28). */
typedef struct {
  int sign;
  int zero;
  long exp;
  int WN;
  u64 M[2 * ORC_MAXN64];
} wterm_t;

/* exact a*b as a normalised wide term (cu_mk_term, cu_fcomplex.cuh:30-42) */
static void mk_term(int P, wterm_t *t, const elem_t *a, const elem_t *b) {
  const int N = n64_of(P);
  t->WN = 2 * N;
  if (is_zero(a) || is_zero(b)) {
    t->zero = 1;
    t->sign = 1;
    t->exp = 0;
    memset(t->M, 0, sizeof(u64) * 2 * N);
    return;
  }
  t->zero = 0;
  t->sign = a->sign * b->sign;
  mul_exact(N, t->M, a->m, b->m);
  if (t->M[2 * N - 1] >> 63) {
    t->exp = a->exp + b->exp;
  } else {
    for (int i = 2 * N - 1; i > 0; i--) t->M[i] = (t->M[i] << 1) | (t->M[i - 1] >> 63);
    t->M[0] <<= 1;
    t->exp = a->exp + b->exp - 1;
  }
}
/* a plain element as a wide term (exact; the low N limbs are zero) */
static void elem_term(int P, wterm_t *t, const elem_t *c) {
  const int N = n64_of(P);
  t->WN = 2 * N;
  memset(t->M, 0, sizeof(u64) * 2 * N);
  if (is_zero(c)) {
    t->zero = 1;
    t->sign = 1;
    t->exp = 0;
    return;
  }
  t->zero = 0;
  t->sign = c->sign;
  t->exp = c->exp;
  memcpy(t->M + N, c->m, sizeof(u64) * N);
}
static int wterm_cmp(const wterm_t *a, const wterm_t *b) {
  if (a->exp != b->exp) return a->exp > b->exp ? 1 : -1;
  for (int i = a->WN - 1; i >= 0; i--)
    if (a->M[i] != b->M[i]) return a->M[i] > b->M[i] ? 1 : -1;
  return 0;
}

/* r = round(A + B), one rounding of the exact sum of two wide terms
 * (cu_round_sum2, cu_fcomplex.cuh:53-88): order by magnitude, place the larger
 * at limbs [2, WN+2) of a WN+3 limb buffer (2 guard limbs + carry limb), align
 * the smaller with sticky, add or subtract (same borrow-by-sticky rule as
 * submag), then round once. */
static void round_sum2(int P, elem_t *r, const wterm_t *A0, const wterm_t *B0) {
  const wterm_t *A = A0, *B = B0;
  const int WN = A->WN, WB = WN + 3;
  if (A->zero && B->zero) {
    set_zero(P, r);
    return;
  }
  if (A->zero) {
    round_into(P, r, B->M, WN, 64L * WN - 1, B->exp - 1, 0, 0, B->sign);
    return;
  }
  if (B->zero) {
    round_into(P, r, A->M, WN, 64L * WN - 1, A->exp - 1, 0, 0, A->sign);
    return;
  }
  if (wterm_cmp(A, B) < 0) {
    const wterm_t *t = A;
    A = B;
    B = t;
  }
  long d = A->exp - B->exp;
  u64 AB[2 * ORC_MAXN64 + 3], T[2 * ORC_MAXN64 + 3], BB[2 * ORC_MAXN64 + 3], D[2 * ORC_MAXN64 + 3];
  memset(AB, 0, sizeof(u64) * WB);
  memset(T, 0, sizeof(u64) * WB);
  for (int i = 0; i < WN; i++) {
    AB[i + 2] = A->M[i];
    T[i + 2] = B->M[i];
  }
  u64 st;
  if (d < 64L * WB) {
    st = any_below(T, WB, d);
    for (int i = 0; i < WB; i++) BB[i] = bits64_at(T, WB, d + 64L * i);
  } else {
    st = 1;
    memset(BB, 0, sizeof(u64) * WB);
  }
  if (A->sign == B->sign) {
    u64 c = 0;
    for (int i = 0; i < WB; i++) {
      u128 s = (u128)AB[i] + BB[i] + c;
      D[i] = (u64)s;
      c = (u64)(s >> 64);
    }
  } else {
    u64 br = 0;
    for (int i = 0; i < WB; i++) {
      u128 s = (u128)AB[i] - BB[i] - br;
      D[i] = (u64)s;
      br = (u64)(s >> 64) & 1;
    }
    if (st) {
      for (int i = 0; i < WB; i++) {
        u64 old = D[i];
        D[i] = old - 1;
        if (old != 0) break;
      }
    }
  }
  long msb = top_bit(D, WB);
  if (msb < 0) {
    set_zero(P, r);
    return;
  }
  round_into(P, r, D, WB, msb, A->exp - 64L * (WN + 2) + msb, 0, st, A->sign);
}

/* round(a*b - c*d) and round(a*b + c*d)  (cu_fmms / cu_fmma, cu_fcomplex.cuh:91-96) */
static void o_fmms(int P, elem_t *r, const elem_t *a, const elem_t *b, const elem_t *c,
                   const elem_t *d) {
  wterm_t t1, t2;
  mk_term(P, &t1, a, b);
  mk_term(P, &t2, c, d);
  t2.sign = -t2.sign;
  round_sum2(P, r, &t1, &t2);
}
static void o_fmma(int P, elem_t *r, const elem_t *a, const elem_t *b, const elem_t *c,
                   const elem_t *d) {
  wterm_t t1, t2;
  mk_term(P, &t1, a, b);
  mk_term(P, &t2, c, d);
  round_sum2(P, r, &t1, &t2);
}
/* round(a*b + c), a single rounding (mpfr_fma semantics; the reference has no
 * fma -- the restatement reuses the exact two-term rounding of cu_round_sum2). */
static void o_fma(int P, elem_t *r, const elem_t *a, const elem_t *b, const elem_t *c) {
  wterm_t t1, t2;
  mk_term(P, &t1, a, b);
  elem_term(P, &t2, c);
  round_sum2(P, r, &t1, &t2);
}

/* complex: z = {re, im} consecutive elements */
#define RE(z) (z)
#define IM(z, esz) ((elem_t *)((char *)(z) + (esz)))
#define CIM(z, esz) ((const elem_t *)((const char *)(z) + (esz)))

/* MPC_RNDNN product (cu_cmul, cu_fcomplex.cuh:121-124) */
static void o_cmul(int P, elem_t *r, const elem_t *a, const elem_t *b) {
  size_t es = esz_of(P);
  o_fmms(P, RE(r), RE(a), RE(b), CIM(a, es), CIM(b, es));
  o_fmma(P, IM(r, es), RE(a), CIM(b, es), CIM(a, es), RE(b));
}
/* cu_cadd / cu_csub (cu_fcomplex.cuh:115-120) */
static void o_cadd(int P, elem_t *r, const elem_t *a, const elem_t *b) {
  size_t es = esz_of(P);
  o_add(P, RE(r), RE(a), RE(b));
  o_add(P, IM(r, es), CIM(a, es), CIM(b, es));
}
static void o_csub(int P, elem_t *r, const elem_t *a, const elem_t *b) {
  size_t es = esz_of(P);
  o_sub(P, RE(r), RE(a), RE(b));
  o_sub(P, IM(r, es), CIM(a, es), CIM(b, es));
}

/* ---------------- exact sums (single rounding) ---------------- */
/* Correctly rounded sum of nt exact wide terms (each value sign*M*2^(exp-64WN)),
 * rounded once to P bits.  This is the semantics of MPFR's mpfr_dot / mpfr_sum
 * (exact products, one rounding; mirrored on the device by the reference's
 * runtime port, src/mpfr_cuda/dot.c:27-61).  Implementation: a two's-complement
 * fixed-point accumulator wide enough for every term plus carry room. */
static void round_exact_sum(int P, elem_t *r, const wterm_t *t, long nt) {
  long emin = 0, emax = 0;
  int any = 0;
  for (long k = 0; k < nt; k++) {
    if (t[k].zero) continue;
    long lo = t[k].exp - 64L * t[k].WN, hi = t[k].exp;
    if (!any || lo < emin) emin = lo;
    if (!any || hi > emax) emax = hi;
    any = 1;
  }
  if (!any) {
    set_zero(P, r);
    return;
  }
  int carry_bits = 2;
  while ((1L << (carry_bits - 2)) < nt) carry_bits++;
  long width = emax - emin + carry_bits + 1;
  int L = (int)((width + 63) / 64) + 1;
  u64 *acc = (u64 *)calloc((size_t)L, sizeof(u64));
  for (long k = 0; k < nt; k++) {
    if (t[k].zero) continue;
    const int WN = t[k].WN;
    long off = t[k].exp - 64L * WN - emin; /* bit offset of the term's bit 0 */
    long w = off >> 6;
    int b = (int)(off & 63);
    /* shifted term, WN+1 limbs starting at limb w */
    if (t[k].sign > 0) {
      u64 c = 0;
      for (int i = 0; i <= WN; i++) {
        u64 lo = (i < WN) ? t[k].M[i] : 0, lo2 = (i > 0) ? t[k].M[i - 1] : 0;
        u64 v = b ? (lo << b) | (lo2 >> (64 - b)) : lo;
        u128 s = (u128)acc[w + i] + v + c;
        acc[w + i] = (u64)s;
        c = (u64)(s >> 64);
      }
      for (long j = w + WN + 1; j < L && c; j++) {
        acc[j] += 1;
        c = (acc[j] == 0);
      }
    } else {
      u64 br = 0;
      for (int i = 0; i <= WN; i++) {
        u64 lo = (i < WN) ? t[k].M[i] : 0, lo2 = (i > 0) ? t[k].M[i - 1] : 0;
        u64 v = b ? (lo << b) | (lo2 >> (64 - b)) : lo;
        u128 s = (u128)acc[w + i] - v - br;
        acc[w + i] = (u64)s;
        br = (u64)(s >> 64) & 1;
      }
      for (long j = w + WN + 1; j < L && br; j++) {
        br = (acc[j] == 0);
        acc[j] -= 1;
      }
    }
  }
  int sgn = 1;
  if (acc[L - 1] >> 63) { /* negative: take the magnitude */
    sgn = -1;
    u64 c = 1;
    for (int i = 0; i < L; i++) {
      u128 s = (u128)(~acc[i]) + c;
      acc[i] = (u64)s;
      c = (u64)(s >> 64);
    }
  }
  long msb = top_bit(acc, L);
  if (msb < 0)
    set_zero(P, r);
  else
    round_into(P, r, acc, L, msb, emin + msb, 0, 0, sgn);
  free(acc);
}

/* ================== exported: elementwise (restatement) ================== */
typedef void (*binop_t)(int, elem_t *, const elem_t *, const elem_t *);

static void run_binop(binop_t f, int P, long n, const void *A, const void *B, void *R,
                      size_t es) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) f(P, at(R, es, i), cat(A, es, i), cat(B, es, i));
}

size_t orc_elem_bytes(int P) { return esz_of(P); }
int orc_max_prec(void) { return 64 * ORC_MAXN64; }

void orc_mul(int P, long n, const void *A, const void *B, void *R) {
  run_binop(o_mul, P, n, A, B, R, esz_of(P));
}
void orc_add(int P, long n, const void *A, const void *B, void *R) {
  run_binop(o_add, P, n, A, B, R, esz_of(P));
}
void orc_sub(int P, long n, const void *A, const void *B, void *R) {
  run_binop(o_sub, P, n, A, B, R, esz_of(P));
}
void orc_fma(int P, long n, const void *A, const void *B, const void *C, void *R) {
  size_t es = esz_of(P);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) o_fma(P, at(R, es, i), cat(A, es, i), cat(B, es, i), cat(C, es, i));
}
void orc_cmul(int P, long n, const void *A, const void *B, void *R) {
  run_binop(o_cmul, P, n, A, B, R, 2 * esz_of(P));
}
void orc_cadd(int P, long n, const void *A, const void *B, void *R) {
  run_binop(o_cadd, P, n, A, B, R, 2 * esz_of(P));
}
void orc_csub(int P, long n, const void *A, const void *B, void *R) {
  run_binop(o_csub, P, n, A, B, R, 2 * esz_of(P));
}

/* Z[i] = round(round(a*X[i]) + Y[i])  (freal_axpy, demos/bench_3way.cu:44-50) */
void orc_axpy_r(int P, long n, const void *a, const void *X, const void *Y, void *Z) {
  size_t es = esz_of(P);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    u64 tb[2 + ORC_MAXN64];
    elem_t *t = (elem_t *)tb;
    o_mul(P, t, (const elem_t *)a, cat(X, es, i));
    o_add(P, at(Z, es, i), t, cat(Y, es, i));
  }
}
/* Z[i] = cadd(cmul(a, X[i]), Y[i])  (fcplx_axpy, demos/bench_3way.cu:51-59;
 * axpyc, tools/axpy_fast_complex.cu:32-40) */
void orc_axpy_c(int P, long n, const void *a, const void *X, const void *Y, void *Z) {
  size_t es = 2 * esz_of(P);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    u64 tb[2 * (2 + ORC_MAXN64)];
    elem_t *t = (elem_t *)tb;
    o_cmul(P, t, (const elem_t *)a, cat(X, es, i));
    o_cadd(P, at(Z, es, i), t, cat(Y, es, i));
  }
}

/* Row-major matrices, element strides lda/ldb/ldc.
 * Sequential-k dot with a rounding after every operation:
 *   acc = +0; for k: acc = round(acc + round(a_k * b_k))
 * (matvec_kernel / matmul_kernel, tools/linalg_fast.cu:37-68; host order
 * tools/linalg_fast.cu:71-83; demos/matmul_mpfr.cu:171-190). */
static void seq_dot_r(int P, elem_t *acc, const void *A, long sa, const void *B, long sb, long K) {
  size_t es = esz_of(P);
  u64 tb[2 + ORC_MAXN64], ab[2 + ORC_MAXN64];
  elem_t *t = (elem_t *)tb, *nacc = (elem_t *)ab;
  set_zero(P, acc);
  for (long k = 0; k < K; k++) {
    o_mul(P, t, cat(A, es, k * sa), cat(B, es, k * sb));
    o_add(P, nacc, acc, t);
    copy_elem(P, acc, nacc);
  }
}
/* complex: acc = cadd(acc, cmul(a_k, b_k))  (cdot_ij, demos/matmul_mpc.cu:39-57) */
static void seq_dot_c(int P, elem_t *acc, const void *A, long sa, const void *B, long sb, long K) {
  size_t es = 2 * esz_of(P);
  u64 tb[2 * (2 + ORC_MAXN64)], ab[2 * (2 + ORC_MAXN64)];
  elem_t *t = (elem_t *)tb, *nacc = (elem_t *)ab;
  set_zero(P, RE(acc));
  set_zero(P, IM(acc, esz_of(P)));
  for (long k = 0; k < K; k++) {
    o_cmul(P, t, cat(A, es, k * sa), cat(B, es, k * sb));
    o_cadd(P, nacc, acc, t);
    memcpy(acc, nacc, es);
  }
}

/* y_out[i] = round(dot_i + y_in[i]), dot_i the sequential-k row dot of A and x.
 * The reference matvec has no "+y" (tools/linalg_fast.cu:37-51); this engine
 * defines y = A.x + y as the rounded sequential dot followed by one rounded add. */
void orc_gemv_r(int P, long m, long n, const void *A, long lda, const void *x,
                const void *y_in, void *y_out) {
  size_t es = esz_of(P);
#pragma omp parallel for schedule(dynamic, 4)
  for (long i = 0; i < m; i++) {
    u64 ab[2 + ORC_MAXN64];
    elem_t *acc = (elem_t *)ab;
    seq_dot_r(P, acc, cat(A, es, i * lda), 1, x, 1, n);
    o_add(P, at(y_out, es, i), acc, cat(y_in, es, i));
  }
}
void orc_gemv_c(int P, long m, long n, const void *A, long lda, const void *x,
                const void *y_in, void *y_out) {
  size_t es = 2 * esz_of(P);
#pragma omp parallel for schedule(dynamic, 4)
  for (long i = 0; i < m; i++) {
    u64 ab[2 * (2 + ORC_MAXN64)];
    elem_t *acc = (elem_t *)ab;
    seq_dot_c(P, acc, cat(A, es, i * lda), 1, x, 1, n);
    o_cadd(P, at(y_out, es, i), acc, cat(y_in, es, i));
  }
}
/* C = A.B, sequential k, per-operation rounding; rows [r0, r1) only so that a
 * bounded sample of a large product can be timed. */
void orc_gemm_r(int P, long m, long n, long k, const void *A, long lda, const void *B,
                long ldb, void *C, long ldc, long r0, long r1) {
  size_t es = esz_of(P);
  if (r1 <= 0 || r1 > m) r1 = m;
#pragma omp parallel for collapse(2) schedule(dynamic, 16)
  for (long i = r0; i < r1; i++)
    for (long j = 0; j < n; j++)
      seq_dot_r(P, at(C, es, i * ldc + j), cat(A, es, i * lda), 1, cat(B, es, j), ldb, k);
  (void)m;
}
void orc_gemm_c(int P, long m, long n, long k, const void *A, long lda, const void *B,
                long ldb, void *C, long ldc, long r0, long r1) {
  size_t es = 2 * esz_of(P);
  if (r1 <= 0 || r1 > m) r1 = m;
#pragma omp parallel for collapse(2) schedule(dynamic, 16)
  for (long i = r0; i < r1; i++)
    for (long j = 0; j < n; j++)
      seq_dot_c(P, at(C, es, i * ldc + j), cat(A, es, i * lda), 1, cat(B, es, j), ldb, k);
}

/* C = A.B with every entry the correctly rounded exact dot product (one
 * rounding per entry; mpfr_dot semantics).  Precision P of the inputs, output
 * rounded to Pout bits (Pout >= P gives the "4*PB" ULP oracle). */
void orc_gemm_exact_r(int P, int Pout, long m, long n, long k, const void *A, long lda,
                      const void *B, long ldb, void *C, long ldc, long r0, long r1) {
  size_t es = esz_of(P), eo = esz_of(Pout);
  if (r1 <= 0 || r1 > m) r1 = m;
#pragma omp parallel
  {
    wterm_t *t = (wterm_t *)malloc(sizeof(wterm_t) * (size_t)(k > 0 ? k : 1));
#pragma omp for collapse(2) schedule(dynamic, 16)
    for (long i = r0; i < r1; i++)
      for (long j = 0; j < n; j++) {
        for (long q = 0; q < k; q++)
          mk_term(P, &t[q], cat(A, es, i * lda + q), cat(B, es, q * ldb + j));
        round_exact_sum(Pout, at(C, eo, i * ldc + j), t, k);
      }
    free(t);
  }
}
/* complex: each component rounded once (mpc_dot semantics,
 * src/mpc_cuda/dot.c:28-95):  re = sum(ar*br - ai*bi), im = sum(ar*bi + ai*br) */
void orc_gemm_exact_c(int P, int Pout, long m, long n, long k, const void *A, long lda,
                      const void *B, long ldb, void *C, long ldc, long r0, long r1) {
  size_t es = 2 * esz_of(P), e1 = esz_of(P), eo = 2 * esz_of(Pout);
  if (r1 <= 0 || r1 > m) r1 = m;
#pragma omp parallel
  {
    wterm_t *t = (wterm_t *)malloc(sizeof(wterm_t) * (size_t)(2 * (k > 0 ? k : 1)));
#pragma omp for collapse(2) schedule(dynamic, 16)
    for (long i = r0; i < r1; i++)
      for (long j = 0; j < n; j++) {
        elem_t *c = at(C, eo, i * ldc + j);
        for (long q = 0; q < k; q++) {
          const elem_t *a = cat(A, es, i * lda + q), *b = cat(B, es, q * ldb + j);
          mk_term(P, &t[2 * q], RE(a), RE(b));
          mk_term(P, &t[2 * q + 1], CIM(a, e1), CIM(b, e1));
          t[2 * q + 1].sign = -t[2 * q + 1].sign;
        }
        round_exact_sum(Pout, RE(c), t, 2 * k);
        for (long q = 0; q < k; q++) {
          const elem_t *a = cat(A, es, i * lda + q), *b = cat(B, es, q * ldb + j);
          mk_term(P, &t[2 * q], RE(a), CIM(b, e1));
          mk_term(P, &t[2 * q + 1], CIM(a, e1), RE(b));
        }
        round_exact_sum(Pout, IM(c, esz_of(Pout)), t, 2 * k);
      }
    free(t);
  }
}

/* Exact (lossless) re-rounding of an element to another precision
 * (cu_convert, cu_freal.cuh:316-323). */
void orc_convert(int Pto, int Pfrom, long n, const void *X, void *R) {
  size_t ef = esz_of(Pfrom), et = esz_of(Pto);
  const int Nf = n64_of(Pfrom);
  for (long i = 0; i < n; i++) {
    const elem_t *x = cat(X, ef, i);
    elem_t *r = at(R, et, i);
    if (is_zero(x))
      set_zero(Pto, r);
    else
      round_into(Pto, r, x->m, Nf, 64L * Nf - 1, x->exp - 1, 0, 0, x->sign);
  }
}

/* double -> element, exact for P >= 53 (from_double, cu_freal.cuh:141-149) */
void orc_from_double(int P, long n, const double *d, void *R) {
  size_t es = esz_of(P);
  for (long i = 0; i < n; i++) {
    elem_t *r = at(R, es, i);
    double v = d[i];
    if (v == 0.0) {
      set_zero(P, r);
      continue;
    }
    int sgn = v < 0 ? -1 : 1;
    if (v < 0) v = -v;
    int k;
    double f = __builtin_frexp(v, &k);
    u64 F = (u64)__builtin_ldexp(f, 53);
    round_into(P, r, &F, 1, 52, (long)k - 1, 0, 0, sgn);
  }
}

/* Element-wise equality with mpfr_equal_p semantics (+0 == -0).  Returns the
 * number of mismatching entries; first mismatch index in *first (or -1). */
long orc_count_mismatch(int P, long n, const void *X, const void *Y, long *first) {
  size_t es = esz_of(P);
  const int N = n64_of(P);
  long bad = 0;
  if (first) *first = -1;
  for (long i = 0; i < n; i++) {
    const elem_t *x = cat(X, es, i), *y = cat(Y, es, i);
    int zx = is_zero(x), zy = is_zero(y), eq;
    if (zx || zy)
      eq = zx && zy;
    else
      eq = x->sign == y->sign && x->exp == y->exp && !memcmp(x->m, y->m, 8 * (size_t)N);
    if (!eq) {
      if (first && *first < 0) *first = i;
      bad++;
    }
  }
  return bad;
}

/* ULP distance |x - y| / 2^(exp(y) - Px): the error of a Px-bit result x
 * against a reference y computed at Py >= Px bits, in units of the last place
 * of a Px-bit number with y's exponent.  Used for the exact GEMM's error
 * report against a 4*PB oracle.  Returns 1e300 when x is far off. */
double orc_ulp_err(int Px, const void *xp, int Py, const void *yp) {
  const elem_t *x = (const elem_t *)xp, *y = (const elem_t *)yp;
  const int Nx = n64_of(Px), Ny = n64_of(Py), L = Ny + 3;
  if (is_zero(y)) return is_zero(x) ? 0.0 : 1e300;
  /* common fixed point: LSB weight 2^(y.exp - 64*Ny - 64); y at limbs [1, Ny+1) */
  u64 X[ORC_MAXN64 + 3], Y[ORC_MAXN64 + 3], D[ORC_MAXN64 + 3];
  memset(X, 0, sizeof X);
  memset(Y, 0, sizeof Y);
  for (int i = 0; i < Ny; i++) Y[i + 1] = y->m[i];
  int sx = y->sign;
  if (!is_zero(x)) {
    long s = (x->exp - y->exp) + 64L * (Ny - Nx) + 64; /* left shift of x.M */
    if (s < 0 || s > 64L * (Ny + 1)) return 1e300;
    for (int i = 0; i < L; i++) X[i] = bits64_at(x->m, Nx, 64L * i - s);
    sx = x->sign;
  }
  if (sx == y->sign) {
    u64 br = 0;
    for (int i = 0; i < L; i++) {
      u128 s = (u128)X[i] - Y[i] - br;
      D[i] = (u64)s;
      br = (u64)(s >> 64) & 1;
    }
    if (br) { /* negative: negate */
      u64 c = 1;
      for (int i = 0; i < L; i++) {
        u128 s = (u128)(~D[i]) + c;
        D[i] = (u64)s;
        c = (u64)(s >> 64);
      }
    }
  } else {
    u64 c = 0;
    for (int i = 0; i < L; i++) {
      u128 s = (u128)X[i] + Y[i] + c;
      D[i] = (u64)s;
      c = (u64)(s >> 64);
    }
  }
  int t = L - 1;
  while (t > 0 && D[t] == 0) t--;
  /* top two limbs carry far more than double precision */
  double r = (double)D[t] * 18446744073709551616.0 + (t > 0 ? (double)D[t - 1] : 0.0);
  return __builtin_ldexp(r, (int)(64L * (t - 1) - (64L * Ny + 64 - Px)));
}

/* ================== seeded generators (reference test method) ================== */
/* xorshift64 step (tools/test_freal.cu:15, tools/axpy_fast1024.cu:362) */
static u64 xs_next(u64 *s) {
  u64 x = *s;
  x ^= x << 13;
  x ^= x >> 7;
  x ^= x << 17;
  return *s = x;
}
/* full-width random element with exponent in [-spread, spread]
 * (randf, tools/test_freal.cu:17-27) */
static void xs_elem(int P, elem_t *r, u64 *s, long spread) {
  const int N = n64_of(P), SB = 64 * N - P;
  r->sign = (xs_next(s) & 1) ? 1 : -1;
  r->pad = 0;
  for (int i = 0; i < N; i++) r->m[i] = xs_next(s);
  r->m[N - 1] |= ((u64)1) << 63;
  if (SB) r->m[0] &= ~((((u64)1) << SB) - 1);
  r->exp = (long)(xs_next(s) % (u64)(2 * spread + 1)) - spread;
}
/* M operand pairs: spread 40 for 3 of 4 pairs, PB+200 for every 4th
 * (tools/test_freal.cu:55).  Returns the advanced seed. */
u64 orc_gen_pairs_r(int P, long M, u64 seed, void *A, void *B) {
  size_t es = esz_of(P);
  for (long i = 0; i < M; i++) {
    long sp = (i & 3) ? 40 : P + 200;
    xs_elem(P, at(A, es, i), &seed, sp);
    xs_elem(P, at(B, es, i), &seed, sp);
  }
  return seed;
}
/* complex pairs: A.re, A.im, B.re, B.im in that order (tools/test_fcomplex.cu:55-57) */
u64 orc_gen_pairs_c(int P, long M, u64 seed, void *A, void *B) {
  size_t e1 = esz_of(P), es = 2 * e1;
  for (long i = 0; i < M; i++) {
    long sp = (i & 3) ? 40 : P + 200;
    elem_t *a = at(A, es, i), *b = at(B, es, i);
    xs_elem(P, RE(a), &seed, sp);
    xs_elem(P, IM(a, e1), &seed, sp);
    xs_elem(P, RE(b), &seed, sp);
    xs_elem(P, IM(b, e1), &seed, sp);
  }
  return seed;
}

/* ================== MPFR / MPC (system libraries) ================== */
const char *orc_mpfr_version(void) { return mpfr_get_version(); }
const char *orc_mpc_version(void) { return mpc_get_version(); }

/* wrap an element's limbs as an MPFR number (no copy) */
static void as_mpfr(int P, shim_mpfr_ptr x, const elem_t *e) {
  if (is_zero(e))
    mpfr_custom_init_set(x, SHIM_ZERO_KIND, 0, P, (void *)e->m);
  else
    mpfr_custom_init_set(x, e->sign < 0 ? -SHIM_REGULAR_KIND : SHIM_REGULAR_KIND, e->exp, P,
                         (void *)e->m);
}
/* bind an output element's limbs as an MPFR destination */
static void bind_out(int P, shim_mpfr_ptr x, elem_t *e) {
  mpfr_custom_init_set(x, SHIM_ZERO_KIND, 0, P, (void *)e->m);
}
/* after an MPFR op wrote into a bound destination, fill sign/exp */
static void finish_out(int P, elem_t *e, const shim_mpfr_struct *x, int *negzero) {
  if (mpfr_zero_p(x)) {
    if (negzero && mpfr_signbit(x)) (*negzero)++;
    set_zero(P, e);
  } else {
    e->sign = x->sign < 0 ? -1 : 1;
    e->pad = 0;
    e->exp = x->exp;
  }
}

/* copy a (regularly allocated) MPFR number of precision P into an element */
static void store_mpfr(int P, elem_t *e, const shim_mpfr_struct *x) {
  if (mpfr_zero_p(x)) {
    set_zero(P, e);
    return;
  }
  memcpy(e->m, x->d, 8 * (size_t)n64_of(P));
  e->sign = x->sign < 0 ? -1 : 1;
  e->pad = 0;
  e->exp = x->exp;
}

void mp_mul(int P, long n, const void *A, const void *B, void *R) {
  size_t es = esz_of(P);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    shim_mpfr_t a, b, r;
    as_mpfr(P, a, cat(A, es, i));
    as_mpfr(P, b, cat(B, es, i));
    bind_out(P, r, at(R, es, i));
    mpfr_mul(r, a, b, SHIM_RNDN);
    finish_out(P, at(R, es, i), r, 0);
  }
}
void mp_add(int P, long n, const void *A, const void *B, void *R) {
  size_t es = esz_of(P);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    shim_mpfr_t a, b, r;
    as_mpfr(P, a, cat(A, es, i));
    as_mpfr(P, b, cat(B, es, i));
    bind_out(P, r, at(R, es, i));
    mpfr_add(r, a, b, SHIM_RNDN);
    finish_out(P, at(R, es, i), r, 0);
  }
}
void mp_sub(int P, long n, const void *A, const void *B, void *R) {
  size_t es = esz_of(P);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    shim_mpfr_t a, b, r;
    as_mpfr(P, a, cat(A, es, i));
    as_mpfr(P, b, cat(B, es, i));
    bind_out(P, r, at(R, es, i));
    mpfr_sub(r, a, b, SHIM_RNDN);
    finish_out(P, at(R, es, i), r, 0);
  }
}
/* correctly rounded division and square root via the system MPFR (checker
 * for the engine's div / sqrt; the reference's cu_fdiv / cu_sqrt are
 * faithful only, cu_fmath.cuh:1-14, so MPFR is the specification) */
void mp_div(int P, long n, const void *A, const void *B, void *R) {
  size_t es = esz_of(P);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    shim_mpfr_t a, b, r;
    as_mpfr(P, a, cat(A, es, i));
    as_mpfr(P, b, cat(B, es, i));
    bind_out(P, r, at(R, es, i));
    mpfr_div(r, a, b, SHIM_RNDN);
    finish_out(P, at(R, es, i), r, 0);
  }
}
/* mpfr_exp / mpfr_log at precision Pout (the checker for the engine's
 * faithful exp / log: Pout = 4P measures the error in ULPs) */
typedef int (*mpfr_un_t)(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
static void mp_un(mpfr_un_t f, int P, int Pout, long n, const void *A, void *R) {
  size_t es = esz_of(P), eo = esz_of(Pout);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    shim_mpfr_t a, r;
    as_mpfr(P, a, cat(A, es, i));
    mpfr_init2(r, Pout);
    f(r, a, SHIM_RNDN);
    store_mpfr(Pout, at(R, eo, i), r);
    mpfr_clear(r);
  }
}
void mp_exp(int P, int Pout, long n, const void *A, void *R) { mp_un(mpfr_exp, P, Pout, n, A, R); }
void mp_log(int P, int Pout, long n, const void *A, void *R) { mp_un(mpfr_log, P, Pout, n, A, R); }

/* the real elementary functions at precision Pout, fn numbered as the
 * engine's MPB_FN_* (0 exp .. 13 cbrt unary; 14 pow(a, b), 15 atan2(a, b)):
 * the checker for the faithful drop-in cu_exp .. cu_pow of the reference's
 * cu_fmath.cuh (its tools/test_fmath.cu and test_fmath3.cu compare the same
 * functions with MPFR) */
typedef int (*mpfr_bin_t)(shim_mpfr_ptr, const shim_mpfr_struct *, const shim_mpfr_struct *, shim_rnd_t);
int mp_fn(int fn, int P, int Pout, long n, const void *A, const void *B, void *R) {
  static const mpfr_un_t un[14] = {mpfr_exp,  mpfr_log,  mpfr_expm1, mpfr_log1p, mpfr_sin,  mpfr_cos,  mpfr_tan,
                                   mpfr_atan, mpfr_sinh, mpfr_cosh,  mpfr_atanh, mpfr_asin, mpfr_acos, mpfr_cbrt};
  if (fn < 0 || fn > 15) return -1;
  if (fn < 14) {
    mp_un(un[fn], P, Pout, n, A, R);
    return 0;
  }
  const mpfr_bin_t f = fn == 14 ? mpfr_pow : mpfr_atan2;
  size_t es = esz_of(P), eo = esz_of(Pout);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    shim_mpfr_t a, b, r;
    as_mpfr(P, a, cat(A, es, i));
    as_mpfr(P, b, cat(B, es, i));
    mpfr_init2(r, Pout);
    f(r, a, b, SHIM_RNDN);
    store_mpfr(Pout, at(R, eo, i), r);
    mpfr_clear(r);
  }
  return 0;
}

/* a p-bit MPFR value into a P-bit element (p <= P): the significand in the
 * top limbs, zeros below */
static void store_mpfr_narrow(int P, elem_t *e, const shim_mpfr_struct *x) {
  if (mpfr_zero_p(x)) {
    set_zero(P, e);
    return;
  }
  int n = n64_of(P), nx = (int)((x->prec + 63) / 64);
  memset(e->m, 0, 8 * (size_t)n);
  memcpy(e->m + (n - nx), x->d, 8 * (size_t)nx);
  e->sign = x->sign < 0 ? -1 : 1;
  e->pad = 0;
  e->exp = x->exp;
}

/* op(a, b, c) rounded to nearest at precision p, operands and result in the
 * P-bit element format (op 0 mul, 1 add, 2 sub, 3 fma, 4 div, 5 sqrt): the
 * checker for the engine's runtime-precision arithmetic */
void mp_op_rp(int op, int p, int P, long n, const void *A, const void *B, const void *C, void *R) {
  size_t es = esz_of(P);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    shim_mpfr_t a, b, c, r;
    as_mpfr(P, a, cat(A, es, i));
    as_mpfr(P, b, cat(op == 5 ? A : B, es, i));
    as_mpfr(P, c, cat(op == 3 ? C : A, es, i));
    mpfr_init2(r, p);
    switch (op) {
      case 0: mpfr_mul(r, a, b, SHIM_RNDN); break;
      case 1: mpfr_add(r, a, b, SHIM_RNDN); break;
      case 2: mpfr_sub(r, a, b, SHIM_RNDN); break;
      case 3: mpfr_fma(r, a, b, c, SHIM_RNDN); break;
      case 4: mpfr_div(r, a, b, SHIM_RNDN); break;
      default: mpfr_sqrt(r, a, SHIM_RNDN);
    }
    store_mpfr_narrow(P, at(R, es, i), r);
    mpfr_clear(r);
  }
}

/* round(a / u) (mpfr_div_ui), and pi / ln 2 (which 0 / 1) at precision P */
void mp_div_ui(int P, long n, const void *A, unsigned long u, void *R) {
  size_t es = esz_of(P);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    shim_mpfr_t a, r;
    as_mpfr(P, a, cat(A, es, i));
    mpfr_init2(r, P);
    mpfr_div_ui(r, a, u, SHIM_RNDN);
    store_mpfr(P, at(R, es, i), r);
    mpfr_clear(r);
  }
}
void mp_const(int which, int P, void *R) {
  shim_mpfr_t r;
  mpfr_init2(r, P);
  if (which == 0)
    mpfr_const_pi(r, SHIM_RNDN);
  else
    mpfr_const_log2(r, SHIM_RNDN);
  store_mpfr(P, (elem_t *)R, r);
  mpfr_clear(r);
}

void mp_sqrt(int P, long n, const void *A, void *R) {
  size_t es = esz_of(P);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    shim_mpfr_t a, r;
    as_mpfr(P, a, cat(A, es, i));
    bind_out(P, r, at(R, es, i));
    mpfr_sqrt(r, a, SHIM_RNDN);
    finish_out(P, at(R, es, i), r, 0);
  }
}

void mp_fma(int P, long n, const void *A, const void *B, const void *C, void *R) {
  size_t es = esz_of(P);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    shim_mpfr_t a, b, c, r;
    as_mpfr(P, a, cat(A, es, i));
    as_mpfr(P, b, cat(B, es, i));
    as_mpfr(P, c, cat(C, es, i));
    bind_out(P, r, at(R, es, i));
    mpfr_fma(r, a, b, c, SHIM_RNDN);
    finish_out(P, at(R, es, i), r, 0);
  }
}

static void as_mpc(int P, shim_mpc_ptr z, const elem_t *e) {
  as_mpfr(P, z->re, RE(e));
  as_mpfr(P, z->im, CIM(e, esz_of(P)));
}
static void bind_out_c(int P, shim_mpc_ptr z, elem_t *e) {
  bind_out(P, z->re, RE(e));
  bind_out(P, z->im, IM(e, esz_of(P)));
}
static void finish_out_c(int P, elem_t *e, const shim_mpc_struct *z) {
  finish_out(P, RE(e), z->re, 0);
  finish_out(P, IM(e, esz_of(P)), z->im, 0);
}

typedef int (*mpc_binop_t)(shim_mpc_ptr, const shim_mpc_struct *, const shim_mpc_struct *, int);
static void mp_cbin(mpc_binop_t f, int P, long n, const void *A, const void *B, void *R) {
  size_t es = 2 * esz_of(P);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    shim_mpc_t a, b, r;
    as_mpc(P, a, cat(A, es, i));
    as_mpc(P, b, cat(B, es, i));
    bind_out_c(P, r, at(R, es, i));
    f(r, a, b, SHIM_MPC_RNDNN);
    finish_out_c(P, at(R, es, i), r);
  }
}
void mp_cmul(int P, long n, const void *A, const void *B, void *R) { mp_cbin(mpc_mul, P, n, A, B, R); }
void mp_cadd(int P, long n, const void *A, const void *B, void *R) { mp_cbin(mpc_add, P, n, A, B, R); }
void mp_csub(int P, long n, const void *A, const void *B, void *R) { mp_cbin(mpc_sub, P, n, A, B, R); }

/* complex fused multiply-add a*b + c, one rounding per component: the
 * system mpc_fma, and independently mpc_dot over ([a, c], [b, 1]); the
 * reference has no such operation (checker for the engine's cu_cfma) */
/* the complex elementary functions at precision Pout (each component
 * rounded to nearest, MPC_RNDNN), fn numbered as the engine's MPB_CFN_*
 * (0 exp, 1 log, 2 sqrt, 3 sin, 4 cos, 5 tan, 6 sinh, 7 cosh, 8 a / b): the
 * checker for the drop-in cu_cexp .. cu_cdiv of the reference's
 * cu_fcmath.cuh (its tools/test_fcmath.cu compares them with MPC) */
typedef int (*mpc_un_t)(shim_mpc_ptr, const shim_mpc_struct *, int);
int mp_cfn(int fn, int P, int Pout, long n, const void *A, const void *B, void *R) {
  static const mpc_un_t un[8] = {mpc_exp, mpc_log, mpc_sqrt, mpc_sin, mpc_cos, mpc_tan, mpc_sinh, mpc_cosh};
  if (fn < 0 || fn > 8) return -1;
  size_t es = 2 * esz_of(P), eo = 2 * esz_of(Pout);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    shim_mpc_t a, b, r;
    as_mpc(P, a, cat(A, es, i));
    mpc_init2(r, Pout);
    if (fn == 8) {
      as_mpc(P, b, cat(B, es, i));
      mpc_div(r, a, b, SHIM_MPC_RNDNN);
    } else {
      un[fn](r, a, SHIM_MPC_RNDNN);
    }
    store_mpfr(Pout, RE(at(R, eo, i)), r->re);
    store_mpfr(Pout, IM(at(R, eo, i), esz_of(Pout)), r->im);
    mpc_clear(r);
  }
  return 0;
}

void mp_cfma(int P, long n, const void *A, const void *B, const void *C, void *R) {
  size_t es = 2 * esz_of(P);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    shim_mpc_t a, b, c, r;
    as_mpc(P, a, cat(A, es, i));
    as_mpc(P, b, cat(B, es, i));
    as_mpc(P, c, cat(C, es, i));
    mpc_init2(r, P); /* an ordinary destination: the library may swap significands */
    mpc_fma(r, a, b, c, SHIM_MPC_RNDNN);
    store_mpfr(P, RE(at(R, es, i)), r->re);
    store_mpfr(P, IM(at(R, es, i), esz_of(P)), r->im);
    mpc_clear(r);
  }
}
void mp_cfma_dot(int P, long n, const void *A, const void *B, const void *C, void *R) {
  size_t es = 2 * esz_of(P);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    shim_mpc_t a, b, c, one, r;
    as_mpc(P, a, cat(A, es, i));
    as_mpc(P, b, cat(B, es, i));
    as_mpc(P, c, cat(C, es, i));
    mpc_init2(one, 64);
    mpfr_set_d(one->re, 1.0, SHIM_RNDN);
    mpfr_set_d(one->im, 0.0, SHIM_RNDN);
    mpc_init2(r, P);
    shim_mpc_ptr x[2] = {a, c}, y[2] = {b, one};
    mpc_dot(r, x, y, 2, SHIM_MPC_RNDNN);
    store_mpfr(P, RE(at(R, es, i)), r->re);
    store_mpfr(P, IM(at(R, es, i), esz_of(P)), r->im);
    mpc_clear(r);
    mpc_clear(one);
  }
}

/* real AXPY via MPFR, the call sequence of cpu_axpy_real
 * (demos/bench3_cpu.cpp:35-57: mul then add, RNDN, OpenMP static) with the
 * operands bound in place instead of mpfr_set_d.  Each thread owns its
 * temporaries; returns nothing (time it from the caller). */
void mp_axpy_r(int P, long n, const void *a, const void *X, const void *Y, void *Z) {
  size_t es = esz_of(P);
#pragma omp parallel
  {
    shim_mpfr_t ma, t;
    mpfr_init2(t, P);
    as_mpfr(P, ma, (const elem_t *)a);
#pragma omp for schedule(static)
    for (long i = 0; i < n; i++) {
      shim_mpfr_t x, y, r;
      as_mpfr(P, x, cat(X, es, i));
      as_mpfr(P, y, cat(Y, es, i));
      bind_out(P, r, at(Z, es, i));
      mpfr_mul(t, ma, x, SHIM_RNDN);
      mpfr_add(r, t, y, SHIM_RNDN);
      finish_out(P, at(Z, es, i), r, 0);
    }
    mpfr_clear(t);
  }
}
/* complex AXPY via MPC (cpu_axpy_cplx, demos/bench3_cpu.cpp:59-85) */
void mp_axpy_c(int P, long n, const void *a, const void *X, const void *Y, void *Z) {
  size_t es = 2 * esz_of(P);
#pragma omp parallel
  {
    shim_mpc_t ma, t;
    mpc_init2(t, P);
    as_mpc(P, ma, (const elem_t *)a);
#pragma omp for schedule(static)
    for (long i = 0; i < n; i++) {
      shim_mpc_t x, y, r;
      as_mpc(P, x, cat(X, es, i));
      as_mpc(P, y, cat(Y, es, i));
      bind_out_c(P, r, at(Z, es, i));
      mpc_mul(t, ma, x, SHIM_MPC_RNDNN);
      mpc_add(r, t, y, SHIM_MPC_RNDNN);
      finish_out_c(P, at(Z, es, i), r);
    }
    mpc_clear(t);
  }
}

/* per-op-rounded sequential dot via MPFR (tools/linalg_fast.cu:71-83) */
static void mp_seq_dot_r(int P, elem_t *out, const void *A, long sa, const void *B, long sb,
                         long K, const elem_t *yadd) {
  size_t es = esz_of(P);
  shim_mpfr_t acc, t, r;
  mpfr_init2(acc, P);
  mpfr_init2(t, P);
  mpfr_set_zero(acc, 1);
  for (long k = 0; k < K; k++) {
    shim_mpfr_t a, b;
    as_mpfr(P, a, cat(A, es, k * sa));
    as_mpfr(P, b, cat(B, es, k * sb));
    mpfr_mul(t, a, b, SHIM_RNDN);
    mpfr_add(acc, acc, t, SHIM_RNDN);
  }
  bind_out(P, r, out);
  if (yadd) {
    shim_mpfr_t y;
    as_mpfr(P, y, yadd);
    mpfr_add(r, acc, y, SHIM_RNDN);
  } else {
    mpfr_set(r, acc, SHIM_RNDN);
  }
  finish_out(P, out, r, 0);
  mpfr_clear(acc);
  mpfr_clear(t);
}
static void mp_seq_dot_c(int P, elem_t *out, const void *A, long sa, const void *B, long sb,
                         long K, const elem_t *yadd) {
  size_t es = 2 * esz_of(P);
  shim_mpc_t acc, t, r;
  mpc_init2(acc, P);
  mpc_init2(t, P);
  mpfr_set_zero(acc->re, 1);
  mpfr_set_zero(acc->im, 1);
  for (long k = 0; k < K; k++) {
    shim_mpc_t a, b;
    as_mpc(P, a, cat(A, es, k * sa));
    as_mpc(P, b, cat(B, es, k * sb));
    mpc_mul(t, a, b, SHIM_MPC_RNDNN);
    mpc_add(acc, acc, t, SHIM_MPC_RNDNN);
  }
  bind_out_c(P, r, out);
  if (yadd) {
    shim_mpc_t y;
    as_mpc(P, y, yadd);
    mpc_add(r, acc, y, SHIM_MPC_RNDNN);
  } else {
    mpfr_set(r->re, acc->re, SHIM_RNDN);
    mpfr_set(r->im, acc->im, SHIM_RNDN);
  }
  finish_out_c(P, out, r);
  mpc_clear(acc);
  mpc_clear(t);
}
void mp_gemv_r(int P, long m, long n, const void *A, long lda, const void *x, const void *y_in,
               void *y_out) {
  size_t es = esz_of(P);
#pragma omp parallel for schedule(dynamic, 4)
  for (long i = 0; i < m; i++)
    mp_seq_dot_r(P, at(y_out, es, i), cat(A, es, i * lda), 1, x, 1, n, cat(y_in, es, i));
}
void mp_gemv_c(int P, long m, long n, const void *A, long lda, const void *x, const void *y_in,
               void *y_out) {
  size_t es = 2 * esz_of(P);
#pragma omp parallel for schedule(dynamic, 4)
  for (long i = 0; i < m; i++)
    mp_seq_dot_c(P, at(y_out, es, i), cat(A, es, i * lda), 1, x, 1, n, cat(y_in, es, i));
}
void mp_gemm_r(int P, long m, long n, long k, const void *A, long lda, const void *B, long ldb,
               void *C, long ldc, long r0, long r1) {
  size_t es = esz_of(P);
  if (r1 <= 0 || r1 > m) r1 = m;
#pragma omp parallel for collapse(2) schedule(dynamic, 16)
  for (long i = r0; i < r1; i++)
    for (long j = 0; j < n; j++)
      mp_seq_dot_r(P, at(C, es, i * ldc + j), cat(A, es, i * lda), 1, cat(B, es, j), ldb, k, 0);
}
void mp_gemm_c(int P, long m, long n, long k, const void *A, long lda, const void *B, long ldb,
               void *C, long ldc, long r0, long r1) {
  size_t es = 2 * esz_of(P);
  if (r1 <= 0 || r1 > m) r1 = m;
#pragma omp parallel for collapse(2) schedule(dynamic, 16)
  for (long i = r0; i < r1; i++)
    for (long j = 0; j < n; j++)
      mp_seq_dot_c(P, at(C, es, i * ldc + j), cat(A, es, i * lda), 1, cat(B, es, j), ldb, k, 0);
}
/* correctly rounded dot via the system mpfr_dot, output at Pout bits */
void mp_gemm_exact_r(int P, int Pout, long m, long n, long k, const void *A, long lda,
                     const void *B, long ldb, void *C, long ldc, long r0, long r1) {
  size_t es = esz_of(P), eo = esz_of(Pout);
  if (r1 <= 0 || r1 > m) r1 = m;
#pragma omp parallel
  {
    shim_mpfr_struct *xa = (shim_mpfr_struct *)malloc(sizeof(shim_mpfr_struct) * (size_t)k);
    shim_mpfr_struct *xb = (shim_mpfr_struct *)malloc(sizeof(shim_mpfr_struct) * (size_t)k);
    shim_mpfr_ptr *pa = (shim_mpfr_ptr *)malloc(sizeof(shim_mpfr_ptr) * (size_t)k);
    shim_mpfr_ptr *pb = (shim_mpfr_ptr *)malloc(sizeof(shim_mpfr_ptr) * (size_t)k);
    /* mpfr_dot/mpc_dot may swap significands into the destination, so the
     * destination is an ordinary MPFR variable, copied out afterwards */
    shim_mpfr_t r;
    mpfr_init2(r, Pout);
#pragma omp for collapse(2) schedule(dynamic, 16)
    for (long i = r0; i < r1; i++)
      for (long j = 0; j < n; j++) {
        for (long q = 0; q < k; q++) {
          as_mpfr(P, &xa[q], cat(A, es, i * lda + q));
          as_mpfr(P, &xb[q], cat(B, es, q * ldb + j));
          pa[q] = &xa[q];
          pb[q] = &xb[q];
        }
        elem_t *c = at(C, eo, i * ldc + j);
        mpfr_dot(r, pa, pb, (unsigned long)k, SHIM_RNDN);
        store_mpfr(Pout, c, r);
      }
    mpfr_clear(r);
    free(xa);
    free(xb);
    free(pa);
    free(pb);
  }
}
/* correctly rounded complex dot via the system mpc_dot */
void mp_gemm_exact_c(int P, int Pout, long m, long n, long k, const void *A, long lda,
                     const void *B, long ldb, void *C, long ldc, long r0, long r1) {
  size_t es = 2 * esz_of(P), eo = 2 * esz_of(Pout);
  if (r1 <= 0 || r1 > m) r1 = m;
#pragma omp parallel
  {
    shim_mpc_struct *xa = (shim_mpc_struct *)malloc(sizeof(shim_mpc_struct) * (size_t)k);
    shim_mpc_struct *xb = (shim_mpc_struct *)malloc(sizeof(shim_mpc_struct) * (size_t)k);
    shim_mpc_ptr *pa = (shim_mpc_ptr *)malloc(sizeof(shim_mpc_ptr) * (size_t)k);
    shim_mpc_ptr *pb = (shim_mpc_ptr *)malloc(sizeof(shim_mpc_ptr) * (size_t)k);
    shim_mpc_t r;
    mpc_init2(r, Pout);
#pragma omp for collapse(2) schedule(dynamic, 16)
    for (long i = r0; i < r1; i++)
      for (long j = 0; j < n; j++) {
        for (long q = 0; q < k; q++) {
          as_mpc(P, &xa[q], cat(A, es, i * lda + q));
          as_mpc(P, &xb[q], cat(B, es, q * ldb + j));
          pa[q] = &xa[q];
          pb[q] = &xb[q];
        }
        elem_t *c = at(C, eo, i * ldc + j);
        mpc_dot(r, pa, pb, (unsigned long)k, SHIM_MPC_RNDNN);
        store_mpfr(Pout, RE(c), r->re);
        store_mpfr(Pout, IM(c, esz_of(Pout)), r->im);
      }
    mpc_clear(r);
    free(xa);
    free(xb);
    free(pa);
    free(pb);
  }
}

int orc_num_threads(void) {
#ifdef _OPENMP
  extern int omp_get_max_threads(void);
  return omp_get_max_threads();
#else
  return 1;
#endif
}
