"""Seeded synthetic operands for the engine's benchmark workloads.

Every generator returns ``(limbs, heads)``: ``limbs`` is an ``(n, prec/32)``
uint32 array (little-endian, left-justified significands, top bit set) and
``heads`` the packed ``(exp << 1) | negative`` words (``0x80000000`` = zero),
which ``layout.vec_from_parts`` / ``layout.aos_from_parts`` turn into device
tiles or mpc_cuda AoS structs.

Workloads (sizes and value distributions of the engine's benchmark configs):
  axpy_r256   real AXPY, PB=256, n=2^20, a=1.5, x,y FP64 uniform in [-1,1)
  axpy_c1024  complex AXPY, PB=1024, n=2^18, full random 1024-bit parts,
              exponents U[-32,32], 1% exact zeros, random signs
  gemm_r512   real 1024^3 matmul, PB=512, 16 random limbs, exponents U[-16,16]
  gemv_batch  4096 GEMV problems, m,n log-uniform [16,512], PB uniform in
              {64..2048}, exponents U[-24,24]
  gemm_c256   complex 512^3 matmul, PB=256, 8 random limbs, exponents U[-8,8]
"""
from __future__ import annotations

import numpy as np

from .layout import HEAD_ZERO, nlimbs


def pack_heads(exp: np.ndarray, neg: np.ndarray) -> np.ndarray:
    return (((exp.astype(np.int64) << 1) & 0xFFFFFFFF) | neg.astype(np.int64)).astype(np.uint32)


def random_elems(rng: np.random.Generator, prec: int, n: int, exp_lo: int, exp_hi: int,
                 zero_frac: float = 0.0):
    """Full-width random significands (all prec bits random, top bit set),
    random sign, exponent uniform in [exp_lo, exp_hi], a fraction of exact zeros."""
    N = nlimbs(prec)
    limbs = rng.integers(0, 2**32, size=(n, N), dtype=np.uint32)
    limbs[:, N - 1] |= np.uint32(0x80000000)
    neg = rng.integers(0, 2, size=n)
    exp = rng.integers(exp_lo, exp_hi + 1, size=n)
    heads = pack_heads(exp, neg)
    if zero_frac > 0:
        z = rng.random(n) < zero_frac
        heads[z] = HEAD_ZERO
        limbs[z] = 0
    return limbs, heads


def from_doubles(prec: int, d: np.ndarray):
    """Exact conversion of doubles (prec >= 64 holds all 53 bits)."""
    d = np.asarray(d, dtype=np.float64)
    N = nlimbs(prec)
    n = d.shape[0]
    f, k = np.frexp(np.abs(d))
    F = np.ldexp(f, 53).astype(np.uint64)
    limbs = np.zeros((n, N), dtype=np.uint32)
    limbs[:, N - 1] = (F >> np.uint64(21)).astype(np.uint32)
    limbs[:, N - 2] = ((F << np.uint64(11)) & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    heads = pack_heads(k, d < 0)
    z = d == 0
    heads[z] = HEAD_ZERO
    limbs[z] = 0
    return limbs, heads


def axpy_r256(seed: int = 0x5EED1, n: int = 1 << 20, prec: int = 256):
    rng = np.random.default_rng(seed)
    a = from_doubles(prec, np.array([1.5]))
    x = from_doubles(prec, rng.uniform(-1.0, 1.0, n))
    y = from_doubles(prec, rng.uniform(-1.0, 1.0, n))
    return a, x, y


def axpy_c1024(seed: int = 0x5EED2, n: int = 1 << 18, prec: int = 1024):
    """Complex operands as (re, im) pairs of (limbs, heads)."""
    rng = np.random.default_rng(seed)

    def cvec(m):
        re = random_elems(rng, prec, m, -32, 32, 0.01)
        im = random_elems(rng, prec, m, -32, 32, 0.01)
        return re, im

    return cvec(1), cvec(n), cvec(n)


def gemm_r512(seed: int = 0x5EED3, m: int = 1024, n: int = 1024, k: int = 1024, prec: int = 512):
    rng = np.random.default_rng(seed)
    return random_elems(rng, prec, m * k, -16, 16), random_elems(rng, prec, k * n, -16, 16)


def gemm_c256(seed: int = 0x5EED5, m: int = 512, n: int = 512, k: int = 512, prec: int = 256):
    rng = np.random.default_rng(seed)

    def cmat(cnt):
        return random_elems(rng, prec, cnt, -8, 8), random_elems(rng, prec, cnt, -8, 8)

    return cmat(m * k), cmat(k * n)


def gemv_batch_shapes(seed: int = 0x5EED4, count: int = 4096):
    """(m, n, prec) per problem: m, n log-uniform in [16, 512], prec uniform."""
    rng = np.random.default_rng(seed)
    m = np.exp(rng.uniform(np.log(16), np.log(512), count)).round().astype(int)
    n = np.exp(rng.uniform(np.log(16), np.log(512), count)).round().astype(int)
    prec = rng.choice([64, 128, 256, 512, 1024, 2048], size=count)
    return np.clip(m, 16, 512), np.clip(n, 16, 512), prec


def _round32(v):
    return -(-np.asarray(v, dtype=np.int64) // 32) * 32


def gemv_batch(seed: int = 0x5EED4, count: int = 4096, shapes=None, exp_lo: int = -24, exp_hi: int = 24):
    """The batched GEMV workload, generated one precision group at a time.

    Returns ``(problems, pools)``.  ``problems[i]`` is a dict with ``prec, m,
    n, lda`` (``lda`` = n rounded up to 32) and element offsets ``a_off,
    x_off, y_off`` into its precision's pools; every offset is a multiple of
    32, so each operand starts on a tile boundary of the device layout.
    ``pools[prec]`` holds ``A``, ``x``, ``y`` as ``(limbs, heads)`` with the
    padding columns of A and the tails of x and y set to exact zeros.
    """
    m, n, prec = shapes if shapes is not None else gemv_batch_shapes(seed, count)
    m, n, prec = np.asarray(m), np.asarray(n), np.asarray(prec)
    rng = np.random.default_rng(seed ^ 0xB47C)
    problems = [None] * len(m)
    pools = {}
    for p in sorted(set(int(v) for v in prec)):
        idx = np.nonzero(prec == p)[0]
        lda = np.maximum(32, _round32(n[idx]))
        a_sz, x_sz, y_sz = m[idx] * lda, _round32(n[idx]), _round32(m[idx])
        a_off = np.concatenate([[0], np.cumsum(a_sz)[:-1]])
        x_off = np.concatenate([[0], np.cumsum(x_sz)[:-1]])
        y_off = np.concatenate([[0], np.cumsum(y_sz)[:-1]])
        A = random_elems(rng, p, int(a_sz.sum()), exp_lo, exp_hi)
        x = random_elems(rng, p, int(x_sz.sum()), exp_lo, exp_hi)
        y = random_elems(rng, p, int(y_sz.sum()), exp_lo, exp_hi)
        a_pad = np.concatenate([np.tile(np.arange(ld) >= c, r) for r, c, ld in zip(m[idx], n[idx], lda)])
        x_pad = np.concatenate([np.arange(s) >= c for c, s in zip(n[idx], x_sz)])
        y_pad = np.concatenate([np.arange(s) >= r for r, s in zip(m[idx], y_sz)])
        for (limbs, heads), pad in ((A, a_pad), (x, x_pad), (y, y_pad)):
            limbs[pad] = 0
            heads[pad] = HEAD_ZERO
        pools[p] = dict(A=A, x=x, y=y)
        for j, i in enumerate(idx):
            problems[i] = dict(prec=p, m=int(m[i]), n=int(n[i]), lda=int(lda[j]), a_off=int(a_off[j]),
                               x_off=int(x_off[j]), y_off=int(y_off[j]))
    return problems, pools


def gemv_batch_problem(pools, pr):
    """One problem's operands ``(A, x, y)`` as (limbs, heads), A dense m x n."""
    P, m, n, lda = pools[pr["prec"]], pr["m"], pr["n"], pr["lda"]
    la, ha = P["A"]
    sel = slice(pr["a_off"], pr["a_off"] + m * lda)
    A = (la[sel].reshape(m, lda, -1)[:, :n].reshape(m * n, -1), ha[sel].reshape(m, lda)[:, :n].reshape(-1))
    xs, ys = slice(pr["x_off"], pr["x_off"] + n), slice(pr["y_off"], pr["y_off"] + m)
    return A, (P["x"][0][xs], P["x"][1][xs]), (P["y"][0][ys], P["y"][1][ys])


def interleave_complex(prec: int, re, im):
    """(re parts, im parts) -> complex AoS bytes of cu_fcomplex<prec>."""
    from .layout import aos_from_parts

    return np.concatenate([aos_from_parts(prec, *re), aos_from_parts(prec, *im)], axis=1)
