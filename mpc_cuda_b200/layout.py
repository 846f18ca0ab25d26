"""Host-side (numpy) conversions between the mpc_cuda AoS element structs and
the engine's tiled HBM layout.

AoS ``cu_fp::cu_freal<prec>`` (mpc_cuda include/mpc_cuda/cu_freal.cuh:67-81)::

    int32 sign; int32 pad; int64 exp; uint64 m[prec/64]      # 16 + prec/8 bytes
    value = sign * M * 2^(exp - prec), zero <=> exp == -0x7fffffffffffff

``cu_fcomplex<prec>`` is ``{re, im}``.  Tiled layout (include/mpb/layout.cuh):
per 32 elements ``[prec/32/V groups][32 elements][V limbs]`` uint32 limbs,
``V = min(4, prec/32)``, then 32 uint32 heads ``(exp << 1) | negative``
(``0x80000000`` = zero).  Complex vectors interleave ``[re tile][im tile]``.
"""
from __future__ import annotations

import numpy as np

AOS_ZERO_EXP = -0x7FFFFFFFFFFFFF
HEAD_ZERO = 0x80000000
SUPPORTED = (64, 128, 256, 512, 1024, 2048)


def nlimbs(prec: int) -> int:
    return prec // 32


def aos_bytes(prec: int) -> int:
    return 16 + 8 * ((prec + 63) // 64)


def tile_bytes(prec: int) -> int:
    return 128 * (nlimbs(prec) + 1)


def vec_bytes(prec: int, n: int, cplx: bool = False) -> int:
    return (2 if cplx else 1) * ((n + 31) // 32) * tile_bytes(prec)


def _check(prec: int):
    if prec not in SUPPORTED:
        raise ValueError(f"unsupported precision {prec}; use one of {SUPPORTED}")


def _aos_fields(prec: int, aos: np.ndarray):
    es = aos_bytes(prec)
    a = np.ascontiguousarray(aos, dtype=np.uint8).reshape(-1, es)
    sign = a[:, 0:4].copy().view(np.int32)[:, 0]
    exp = a[:, 8:16].copy().view(np.int64)[:, 0]
    limbs = a[:, 16:].copy().view(np.uint32)
    return sign, exp, limbs


def _heads(sign, exp):
    zero = exp == AOS_ZERO_EXP
    e = exp.astype(np.int64)
    h = ((e.astype(np.int64) << 1) & 0xFFFFFFFF) | (sign < 0).astype(np.int64)
    h = np.where(zero, HEAD_ZERO, h).astype(np.uint32)
    return h, zero


def _tiles_from(prec: int, limbs: np.ndarray, heads: np.ndarray) -> np.ndarray:
    N = nlimbs(prec)
    V = min(4, N)
    G = N // V
    n = limbs.shape[0]
    T = (n + 31) // 32
    L = np.zeros((T * 32, N), dtype=np.uint32)
    L[:n] = limbs
    H = np.full(T * 32, HEAD_ZERO, dtype=np.uint32)
    H[:n] = heads
    L = L.reshape(T, 32, G, V).transpose(0, 2, 1, 3).reshape(T, 32 * N)
    return np.concatenate([L, H.reshape(T, 32)], axis=1)  # (T, tile words)


def _from_tiles(prec: int, tiles: np.ndarray, n: int):
    N = nlimbs(prec)
    V = min(4, N)
    G = N // V
    T = tiles.shape[0]
    L = tiles[:, : 32 * N].reshape(T, G, 32, V).transpose(0, 2, 1, 3).reshape(T * 32, N)[:n]
    H = tiles[:, 32 * N:].reshape(T * 32)[:n]
    return L, H


def aos_to_vec(prec: int, aos: np.ndarray, cplx: bool = False) -> np.ndarray:
    """AoS cu_freal/cu_fcomplex array (uint8, n x struct bytes) -> tiled bytes."""
    _check(prec)
    es = aos_bytes(prec)
    a = np.ascontiguousarray(aos, dtype=np.uint8).reshape(-1, (2 if cplx else 1) * es)
    if not cplx:
        sign, exp, limbs = _aos_fields(prec, a)
        h, zero = _heads(sign, exp)
        limbs = np.where(zero[:, None], 0, limbs).astype(np.uint32)
        return _tiles_from(prec, limbs, h).view(np.uint8).reshape(-1)
    parts = []
    for half in (a[:, :es], a[:, es:]):
        sign, exp, limbs = _aos_fields(prec, half)
        h, zero = _heads(sign, exp)
        limbs = np.where(zero[:, None], 0, limbs).astype(np.uint32)
        parts.append(_tiles_from(prec, limbs, h))
    T = parts[0].shape[0]
    return np.stack(parts, axis=1).reshape(T, -1).view(np.uint8).reshape(-1)


def vec_to_aos(prec: int, vec: np.ndarray, n: int, cplx: bool = False) -> np.ndarray:
    """Tiled bytes -> AoS array (n x struct bytes, uint8); zero -> sign +1."""
    _check(prec)
    N = nlimbs(prec)
    T = (n + 31) // 32
    words = np.ascontiguousarray(vec, dtype=np.uint8)[: vec_bytes(prec, n, cplx)].view(np.uint32)
    tw = tile_bytes(prec) // 4
    halves = [words.reshape(T, tw)] if not cplx else list(words.reshape(T, 2, tw).transpose(1, 0, 2))
    outs = []
    for tiles in halves:
        L, H = _from_tiles(prec, np.ascontiguousarray(tiles), n)
        zero = H == HEAD_ZERO
        e = (H.view(np.int32) >> 1).astype(np.int64)
        s = np.where((H & 1) == 1, -1, 1).astype(np.int32)
        out = np.zeros((n, aos_bytes(prec)), dtype=np.uint8)
        out[:, 0:4] = np.where(zero, 1, s).astype(np.int32).view(np.uint8).reshape(n, 4)
        out[:, 8:16] = np.where(zero, AOS_ZERO_EXP, e).astype(np.int64).view(np.uint8).reshape(n, 8)
        out[:, 16:] = np.where(zero[:, None], 0, L).astype(np.uint32).view(np.uint8).reshape(n, 4 * N)
        outs.append(out)
    return outs[0] if not cplx else np.concatenate(outs, axis=1)


def vec_from_parts(prec: int, limbs: np.ndarray, heads: np.ndarray) -> np.ndarray:
    """(n, prec/32) uint32 limbs + n uint32 heads -> tiled bytes (real)."""
    _check(prec)
    return _tiles_from(prec, limbs.astype(np.uint32), heads.astype(np.uint32)).view(np.uint8).reshape(-1)


def aos_from_parts(prec: int, limbs: np.ndarray, heads: np.ndarray) -> np.ndarray:
    """(n, prec/32) uint32 limbs + n uint32 heads -> AoS cu_freal<prec> bytes."""
    _check(prec)
    n, N = limbs.shape
    heads = heads.astype(np.uint32)
    zero = heads == HEAD_ZERO
    e = (heads.view(np.int32) >> 1).astype(np.int64)
    s = np.where((heads & 1) == 1, -1, 1).astype(np.int32)
    out = np.zeros((n, aos_bytes(prec)), dtype=np.uint8)
    out[:, 0:4] = np.where(zero, 1, s).astype(np.int32).view(np.uint8).reshape(n, 4)
    out[:, 8:16] = np.where(zero, AOS_ZERO_EXP, e).astype(np.int64).view(np.uint8).reshape(n, 8)
    out[:, 16:] = np.where(zero[:, None], 0, limbs).astype(np.uint32).view(np.uint8).reshape(n, 4 * N)
    return out


def parts_from_aos(prec: int, aos: np.ndarray):
    """AoS cu_freal<prec> bytes -> ((n, prec/32) uint32 limbs, n uint32 heads)."""
    _check(prec)
    sign, exp, limbs = _aos_fields(prec, aos)
    h, zero = _heads(sign, exp)
    return np.where(zero[:, None], 0, limbs).astype(np.uint32), h
