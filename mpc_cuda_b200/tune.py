"""Autotuning of the choices the library leaves open, with a JSON cache.

Three choices are tuned per precision and problem shape:

* the thread-vs-warp split (``mpb_set_split``) of the kernels that have a
  warp-cooperative form -- lanes per GEMV row and per complex AXPY element at
  1024 and 2048 bits (results are identical for every split; only the speed
  differs).  ``autotune_split`` times every split the library offers on
  operands of the given shape and installs the fastest;
* the block shape of the plain GEMM (``mpb_set_gemm_warps``: 4, 8 or 16 rows
  of C per block) -- ``autotune_gemm_warps`` times the three on the problem;
* the launch shape and split of each precision group of a batched GEMV
  (``BatchGemv.autotune`` in C; ``save_batch`` / ``apply_batch`` keep the
  choice under a signature of the batch).

The cache is a JSON object ``{"split": {"<kind>/<prec>/<bucket>": lanes},
"gemm_warps": {"gemm_r|gemm_c/<prec>/<bucket>": warps},
"batch": {"<signature>": {"<prec>": [block, blocks_per_sm, lanes]}}}``.  A
shape bucket is the power-of-two class of the row count and of the dot length
(the split's benefit depends on how many rows share the GPU and on the length
of each row's sequential chain), so one entry serves nearby shapes.
"""
from __future__ import annotations

import json
import math
import os

from . import SPLIT_AXPY_C, SPLIT_GEMV_R, get_gemm_warps, get_split, set_gemm_warps, set_split

KINDS = {"axpy_c": SPLIT_AXPY_C, "gemv_r": SPLIT_GEMV_R}
SPLITS = {("gemv_r", 1024): (1, 4, 8), ("gemv_r", 2048): (1, 8, 16), ("axpy_c", 1024): (1, 4, 8)}
GEMM_WARPS = (4, 8, 16)


def bucket(rows: int, cols: int = 1) -> str:
    """power-of-two class of (rows, cols): 'r<2^a>c<2^b>'"""
    def p2(v):
        return 1 << max(0, math.ceil(math.log2(max(1, v))))

    return f"r{p2(rows)}c{p2(cols)}"


def key(kind: str, prec: int, rows: int, cols: int = 1) -> str:
    return f"{kind}/{prec}/{bucket(rows, cols)}"


class TuningCache:
    """The JSON cache of tuned choices (a plain dict on disk)."""

    def __init__(self, path: str | None = None):
        self.path = path
        self.data = {"split": {}, "gemm_warps": {}, "batch": {}}
        if path and os.path.exists(path):
            with open(path) as f:
                loaded = json.load(f)
            for sec in self.data:
                self.data[sec].update(loaded.get(sec, {}))

    def save(self, path: str | None = None) -> None:
        path = path or self.path
        if not path:
            raise ValueError("no cache path")
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)

    # ---- thread-vs-warp split ----
    def record_split(self, kind: str, prec: int, rows: int, cols: int, lanes: int) -> None:
        if lanes not in SPLITS.get((kind, prec), (1,)):
            raise ValueError(f"{kind} at {prec} bits offers no split of {lanes} lanes")
        self.data["split"][key(kind, prec, rows, cols)] = int(lanes)

    def lookup_split(self, kind: str, prec: int, rows: int, cols: int = 1):
        return self.data["split"].get(key(kind, prec, rows, cols))

    def apply_split(self, kind: str, prec: int, rows: int, cols: int = 1) -> int:
        """Install the cached split for this shape (if any); returns the split in force."""
        lanes = self.lookup_split(kind, prec, rows, cols)
        if lanes is not None:
            set_split(KINDS[kind], prec, lanes)
        return get_split(KINDS[kind], prec)

    # ---- plain GEMM block shape ----
    def record_gemm_warps(self, prec: int, m: int, n: int, warps: int, cplx: bool = False) -> None:
        if warps not in GEMM_WARPS:
            raise ValueError(f"the plain GEMM offers no block of {warps} warps")
        self.data["gemm_warps"][key("gemm_c" if cplx else "gemm_r", prec, m, n)] = int(warps)

    def lookup_gemm_warps(self, prec: int, m: int, n: int, cplx: bool = False):
        return self.data["gemm_warps"].get(key("gemm_c" if cplx else "gemm_r", prec, m, n))

    def apply_gemm_warps(self, prec: int, m: int, n: int, cplx: bool = False) -> int:
        """Install the cached block shape for this C shape (if any); returns the one in force."""
        w = self.lookup_gemm_warps(prec, m, n, cplx)
        if w is not None:
            set_gemm_warps(prec, w, cplx)
        return get_gemm_warps(prec, cplx)

    # ---- batched GEMV ----
    @staticmethod
    def batch_signature(problems) -> str:
        """(prec, m, n) multiset of a batch, summarised per precision: count and
        power-of-two classes of the total and the longest row"""
        per = {}
        for prec, m, n in problems:
            c, tot, longest = per.get(prec, (0, 0, 0))
            per[prec] = (c + 1, tot + m * n, max(longest, n))
        parts = [f"{p}:{c}:{bucket(tot)}:{bucket(longest)}" for p, (c, tot, longest) in sorted(per.items())]
        return "|".join(parts)

    def save_batch(self, signature: str, batch) -> None:
        tun, spl = batch.tuning(), batch.splits()
        self.data["batch"][signature] = {str(p): [int(tun[p][0]), int(tun[p][1]), int(spl[p])] for p in tun}

    def apply_batch(self, signature: str, batch) -> bool:
        """Install a cached choice on a planned batch; False when none is cached."""
        entry = self.data["batch"].get(signature)
        if not entry:
            return False
        for p, (block, bps, lanes) in entry.items():
            batch.set_tuning({int(p): (block, bps)})
            batch.set_split(int(p), lanes)
        return True


def autotune_split(kind: str, prec: int, rows: int, cols: int = 1, reps: int = 3, cache: TuningCache | None = None,
                   seed: int = 0x7E57):
    """Time every split `kind` offers at `prec` on random operands of the shape
    (GEMV: rows x cols; complex AXPY: rows elements), install the fastest and
    record it in `cache`.  Returns {lanes: ms}."""
    import numpy as np
    import torch

    from . import axpy, empty, gemv
    from . import layout, synth

    splits = SPLITS.get((kind, prec))
    if not splits:
        return {get_split(KINDS[kind], prec): 0.0}
    rng = np.random.default_rng(seed)

    def vec(n, cplx=False):
        if cplx:
            re, im = synth.random_elems(rng, prec, n, -24, 24), synth.random_elems(rng, prec, n, -24, 24)
            return torch.from_numpy(layout.aos_to_vec(prec, synth.interleave_complex(prec, re, im), True).copy()).cuda()
        lm, hd = synth.random_elems(rng, prec, n, -24, 24)
        return torch.from_numpy(layout.vec_from_parts(prec, lm, hd).copy()).cuda()

    if kind == "gemv_r":
        ld = -(-cols // 32) * 32
        A, x, y, yo = vec(rows * ld), vec(cols), vec(rows), empty(prec, rows)
        run = lambda: gemv(prec, rows, cols, A, ld, x, y, yo)  # noqa: E731
    else:
        a, x, y, z = vec(1, True), vec(rows, True), vec(rows, True), empty(prec, rows, True)
        run = lambda: axpy(prec, rows, a, x, y, z, cplx=True)  # noqa: E731
    times = {}
    for lanes in splits:
        set_split(KINDS[kind], prec, lanes)
        run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            run()
        e1.record()
        torch.cuda.synchronize()
        times[lanes] = e0.elapsed_time(e1) / reps
    best = min(times, key=times.get)
    set_split(KINDS[kind], prec, best)
    if cache is not None:
        cache.record_split(kind, prec, rows, cols, best)
    return times


def autotune_gemm_warps(prec: int, m: int, n: int, k: int, cplx: bool = False, reps: int = 2,
                        cache: TuningCache | None = None, seed: int = 0x7E58):
    """Time the plain GEMM's block shapes (4, 8, 16 warps) on random m x k and
    k x n operands at `prec`, install the fastest and record it in `cache`
    under the shape bucket of C.  Returns {warps: ms}."""
    import numpy as np
    import torch

    from . import empty, gemm, layout, synth

    rng = np.random.default_rng(seed)
    lda, ldb = -(-k // 32) * 32, -(-n // 32) * 32

    def mat(rows, cols, ld):
        if cplx:
            re = synth.random_elems(rng, prec, rows * ld, -16, 16)
            im = synth.random_elems(rng, prec, rows * ld, -16, 16)
            aos = synth.interleave_complex(prec, re, im)
            return torch.from_numpy(layout.aos_to_vec(prec, aos, True).copy()).cuda()
        lm, hd = synth.random_elems(rng, prec, rows * ld, -16, 16)
        return torch.from_numpy(layout.vec_from_parts(prec, lm, hd).copy()).cuda()

    A, B, Cd = mat(m, k, lda), mat(k, n, ldb), empty(prec, m * ldb, cplx)
    times = {}
    for w in GEMM_WARPS:
        set_gemm_warps(prec, w, cplx)
        gemm(prec, m, n, k, A, lda, B, ldb, Cd, ldb, cplx=cplx)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            gemm(prec, m, n, k, A, lda, B, ldb, Cd, ldb, cplx=cplx)
        e1.record()
        torch.cuda.synchronize()
        times[w] = e0.elapsed_time(e1) / reps
    best = min(times, key=times.get)
    set_gemm_warps(prec, best, cplx)
    if cache is not None:
        cache.record_gemm_warps(prec, m, n, best, cplx)
    return times
