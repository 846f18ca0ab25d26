"""The tuning cache (mpc_cuda_b200/tune.py): keys, JSON round trip, and the
thread-vs-warp split it installs through mpb_set_split (host-side state, no GPU
needed); on a GPU, autotune_split must pick the fastest split it measured and
a cached batch tuning must reinstall on a new plan."""
import os

import pytest

from mpc_cuda_b200 import tune


def test_bucket_and_key():
    assert tune.bucket(512, 256) == "r512c256"
    assert tune.bucket(500, 200) == "r512c256"
    assert tune.bucket(1) == "r1c1"
    assert tune.key("gemv_r", 2048, 300, 60) == "gemv_r/2048/r512c64"


def test_cache_round_trip_and_apply(mpb, tmp_path):
    path = os.path.join(tmp_path, "tune.json")
    c = tune.TuningCache(path)
    c.record_split("gemv_r", 2048, 512, 256, 16)
    c.record_split("axpy_c", 1024, 1 << 18, 1, 1)
    with pytest.raises(ValueError):
        c.record_split("gemv_r", 512, 64, 64, 8)  # no cooperative form at 512 bits
    c.save()
    c2 = tune.TuningCache(path)
    assert c2.lookup_split("gemv_r", 2048, 500, 250) == 16
    assert c2.lookup_split("gemv_r", 2048, 4096, 64) is None
    old = mpb.get_split(mpb.SPLIT_GEMV_R, 2048)
    try:
        assert c2.apply_split("gemv_r", 2048, 512, 256) == 16
        assert mpb.get_split(mpb.SPLIT_GEMV_R, 2048) == 16
        assert c2.apply_split("gemv_r", 2048, 4096, 64) == 16  # nothing cached: unchanged
    finally:
        mpb.set_split(mpb.SPLIT_GEMV_R, 2048, old)


def test_batch_signature_is_order_free():
    a = [(1024, 40, 30), (64, 10, 5), (1024, 3, 300)]
    assert tune.TuningCache.batch_signature(a) == tune.TuningCache.batch_signature(a[::-1])


@pytest.mark.gpu
def test_autotune_split_picks_the_fastest(mpb, tmp_path):
    c = tune.TuningCache(os.path.join(tmp_path, "t.json"))
    old = mpb.get_split(mpb.SPLIT_GEMV_R, 2048)
    try:
        times = tune.autotune_split("gemv_r", 2048, 256, 64, cache=c)
        assert set(times) == {1, 8, 16}
        best = min(times, key=times.get)
        assert mpb.get_split(mpb.SPLIT_GEMV_R, 2048) == best
        assert c.lookup_split("gemv_r", 2048, 256, 64) == best
    finally:
        mpb.set_split(mpb.SPLIT_GEMV_R, 2048, old)


@pytest.mark.gpu
def test_batch_tuning_reinstalls_from_cache(mpb, tmp_path):
    from test_gpu_batch import make_batch, plan

    probs = make_batch(40, 0xE1, hi=60, precs=(256, 2048))
    b = plan(mpb, probs)
    b.autotune()
    c = tune.TuningCache(os.path.join(tmp_path, "b.json"))
    sig = tune.TuningCache.batch_signature([(p["prec"], p["m"], p["n"]) for p in probs])
    c.save_batch(sig, b)
    c.save()
    b2 = plan(mpb, probs)
    assert tune.TuningCache(c.path).apply_batch(sig, b2)
    assert b2.tuning() == b.tuning() and b2.splits() == b.splits()
    b.close()
    b2.close()


def test_gemm_warps_setting_and_cache(mpb, tmp_path):
    old = mpb.get_gemm_warps(512)
    try:
        mpb.set_gemm_warps(512, 4)
        assert mpb.get_gemm_warps(512) == 4
        assert mpb.get_gemm_warps(512, cplx=True) == 8  # real and complex are separate
        with pytest.raises(mpb.MpbError):
            mpb.set_gemm_warps(512, 6)
        with pytest.raises(mpb.MpbError):
            mpb.set_gemm_warps(300, 8)
        c = tune.TuningCache(os.path.join(tmp_path, "g.json"))
        c.record_gemm_warps(512, 128, 128, 16)
        c.record_gemm_warps(256, 512, 512, 4, cplx=True)
        with pytest.raises(ValueError):
            c.record_gemm_warps(512, 128, 128, 32)
        c.save()
        c2 = tune.TuningCache(c.path)
        assert c2.apply_gemm_warps(512, 120, 100) == 16
        assert mpb.get_gemm_warps(512) == 16
        assert c2.lookup_gemm_warps(256, 512, 512, cplx=True) == 4
        assert c2.lookup_gemm_warps(256, 512, 512) is None
    finally:
        mpb.set_gemm_warps(512, old)


@pytest.mark.gpu
def test_autotune_gemm_warps_picks_the_fastest(mpb, tmp_path):
    c = tune.TuningCache(os.path.join(tmp_path, "t.json"))
    old = mpb.get_gemm_warps(512)
    try:
        times = tune.autotune_gemm_warps(512, 128, 128, 64, cache=c)
        assert set(times) == {4, 8, 16}
        best = min(times, key=times.get)
        assert mpb.get_gemm_warps(512) == best
        assert c.lookup_gemm_warps(512, 128, 128) == best
    finally:
        mpb.set_gemm_warps(512, old)
