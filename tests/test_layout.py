"""Host-side layout logic: AoS <-> tiles round trips, sizes, generators."""
import numpy as np
import pytest

from mpc_cuda_b200 import layout, synth


@pytest.mark.parametrize("cplx", (False, True))
@pytest.mark.parametrize("prec", layout.SUPPORTED)
@pytest.mark.parametrize("n", (1, 31, 32, 33, 100))
def test_aos_roundtrip(orc, prec, n, cplx):
    A, _ = orc.gen_pairs(prec, n, 0x123 + n, cplx)
    v = layout.aos_to_vec(prec, A, cplx)
    assert v.size == layout.vec_bytes(prec, n, cplx)
    back = layout.vec_to_aos(prec, v, n, cplx)
    assert orc.mismatches(prec, back, A, cplx)[0] == 0
    assert np.array_equal(back, A)  # random values are nonzero: bytes identical


@pytest.mark.parametrize("prec", layout.SUPPORTED)
def test_tile_geometry(prec):
    N = prec // 32
    assert layout.tile_bytes(prec) == 32 * (4 * N + 4)
    assert layout.tile_bytes(prec) % 128 == 0
    # limb k of element e in tile 0: group k//V, lane e, slot k%V
    limbs = np.arange(32 * N, dtype=np.uint32).reshape(32, N)
    heads = np.arange(32, dtype=np.uint32)
    words = layout.vec_from_parts(prec, limbs, heads).view(np.uint32)
    V = min(4, N)
    for e in (0, 5, 31):
        for k in range(N):
            g, s = divmod(k, V)
            assert words[g * 32 * V + e * V + s] == limbs[e, k]
        assert words[32 * N + e] == heads[e]


def test_zero_is_canonical(orc):
    prec = 256
    A, _ = orc.gen_pairs(prec, 40, 1)
    limbs, heads = layout.parts_from_aos(prec, A)
    heads[3] = layout.HEAD_ZERO
    aos = layout.aos_from_parts(prec, limbs, heads)
    back_l, back_h = layout.parts_from_aos(prec, aos)
    assert back_h[3] == layout.HEAD_ZERO and not back_l[3].any()


def test_from_doubles_exact(orc):
    d = np.array([1.5, -0.25, 1.0 / 3.0, 0.0, 1e-300, -7.0e200])
    for prec in (64, 256):
        limbs, heads = synth.from_doubles(prec, d)
        ref = np.zeros((d.size, 16 + prec // 8), np.uint8)
        orc.lib().orc_from_double(prec, d.size, d.ctypes.data, ref.ctypes.data)
        assert orc.mismatches(prec, layout.aos_from_parts(prec, limbs, heads), ref)[0] == 0


def test_generators_shape_and_distribution():
    limbs, heads = synth.random_elems(np.random.default_rng(1), 1024, 5000, -32, 32, 0.01)
    nz = heads != layout.HEAD_ZERO
    assert (limbs[nz, -1] >> 31 == 1).all()
    e = heads[nz].view(np.int32) >> 1
    assert e.min() >= -32 and e.max() <= 32
    assert 0.003 < (~nz).mean() < 0.02
    m, n, p = synth.gemv_batch_shapes(count=4096)
    assert m.min() >= 16 and m.max() <= 512 and set(np.unique(p)) <= set(layout.SUPPORTED)


def test_gemv_batch_pools_are_tile_aligned_and_zero_padded(orc):
    """The batched GEMV workload generator: every operand starts on a tile
    boundary, padding is exact zeros, and a problem's operands come back out
    of the pools with the shapes the problem names."""
    m, n, prec = synth.gemv_batch_shapes(count=60)
    assert m.min() >= 16 and m.max() <= 512 and n.min() >= 16 and n.max() <= 512
    assert set(prec.tolist()) <= set(layout.SUPPORTED)
    probs, pools = synth.gemv_batch(count=60)
    assert len(probs) == 60
    for pr in probs:
        assert pr["lda"] % 32 == 0 and pr["lda"] >= pr["n"]
        assert pr["a_off"] % 32 == 0 and pr["x_off"] % 32 == 0 and pr["y_off"] % 32 == 0
        P = pools[pr["prec"]]
        la, ha = P["A"]
        rows = ha[pr["a_off"]:pr["a_off"] + pr["m"] * pr["lda"]].reshape(pr["m"], pr["lda"])
        assert (rows[:, pr["n"]:] == layout.HEAD_ZERO).all() and (rows[:, :pr["n"]] != layout.HEAD_ZERO).all()
        A, x, y = synth.gemv_batch_problem(pools, pr)
        N = pr["prec"] // 32
        assert A[0].shape == (pr["m"] * pr["n"], N) and x[0].shape == (pr["n"], N) and y[0].shape == (pr["m"], N)
        assert (A[0][:, -1] >> 31).all() and (x[0][:, -1] >> 31).all()
    # a sample through the oracle: the AoS of the padded pool with lda gives the dense problem's result
    pr = min(probs, key=lambda p: p["m"] * p["n"])
    p = pr["prec"]
    A, x, y = synth.gemv_batch_problem(pools, pr)
    dense = orc.gemv(p, pr["m"], pr["n"], layout.aos_from_parts(p, *A), pr["n"], layout.aos_from_parts(p, *x),
                     layout.aos_from_parts(p, *y))
    Ap = layout.aos_from_parts(p, *pools[p]["A"])[pr["a_off"]:pr["a_off"] + pr["m"] * pr["lda"]]
    padded = orc.gemv(p, pr["m"], pr["n"], Ap, pr["lda"], layout.aos_from_parts(p, *x), layout.aos_from_parts(p, *y))
    assert orc.mismatches(p, dense, padded)[0] == 0
