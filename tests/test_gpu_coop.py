"""The warp-cooperative forms for wide operands (mpb/coop.cuh): a GEMV row or a
complex AXPY element held by a group of lanes.  Every thread-vs-warp split the
library offers is forced in turn (mpb_set_split / the batch plan's split) and
its results are compared with MPFR / MPC bit for bit (integer arithmetic, no
tolerance), on random operands and on constructed cases for the cooperative
sum: exact cancellation to zero, deep cancellation, a negative difference of
equal exponents, carries out of every word, zero operands and huge exponent
gaps."""
import numpy as np
import pytest

from conftest import to_dev, to_host
from mpc_cuda_b200 import layout, synth

pytestmark = pytest.mark.gpu
SPLITS = {1024: (1, 4, 8), 2048: (1, 8, 16)}


def dvec(prec, aos, cplx=False):
    return to_dev(layout.aos_to_vec(prec, aos, cplx))


def hvec(prec, t, n, cplx=False):
    return layout.vec_to_aos(prec, to_host(t), n, cplx)


def _with_split(mpb, kind, prec, lanes, fn):
    old = mpb.get_split(kind, prec)
    mpb.set_split(kind, prec, lanes)
    try:
        return fn()
    finally:
        mpb.set_split(kind, prec, old)


def _hard_rows(orc, prec, m, n, seed):
    """A (m x n), x, y with rows that cancel: row 0 sums pairs a*x - a*x to
    exact zeros, row 1 ends at -y (zero result), row 2 holds all-ones
    significands (carries through every word), row 3 mixes exponents 2^-200 ..
    2^200 apart; the other rows are random."""
    A = orc.rand_elems(prec, m * n, seed, -20, 20).reshape(m, n, -1)
    x = orc.rand_elems(prec, n, seed + 1, -20, 20)
    y = orc.rand_elems(prec, m, seed + 2, -20, 20)
    es = A.shape[2]
    neg = lambda e: np.concatenate([(-np.frombuffer(e[0:4].tobytes(), np.int32)).view(np.uint8), e[4:]])  # noqa: E731
    for k in range(0, n - 1, 2):  # row 0: A[0,k+1] = A[0,k], x[k+1] = -x[k]
        A[0, k + 1] = A[0, k]
        x[k + 1] = neg(x[k])
    if n % 2:
        A[0, n - 1] = orc.from_double(prec, [0.0])[0]
    n64 = (prec + 63) // 64
    ones = np.full(n64, np.uint64(0xFFFFFFFFFFFFFFFF)).view(np.uint8)
    if m > 2:
        A[2, :, 16:] = ones
    if m > 3:
        ex = np.frombuffer(A[3, :, 8:16].tobytes(), np.int64).copy()
        ex[::3] += 200
        ex[1::3] -= 200
        A[3, :, 8:16] = ex.view(np.uint8).reshape(-1, 8)
    A = A.reshape(m * n, es)
    if m > 1:  # row 1: y = -(the row's dot product), rounded the same way
        dot = orc.gemv(prec, 1, n, A[n:2 * n], n, x, orc.from_double(prec, [0.0]), impl="mp")
        y[1] = neg(dot[0])
    return A, x, y


@pytest.mark.parametrize("prec", (1024, 2048))
def test_gemv_every_split(orc, mpb, prec):
    m, n = (37, 45) if prec == 1024 else (19, 23)
    A, x, y = _hard_rows(orc, prec, m, n, 0xC0 + prec)
    lda = -(-n // 32) * 32
    from test_gpu_ops import pad_rows

    dA, dx, dy = dvec(prec, pad_rows(prec, A, m, n, lda)), dvec(prec, x), dvec(prec, y)
    exp = orc.gemv(prec, m, n, A, n, x, y, impl="mp")
    for lanes in SPLITS[prec]:
        yo = mpb.empty(prec, m)
        _with_split(mpb, mpb.SPLIT_GEMV_R, prec, lanes, lambda: mpb.gemv(prec, m, n, dA, lda, dx, dy, yo))
        bad, first = orc.mismatches(prec, hvec(prec, yo, m), exp)
        assert bad == 0, f"GEMV PB={prec} lanes={lanes}: {bad} rows differ from MPFR (first {first})"


@pytest.mark.parametrize("lanes", (1, 4, 8))
def test_complex_axpy_1024_every_split(orc, mpb, lanes):
    prec, n = 1024, 3000
    A, X, Y = synth.axpy_c1024(seed=0x77, n=n, prec=prec)
    Aa, Xa, Ya = (synth.interleave_complex(prec, *p) for p in (A, X, Y))
    es = layout.aos_bytes(prec)
    # y = -(a x) rounded per component on a stretch: exact cancellation in the add
    ax = orc.axpy(prec, Aa, Xa[:40], np.repeat(np.concatenate([orc.from_double(prec, [0.0])] * 2, axis=1), 40,
                                                axis=0), True, impl="mp")
    for c in (0, 1):
        part = ax[:, c * es:(c + 1) * es].copy()
        part[:, 0:4] = (-np.frombuffer(part[:, 0:4].tobytes(), np.int32)).view(np.uint8).reshape(-1, 4)
        Ya[:40, c * es:(c + 1) * es] = part
    exp = orc.axpy(prec, Aa, Xa, Ya, True, impl="mp")
    z = mpb.empty(prec, n, True)
    _with_split(mpb, mpb.SPLIT_AXPY_C, prec, lanes,
                lambda: mpb.axpy(prec, n, dvec(prec, Aa, True), dvec(prec, Xa, True), dvec(prec, Ya, True), z,
                                 cplx=True))
    bad, first = orc.mismatches(prec, hvec(prec, z, n, True), exp, True)
    assert bad == 0, f"complex AXPY lanes={lanes}: {bad} differ from MPC (first {first})"


def test_batch_every_split(orc, mpb):
    from test_gpu_batch import expected, got, make_batch, plan

    probs = make_batch(60, 0xB7, hi=90, precs=(1024, 2048))
    b = plan(mpb, probs)
    for lanes_1024, lanes_2048 in ((1, 1), (4, 8), (8, 16)):
        b.set_split(1024, lanes_1024)
        b.set_split(2048, lanes_2048)
        assert b.splits()[1024] == lanes_1024 and b.splits()[2048] == lanes_2048
        for p in probs:
            p["dyo"].zero_()
        b.run()
        for i, p in enumerate(probs):
            if p["m"] == 0:
                continue
            bad, first = orc.mismatches(p["prec"], got(p), expected(orc, p))
            assert bad == 0, f"problem {i} PB={p['prec']} lanes {lanes_1024}/{lanes_2048}: first mismatch {first}"
    b.close()


def test_split_validation(mpb):
    with pytest.raises(mpb.MpbError):
        mpb.set_split(mpb.SPLIT_GEMV_R, 512, 8)  # no cooperative form below 1024 bits
    with pytest.raises(mpb.MpbError):
        mpb.set_split(mpb.SPLIT_AXPY_C, 2048, 8)
    with pytest.raises(mpb.MpbError):
        mpb.set_split(mpb.SPLIT_GEMV_R, 1024, 16)
    assert mpb.get_split(mpb.SPLIT_GEMV_R, 512) == 1
