"""Linear algebra and elementary functions at a runtime precision p
(mpb_axpy_r_rp, mpb_gemv_r_rp, mpb_gemm_r_rp, mpb_fmath_r_rp): vectors in the
storage format PB = mpb_storage_prec(p), every operation rounded at p bits.

AXPY / GEMV / GEMM must equal the system MPFR with p-bit destinations in the
same order (one mpfr_mul and one mpfr_add per step, bit for bit: integer
arithmetic, no tolerance); the expected values are built from the oracle's
MPFR operations at p (mp_op_rp).  The elementary functions must lie within
1 ULP of p bits of MPFR's value at 4 PB bits (their faithful contract).
"""
import numpy as np
import pytest

from conftest import to_dev, to_host
from mpc_cuda_b200 import layout

pytestmark = pytest.mark.gpu
PS = (2, 53, 100, 200, 255, 300, 511, 700, 1023, 2046)


def dvec(prec, aos):
    return to_dev(layout.aos_to_vec(prec, aos))


def hvec(prec, t, n):
    return layout.vec_to_aos(prec, to_host(t), n)


def _operands(orc, p, n, seed):
    """random PB-bit operands rounded to p bits (the values a p-bit caller holds)"""
    pb = 64
    while pb < p + 2:
        pb *= 2
    A, B = orc.gen_pairs(pb, n, seed)
    zero = orc.from_double(pb, np.zeros(n))
    one = np.repeat(orc.from_double(pb, [1.0]), n, axis=0)
    return pb, orc.op_rp("mul", p, pb, A, one, zero), orc.op_rp("mul", p, pb, B, one, zero)


@pytest.mark.parametrize("p", PS)
def test_axpy_rp(orc, mpb, p):
    n = 3000
    pb, X, Y = _operands(orc, p, n, 0xA10 + p)
    a = X[5:6].copy()
    z = mpb.empty(pb, n)
    mpb.axpy_rp(p, n, dvec(pb, a), dvec(pb, X), dvec(pb, Y), z)
    t = orc.op_rp("mul", p, pb, np.repeat(a, n, axis=0), X)
    want = orc.op_rp("add", p, pb, t, Y)
    bad, first = orc.mismatches(pb, hvec(pb, z, n), want)
    assert bad == 0, f"AXPY p={p}: {bad} differ from MPFR (first {first})"


def _dot_rows(orc, p, pb, A, m, k, xs):
    """per row i: acc = +0; acc = round_p(acc + round_p(A[i,k] x[k])) in k order"""
    acc = orc.from_double(pb, np.zeros(m))
    Ar = A.reshape(m, k, -1)
    for kk in range(k):
        t = orc.op_rp("mul", p, pb, np.ascontiguousarray(Ar[:, kk]), np.ascontiguousarray(xs[kk]))
        acc = orc.op_rp("add", p, pb, acc, t)
    return acc


@pytest.mark.parametrize("p", PS)
def test_gemv_rp(orc, mpb, p):
    m, n = (45, 37) if p <= 1023 else (20, 17)
    pb, A, _ = _operands(orc, p, m * n, 0xB10 + p)
    _, x, y = _operands(orc, p, max(m, n), 0xB20 + p)
    x, y = x[:n], y[:m]
    lda = -(-n // 32) * 32
    from test_gpu_ops import pad_rows

    yo = mpb.empty(pb, m)
    mpb.gemv_rp(p, m, n, dvec(pb, pad_rows(pb, A, m, n, lda)), lda, dvec(pb, x), dvec(pb, y), yo)
    xs = [np.repeat(x[kk:kk + 1], m, axis=0) for kk in range(n)]
    want = orc.op_rp("add", p, pb, _dot_rows(orc, p, pb, A, m, n, xs), y)
    bad, first = orc.mismatches(pb, hvec(pb, yo, m), want)
    assert bad == 0, f"GEMV p={p}: {bad} rows differ from MPFR (first {first})"


@pytest.mark.parametrize("p", PS)
def test_gemm_rp(orc, mpb, p):
    m, n, k = (9, 33, 21) if p <= 1023 else (5, 7, 9)
    pb, A, B = _operands(orc, p, max(m * k, k * n), 0xC10 + p)
    A, B = A[:m * k], B[:k * n]
    lda, ldb, ldc = -(-k // 32) * 32, -(-n // 32) * 32, -(-n // 32) * 32
    from test_gpu_ops import pad_rows, unpad_rows

    Cd = mpb.empty(pb, m * ldc)
    mpb.gemm_rp(p, m, n, k, dvec(pb, pad_rows(pb, A, m, k, lda)), lda, dvec(pb, pad_rows(pb, B, k, n, ldb)), ldb,
                Cd, ldc)
    got = unpad_rows(hvec(pb, Cd, m * ldc), m, n, ldc)
    # entry (i, j): row i of A against column j of B, as m*n independent dots
    Ae = np.repeat(A.reshape(m, 1, k, -1), n, axis=1).reshape(m * n * k, -1)
    Br = B.reshape(k, n, -1)
    xs = [np.ascontiguousarray(np.tile(Br[kk], (m, 1))) for kk in range(k)]
    want = _dot_rows(orc, p, pb, Ae, m * n, k, xs)
    bad, first = orc.mismatches(pb, got, want)
    assert bad == 0, f"GEMM p={p}: {bad} entries differ from MPFR (first {first})"


@pytest.mark.parametrize("p", (53, 200, 700, 2046))
@pytest.mark.parametrize("name", ("exp", "log", "sin", "atan"))
def test_fmath_rp_within_one_ulp(orc, mpb, p, name):
    n = 300 if p <= 700 else 80
    pb = 64
    while pb < p + 2:
        pb *= 2
    A = orc.rand_elems(pb, n, 0xD10 + p, -3, 3, positive=(name == "log"))
    r = mpb.empty(pb, n)
    mpb.fmath_rp(name, p, n, dvec(pb, A), r)
    got = hvec(pb, r, n)
    pref = min(4 * pb, orc.lib().orc_max_prec())
    ulp_pb = orc.ulp_errors(pb, got, pref, orc.fn(name, pb, A, None, pref))
    ulp_p = ulp_pb / 2.0 ** (pb - p)  # one ULP of p bits is 2^(PB-p) ULPs of PB bits
    assert ulp_p.max() <= 1.0, f"{name} p={p}: {ulp_p.max():.3g} ULP of {p} bits"
    # the result carries p significant bits: rounding it again to p bits changes nothing
    zero = orc.from_double(pb, np.zeros(n))
    assert orc.mismatches(pb, got, orc.op_rp("add", p, pb, got, zero))[0] == 0
