"""The drop-in header's conversions and utilities against the reference's own
header built for the host (CPU only).

cu_freal's finalize, from_double / to_double, cu_cmp, cu_cmpmag, cu_convert,
cu_from_si and cu_lround are written on the mpb core here; the reference
implements them over its 64-bit limbs (include/mpc_cuda/cu_freal.cuh:83-165,
215-222, 304-356).  Both are built for the host and run on the same inputs,
including the edge cases of each: ties for lround, carries out of the top in
finalize and convert, zeros, equal magnitudes of opposite sign, LONG_MIN, the
result's last bit just above, at and below D's bit 0 for finalize.  The results
must agree field for field (sign, exponent, every limb).
"""
import ctypes as C

import numpy as np
import pytest

PBS = (32, 64, 96, 128, 160, 256, 288, 512, 1024, 1056, 2048)
SMALL = (32, 96, 160, 256, 288, 1056)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.fixture(scope="module")
def libs(orc, mpb):
    if not orc.ref_available():
        pytest.skip("reference host build (oracle/_ref) not present")
    R, H = orc.ref(), mpb.host_lib()
    for L, pre in ((R, "ref"), (H, "mpbh")):
        getattr(L, pre + "_util").argtypes = [C.c_int, C.c_int, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p]
        getattr(L, pre + "_finalize").argtypes = [C.c_int, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p]
        getattr(L, pre + "_convert").argtypes = [C.c_int, C.c_int, C.c_long, C.c_void_p, C.c_void_p]
    return R, H


def _fields(X):
    """sign, exponent and limbs of AoS elements (the 4 padding bytes after the sign excluded)."""
    return np.concatenate([X[:, 0:4], X[:, 8:]], axis=1)


def _edge_values(orc, prec, seed):
    """random values, plus all-ones significands (carry on any rounding), ties and small integers."""
    n64 = (prec + 63) // 64
    A = orc.rand_elems(prec, 200, seed, -8, 70)
    ones = A[:8].copy()
    m = np.full((8, n64), np.uint64(0xFFFFFFFFFFFFFFFF))
    sb = 64 * n64 - prec
    if sb:
        m[:, 0] &= ~np.uint64((1 << sb) - 1)
    ones[:, 16:] = m.view(np.uint8).reshape(8, -1)
    d = np.array([0.5, -0.5, 1.5, -1.5, 2.5, -2.5, 3.5, 0.49999999999, 0.75, -0.75, 1e10 + 0.5, 2.0 ** 40 + 0.5,
                  -(2.0 ** 52) - 1, 0.0, 1.0, -7.0, 1e-300, 2.0 ** 61, 0.5000000001, 123456.5])
    return np.concatenate([A, ones, orc.from_double(prec, d)])


@pytest.mark.parametrize("prec", PBS)
def test_compare_and_lround_match_reference(orc, libs, prec):
    R, H = libs
    X = _edge_values(orc, prec, 0x1001 + prec)
    Y = np.concatenate([X[1:], X[:1]])
    Y[:10] = X[:10]  # equal pairs
    Y[10:20] = X[10:20]
    Y[10:20, 0:4] = (-np.frombuffer(X[10:20, 0:4].tobytes(), np.int32)).view(np.uint8).reshape(10, 4)
    n = X.shape[0]
    for op in (0, 1, 2):
        want, got = np.zeros(n, np.int64), np.zeros(n, np.int64)
        if op == 2:  # lround: |x| < 2^62 as the reference requires
            keep = np.frombuffer(X[:, 8:16].tobytes(), np.int64) <= 61
            Xs = np.ascontiguousarray(X[keep])
            want, got = want[: Xs.shape[0]], got[: Xs.shape[0]]
            assert R.ref_util(2, prec, Xs.shape[0], _p(Xs), _p(Xs), _p(want), None) == 0
            assert H.mpbh_util(2, prec, Xs.shape[0], _p(Xs), _p(Xs), _p(got), None) == 0
        else:
            assert R.ref_util(op, prec, n, _p(X), _p(Y), _p(want), None) == 0
            assert H.mpbh_util(op, prec, n, _p(X), _p(Y), _p(got), None) == 0
        assert np.array_equal(got, want), f"op {op}: first difference at {np.nonzero(got != want)[0][:5]}"


@pytest.mark.parametrize("prec", PBS)
def test_from_si_matches_reference(orc, libs, prec):
    R, H = libs
    rng = np.random.default_rng(prec)
    v = np.concatenate([np.array([0, 1, -1, 2, 3, -3, 255, 2 ** 31 - 1, 2 ** 32 + 1, 2 ** 53 + 1,
                                  np.iinfo(np.int64).max, np.iinfo(np.int64).min, -(2 ** 62) - 12345], np.int64),
                        rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, 200, dtype=np.int64),
                        rng.integers(-1000, 1000, 50, dtype=np.int64)])
    n = v.shape[0]
    want, got = orc.empty(prec, n), orc.empty(prec, n)
    assert R.ref_util(3, prec, n, None, None, _p(v), _p(want)) == 0
    assert H.mpbh_util(3, prec, n, None, None, _p(v), _p(got)) == 0
    assert np.array_equal(_fields(got), _fields(want))


@pytest.mark.parametrize("prec", PBS)
def test_double_conversions_match_reference(orc, libs, prec):
    R, H = libs
    rng = np.random.default_rng(7 + prec)
    d = np.concatenate([rng.standard_normal(300) * 10.0 ** rng.integers(-30, 30, 300),
                        [0.0, -0.0, 1.0, -1.0, 2.0 ** -1000, 1.7976931348623157e308, 5e-324, 1 / 3]])
    n = d.shape[0]
    want, got = orc.empty(prec, n), orc.empty(prec, n)
    R.ref_from_double(prec, n, _p(d), _p(want))
    H.mpbh_from_double(prec, n, _p(d), _p(got))
    assert np.array_equal(_fields(got), _fields(want))
    X = _edge_values(orc, prec, 0x2002 + prec)
    dw, dg = np.zeros(X.shape[0]), np.zeros(X.shape[0])
    R.ref_to_double(prec, X.shape[0], _p(X), _p(dw))
    H.mpbh_to_double(prec, X.shape[0], _p(X), _p(dg))
    assert np.array_equal(dg.view(np.int64), dw.view(np.int64))


@pytest.mark.parametrize("frm", SMALL)
def test_convert_matches_reference(orc, libs, frm):
    R, H = libs
    X = _edge_values(orc, frm, 0x3003 + frm)
    n = X.shape[0]
    for to in SMALL:
        want, got = orc.empty(to, n), orc.empty(to, n)
        assert R.ref_convert(to, frm, n, _p(X), _p(want)) == 0
        assert H.mpbh_convert(to, frm, n, _p(X), _p(got)) == 0
        assert np.array_equal(_fields(got), _fields(want)), f"{frm} -> {to}"


@pytest.mark.parametrize("prec", PBS)
def test_finalize_matches_reference(orc, libs, prec):
    """finalize on random magnitudes of 1-4 limbs with the leading one at every
    kind of position: result exact (fewer than PB bits), last bit at D's bit 0
    (round bit = brnd), above it (round bit inside D)."""
    R, H = libs
    rng = np.random.default_rng(0xF1 + prec)
    n = 600
    D = rng.integers(0, 2 ** 63, (n, 4), dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, (n, 4),
                                                                                        dtype=np.uint64)
    q = np.zeros((n, 6), np.int64)
    for i in range(n):
        ln = int(rng.integers(1, 5))
        if i % 3 == 0:  # last bit exactly at bit 0: msb = PB - 1, when it fits
            msb = min(prec - 1, 64 * ln - 1)
        elif i % 3 == 1:
            msb = int(rng.integers(0, 64 * ln))
        else:
            msb = 64 * ln - 1 - int(rng.integers(0, 3))
        if i % 50 == 7:
            msb = -1  # zero
        if msb >= 0:  # bits above msb clear, bit msb set
            for w in range(4):
                lo = 64 * w
                if lo > msb or w >= ln:
                    D[i, w] = 0
                elif msb < lo + 64:
                    b = msb - lo
                    D[i, w] = (D[i, w] & np.uint64((1 << b) - 1 if b < 64 else (1 << 64) - 1)) | np.uint64(1 << b)
        if i % 7 == 3:  # all ones under the leading one: rounding carries out
            for w in range(ln):
                lo = 64 * w
                if lo <= msb:
                    b = min(63, msb - lo)
                    D[i, w] = np.uint64((1 << (b + 1)) - 1) if b < 63 else np.uint64((1 << 64) - 1)
        q[i] = (ln, msb, int(rng.integers(-50, 50)), int(rng.integers(0, 2)), int(rng.integers(0, 2)),
                1 if rng.integers(0, 2) else -1)
    want, got = orc.empty(prec, n), orc.empty(prec, n)
    assert R.ref_finalize(prec, n, _p(D), _p(q), _p(want)) == 0
    assert H.mpbh_finalize(prec, n, _p(D), _p(q), _p(got)) == 0
    bad = np.nonzero((_fields(got) != _fields(want)).any(axis=1))[0]
    assert bad.size == 0, f"first differences at rows {bad[:5]}: q={q[bad[:1]]}"


@pytest.mark.parametrize("prec", PBS)
def test_product_terms_match_reference(orc, libs, prec):
    """cu_mk_term (the exact product as a wide term) and cu_round_sum2 (one
    rounding of a sum of two terms), including zeros and cancelling sums."""
    R, H = libs
    A, B = orc.gen_pairs(prec, 300, 0x77 + prec)
    Cc, Dd = A.copy(), B.copy()
    Cc[100:200], Dd[100:200] = orc.gen_pairs(prec, 100, 0x99 + prec)  # unrelated second terms
    Cc[200:210] = orc.from_double(prec, np.zeros(10))  # zero terms
    A[210:215] = orc.from_double(prec, np.zeros(5))
    n, wn = A.shape[0], 2 * ((prec + 63) // 64)
    out = []
    for L, f in ((R, "ref_terms"), (H, "mpbh_terms")):
        getattr(L, f).argtypes = [C.c_int, C.c_long] + [C.c_void_p] * 7
        hdr, M, r = np.zeros((n, 3), np.int64), np.zeros((n, wn), np.uint64), orc.empty(prec, n)
        assert getattr(L, f)(prec, n, _p(A), _p(B), _p(Cc), _p(Dd), _p(hdr), _p(M), _p(r)) == 0
        out.append((hdr, M, r))
    (h0, m0, r0), (h1, m1, r1) = out
    nz = h0[:, 2] == 0
    assert np.array_equal(h0[:, 2], h1[:, 2])
    assert np.array_equal(h0[nz], h1[nz]) and np.array_equal(m0[nz], m1[nz])
    assert np.array_equal(_fields(r0), _fields(r1))
