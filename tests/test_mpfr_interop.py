"""Host interop with MPFR / MPC objects (mpb_aos_to_mpfr / mpb_aos_from_mpfr and
the mpc_t forms): CPU only, against the system MPFR 4.2.1.

The reference's tests convert with mpz_import + mpfr_set_z (RNDN) +
mpfr_mul_2si (tools/test_freal.cu:28-39): the value rounded to nearest at the
mpfr_t's precision.  Checked here: exact round trips at equal precision,
rounding to smaller precisions equal to mpfr_set (RNDN) from an exact copy,
larger precisions exact, zero, and NaN / infinity refused.
"""
import ctypes as C

import numpy as np
import pytest

MPFR_PATH = "/usr/lib/x86_64-linux-gnu/libmpfr.so.6"
RNDN = 0


class MpfrStruct(C.Structure):
    _fields_ = [("prec", C.c_long), ("sign", C.c_int), ("exp", C.c_long), ("d", C.c_void_p)]


@pytest.fixture(scope="module")
def mpfr():
    L = C.CDLL(MPFR_PATH)
    P = C.POINTER(MpfrStruct)
    L.mpfr_init2.argtypes = [P, C.c_long]
    L.mpfr_clear.argtypes = [P]
    L.mpfr_set.argtypes = [P, P, C.c_int]
    L.mpfr_equal_p.argtypes = [P, P]
    L.mpfr_zero_p.argtypes = [P]
    L.mpfr_set_nan.argtypes = [P]
    L.mpfr_set_inf.argtypes = [P, C.c_int]
    L.mpfr_set_zero.argtypes = [P, C.c_int]
    L.mpfr_signbit.argtypes = [P]
    return L


def _objs(L, prec, n):
    arr = (MpfrStruct * n)()
    for i in range(n):
        L.mpfr_init2(C.byref(arr[i]), prec)
    ptrs = (C.c_void_p * n)(*[C.addressof(arr[i]) for i in range(n)])
    return arr, ptrs


def _free(L, arr):
    for z in arr:
        L.mpfr_clear(C.byref(z))


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.mark.parametrize("prec", (64, 128, 256, 512, 1024, 2048))
def test_mpfr_round_trip_and_rounding(orc, mpb, mpfr, prec):
    L, lib = mpfr, mpb.lib()
    n = 200
    A, _ = orc.gen_pairs(prec, n, 0x5151 + prec)
    A[7] = orc.from_double(prec, [0.0])[0]
    exact, pe = _objs(L, prec, n)
    assert lib.mpb_aos_to_mpfr(prec, n, _p(A), pe) == 0
    back = orc.empty(prec, n)
    assert lib.mpb_aos_from_mpfr(prec, n, pe, _p(back)) == 0
    assert orc.mismatches(prec, back, A)[0] == 0 and (back == A).all()
    assert L.mpfr_zero_p(C.byref(exact[7]))
    for q in (prec + 37, prec - 13, 53, 2):  # rounding at the destination's precision
        got, pg = _objs(L, q, n)
        want, _ = _objs(L, q, n)
        assert lib.mpb_aos_to_mpfr(prec, n, _p(A), pg) == 0
        for i in range(n):
            L.mpfr_set(C.byref(want[i]), C.byref(exact[i]), RNDN)
            assert L.mpfr_equal_p(C.byref(got[i]), C.byref(want[i])) or \
                (L.mpfr_zero_p(C.byref(got[i])) and L.mpfr_zero_p(C.byref(want[i]))), f"q={q} i={i}"
        _free(L, want)
        if q > prec:  # exact: back to prec bits unchanged
            b2 = orc.empty(prec, n)
            assert lib.mpb_aos_from_mpfr(prec, n, pg, _p(b2)) == 0
            assert (b2 == A).all()
        _free(L, got)
    # from a wider mpfr_t (2 prec bits): rounded to nearest at prec bits, like mpfr_set
    _free(L, exact)
    pb = 2 * prec
    if pb > 2048:
        return
    wide, pw = _objs(L, pb, n)
    B, _ = orc.gen_pairs(pb, n, 0x77 + prec)
    assert lib.mpb_aos_to_mpfr(pb, n, _p(B), pw) == 0
    got = orc.empty(prec, n)
    assert lib.mpb_aos_from_mpfr(prec, n, pw, _p(got)) == 0
    ref, pr = _objs(L, prec, n)
    for i in range(n):
        L.mpfr_set(C.byref(ref[i]), C.byref(wide[i]), RNDN)
    want = orc.empty(prec, n)
    assert lib.mpb_aos_from_mpfr(prec, n, pr, _p(want)) == 0
    assert (got == want).all()
    assert orc.mismatches(prec, got, orc.convert(prec, pb, B))[0] == 0
    for arr in (wide, ref):
        _free(L, arr)


def test_mpfr_special_values(orc, mpb, mpfr):
    L, lib, prec = mpfr, mpb.lib(), 256
    z, pz = _objs(L, prec, 3)
    L.mpfr_set_zero(C.byref(z[0]), -1)  # -0 becomes +0
    L.mpfr_set_nan(C.byref(z[1]))
    L.mpfr_set_inf(C.byref(z[2]), 1)
    out = orc.empty(prec, 3)
    assert lib.mpb_aos_from_mpfr(prec, 1, pz, _p(out)) == 0
    assert (out[0] == orc.from_double(prec, [0.0])[0]).all()
    for i in (1, 2):
        one = (C.c_void_p * 1)(pz[i])
        assert lib.mpb_aos_from_mpfr(prec, 1, one, _p(out)) == -7  # MPB_ERR_ARG
    assert lib.mpb_aos_from_mpfr(96, 1, pz, _p(out)) == -1  # MPB_ERR_PREC
    _free(L, z)


@pytest.mark.parametrize("prec", (128, 1024))
def test_mpc_round_trip(orc, mpb, mpfr, prec):
    L, lib = mpfr, mpb.lib()
    n = 64
    A, _ = orc.gen_pairs(prec, n, 0x6161 + prec, cplx=True)
    arr = (MpfrStruct * (2 * n))()
    for i in range(2 * n):
        L.mpfr_init2(C.byref(arr[i]), prec)
    ptrs = (C.c_void_p * n)(*[C.addressof(arr[2 * i]) for i in range(n)])
    assert lib.mpb_caos_to_mpc(prec, n, _p(A), ptrs) == 0
    back = orc.empty(prec, n, True)
    assert lib.mpb_caos_from_mpc(prec, n, ptrs, _p(back)) == 0
    assert (back == A).all()
    _free(L, arr)


def _elem(prec, sign, exp, limbs):
    """One AoS cu_freal<prec> element: { int sign; long exp; uint64 m[] }."""
    n64 = (prec + 63) // 64
    e = np.zeros(16 + 8 * n64, np.uint8)
    e[0:4] = np.array([sign], np.int32).view(np.uint8)
    e[8:16] = np.array([exp], np.int64).view(np.uint8)
    e[16:] = np.array(limbs, np.uint64).view(np.uint8)
    return e.reshape(1, -1)


def test_mpfr_exponent_range_edges(mpb, mpfr):
    """Results outside MPFR's default exponent range [1 - 2^30, 2^30 - 1] are
    refused (MPB_ERR_ARG) in both directions, and the destination keeps its
    old value; values at the edges themselves convert."""
    L, lib, prec = mpfr, mpb.lib(), 128
    emax, emin = (1 << 30) - 1, 1 - (1 << 30)
    ones = [0xFFFFFFFFFFFFFFFF, 0xFFFFFFFFFFFFFFFF]
    top = [0, 1 << 63]
    z, pz = _objs(L, 64, 1)
    L.mpfr_set_zero(C.byref(z[0]), 1)
    # at the top edge without a carry: converts
    assert lib.mpb_aos_to_mpfr(prec, 1, _p(_elem(prec, 1, emax, top)), pz) == 0
    assert z[0].exp == emax
    # 1 - 2^-128 at 2^emax rounds to 2^(emax+1) at 64 bits: refused, unchanged
    assert lib.mpb_aos_to_mpfr(prec, 1, _p(_elem(prec, 1, emax, ones)), pz) == -7
    assert z[0].exp == emax
    # the bottom edge converts, one below it (a head the engine can hold) is refused
    assert lib.mpb_aos_to_mpfr(prec, 1, _p(_elem(prec, -1, emin, top)), pz) == 0
    assert z[0].exp == emin and z[0].sign == -1
    assert lib.mpb_aos_to_mpfr(prec, 1, _p(_elem(prec, 1, emin - 1, top)), pz) == -7
    assert z[0].exp == emin and z[0].sign == -1
    _free(L, z)
    # from a 128-bit mpfr_t of all ones at 2^emax into 64 bits: the carry leaves
    # the engine's range, so the element is refused and keeps its old limbs and head
    w, pw = _objs(L, prec, 1)
    assert lib.mpb_aos_to_mpfr(prec, 1, _p(_elem(prec, 1, emax, ones)), pw) == 0
    old = _elem(64, 1, 5, [0x8000000000000001])
    out = old.copy()
    assert lib.mpb_aos_from_mpfr(64, 1, pw, _p(out)) == -7
    assert (out == old).all()
    _free(L, w)
