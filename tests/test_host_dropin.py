"""The drop-in cu_fp surface, built for the host CPU, against MPFR/MPC.

This exercises the exact code the device runs (the mpb core), with each PTX
carry-chain instruction emulated on the host, on the reference's own test
method: seeded xorshift operand pairs (tools/test_freal.cu:17-27,55),
precisions including the sub-limb SB=32 cases (96, 160, 288, 1056), and
equality in mpfr_equal_p / mpc_cmp semantics.
"""
import ctypes as C

import numpy as np
import pytest

PRECS = (32, 64, 96, 128, 160, 256, 288, 512, 1024, 1056, 2048)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.mark.parametrize("prec", PRECS)
def test_real_ops(orc, mpb, prec):
    H = mpb.host_lib()
    M = 12000 if prec <= 1056 else 3000
    A, B = orc.gen_pairs(prec, M, 0x1111 * (prec // 32))
    for op, kind in enumerate(("mul", "add", "sub")):
        R = orc.empty(prec, M)
        assert H.mpbh_binop(prec, op, M, _p(A), _p(B), _p(R)) == 0
        bad, first = orc.mismatches(prec, R, orc.binop(kind, prec, A, B, "mp"))
        assert bad == 0, f"{kind} PB={prec}: first mismatch {first}"
    Cc, _ = orc.gen_pairs(prec, M, 0x77 + prec)
    R = orc.empty(prec, M)
    assert H.mpbh_fma(prec, M, _p(A), _p(B), _p(Cc), _p(R)) == 0
    assert orc.mismatches(prec, R, orc.fma(prec, A, B, Cc, "mp"))[0] == 0


@pytest.mark.parametrize("prec", PRECS)
def test_complex_ops(orc, mpb, prec):
    H = mpb.host_lib()
    M = 3000 if prec <= 1056 else 800
    A, B = orc.gen_pairs(prec, M, 0x11 * (prec // 32), cplx=True)
    for op, kind in enumerate(("cmul", "cadd", "csub")):
        R = orc.empty(prec, M, True)
        assert H.mpbh_cbinop(prec, op, M, _p(A), _p(B), _p(R)) == 0
        bad, first = orc.mismatches(prec, R, orc.binop(kind, prec, A, B, "mp"), True)
        assert bad == 0, f"{kind} PB={prec}: first mismatch {first}"


def window_operands(prec, count, seed):
    """(limbs_a, limbs_b) pairs of prec-bit significands whose product cannot be
    rounded from the upper columns of the limb product alone: the 64 bits under
    the mantissa of the truncated product lie within 2^39 below the midpoint,
    so the full product decides.  a = 2^(P-1) + small odd, b with a bit
    pattern right under the rounding position: 1000..0 or 0111..1 over 29 bits
    (half the time with nothing below: exact ties), or 1 followed by 63 zeros
    with random bits below, where the truncated product is an exact tie and only
    the omitted low pairs show that the product lies above the midpoint."""
    import random

    P, N = prec, prec // 32
    rng = random.Random(seed)
    limbs = lambda v: [(v >> (32 * i)) & 0xFFFFFFFF for i in range(N)]  # noqa: E731
    out = []
    while len(out) < count:
        M = (1 << (P - 1)) | rng.getrandbits(P - 1)
        if rng.random() < 0.5:
            A = (1 << (P - 1)) + 1
            M = (M & ~(((1 << 64) - 1) << (P - 65))) | ((1 << 63) << (P - 65))
        else:
            A = (1 << (P - 1)) + rng.choice((1, 3, 5))
            pat = rng.choice((1 << 28, (1 << 28) - 1))
            M = (M & ~(((1 << 29) - 1) << (P - 30))) | (pat << (P - 30))
            if rng.random() < 0.5:
                M &= ~((1 << (P - 30)) - 1)
        a, b = limbs(A), limbs(M)
        if rng.random() < 0.5:
            a, b = b, a
        c0 = sum(a[i] * b[N - 2 - i] for i in range(N - 1))
        c1 = sum(a[i] * b[N - 1 - i] for i in range(N))
        sh = 1 - ((A * M) >> (2 * P - 1))
        X = (((c0 + (c1 << 32)) & ((1 << 64) - 1)) << sh) & ((1 << 64) - 1)
        if (1 << 63) - (1 << 39) - 1 < X <= (1 << 63):
            out.append((a, b))
    return out


def window_aos(prec, count, seed):
    from mpc_cuda_b200 import layout

    pairs = window_operands(prec, count, seed)
    rng = np.random.default_rng(seed)

    def heads():
        return ((rng.integers(-40, 40, count).astype(np.int64) << 1) | rng.integers(0, 2, count)).astype(np.uint32)

    A = layout.aos_from_parts(prec, np.array([p[0] for p in pairs], np.uint32), heads())
    B = layout.aos_from_parts(prec, np.array([p[1] for p in pairs], np.uint32), heads())
    return A, B


@pytest.mark.parametrize("prec", (128, 256, 512, 1024, 2048))
def test_mul_uncertain_window_takes_full_product(orc, mpb, prec):
    """Products whose rounding the upper half of the limb product cannot
    decide (near and exact ties) must still round like MPFR."""
    H = mpb.host_lib()
    A, B = window_aos(prec, 200, prec)
    R = orc.empty(prec, A.shape[0])
    assert H.mpbh_binop(prec, 0, A.shape[0], _p(A), _p(B), _p(R)) == 0
    bad, first = orc.mismatches(prec, R, orc.binop("mul", prec, A, B, "mp"))
    assert bad == 0, f"PB={prec}: {bad} mismatches, first at {first}"


def cancelling_complex_pairs(orc, prec, M, seed):
    """Complex (a, b) pairs whose real part a_r b_r - a_i b_i cancels: b = (y, x)
    for a = (x, y) gives exactly 0, and with the last bit of x flipped in b
    the real part is ~2^-PB below its terms.  The complex multiply cannot
    round these from upper-column products and must use the exact ones."""
    es = orc.elem_bytes(prec)
    A, _ = orc.gen_pairs(prec, M, seed, cplx=True)
    B = A.copy()
    B[:, :es], B[:, es:] = A[:, es:], A[:, :es]
    sb = 64 * (-(-prec // 64)) - prec  # zero padding bits under the significand
    B[1::2, es + 16 + sb // 8] ^= 1 << (sb % 8)  # last significand bit of b's imaginary part (x), every other pair
    return A, B


@pytest.mark.parametrize("prec", (128, 160, 256, 512, 1024, 2048))
def test_cmul_cancellation_uses_exact_products(orc, mpb, prec):
    H = mpb.host_lib()
    A, B = cancelling_complex_pairs(orc, prec, 600, 0x5151 + prec)
    R = orc.empty(prec, A.shape[0], True)
    assert H.mpbh_cbinop(prec, 0, A.shape[0], _p(A), _p(B), _p(R)) == 0
    bad, first = orc.mismatches(prec, R, orc.binop("cmul", prec, A, B, "mp"), True)
    assert bad == 0, f"PB={prec}: {bad} mismatches, first at {first}"


def div_sqrt_cases(orc, prec, M, seed):
    """(A, B, S) AoS operands for division (A / B) and square root (S):
    the reference generator's wide-spread pairs, plus exact and structured
    cases -- a / a, division by powers of two, small integers (1/3, 2/3, ...:
    repeating patterns), perfect squares k^2 and small non-squares."""
    A, B = orc.gen_pairs(prec, M, seed)
    ints = np.arange(1, 65, dtype=np.float64)
    small = orc.from_double(prec, np.concatenate([ints, ints]))
    three = orc.from_double(prec, np.concatenate([np.full(64, 3.0), 2.0 ** np.arange(-32, 32)]))
    A = np.concatenate([A, A[:64], small])
    B = np.concatenate([B, A[:64].copy(), three])
    squares = orc.from_double(prec, np.concatenate([ints ** 2, ints, [0.0]]))
    S = A.copy()
    S[:, 0:4] = np.array([1], np.int32).view(np.uint8)  # |a|
    S = np.concatenate([S, squares])
    return A, B, S


@pytest.mark.parametrize("prec", PRECS)
def test_div_sqrt_correctly_rounded(orc, mpb, prec):
    """cu_fdiv / cu_sqrt round the exact quotient / root once (mpfr_div /
    mpfr_sqrt), unlike the reference's faithful Newton versions."""
    H = mpb.host_lib()
    A, B, S = div_sqrt_cases(orc, prec, 3000 if prec <= 1056 else 800, 0xD1 + prec)
    R = orc.empty(prec, A.shape[0])
    assert H.mpbh_div(prec, A.shape[0], _p(A), _p(B), _p(R)) == 0
    bad, first = orc.mismatches(prec, R, orc.div(prec, A, B))
    assert bad == 0, f"div PB={prec}: {bad} mismatches, first at {first}"
    R = orc.empty(prec, S.shape[0])
    assert H.mpbh_sqrt(prec, S.shape[0], _p(S), _p(R)) == 0
    bad, first = orc.mismatches(prec, R, orc.sqrt(prec, S))
    assert bad == 0, f"sqrt PB={prec}: {bad} mismatches, first at {first}"


@pytest.mark.parametrize("prec", (64, 160, 512))
def test_div_by_zero_and_sqrt_of_negative_give_zero(orc, mpb, prec):
    """The format has no infinities or NaN: a / 0 and sqrt(-a) are 0."""
    H = mpb.host_lib()
    A = orc.from_double(prec, np.array([1.5, -2.0, 0.0]))
    Z = orc.from_double(prec, np.zeros(3))
    R = orc.empty(prec, 3)
    assert H.mpbh_div(prec, 3, _p(A), _p(Z), _p(R)) == 0
    assert orc.mismatches(prec, R, Z)[0] == 0
    assert H.mpbh_sqrt(prec, 1, _p(A[1:2].copy()), _p(R)) == 0
    assert orc.mismatches(prec, R[:1], Z[:1])[0] == 0


def exp_log_cases(orc, prec, M, seed):
    """In-range arguments for exp (doubles in [-8, 8] as in the reference's
    test, plus the wide generator's values below 2^8) and positive ones for
    log (|wide generator| plus values within 2^-10 of 1)."""
    A, _ = orc.gen_pairs(prec, M, seed)
    ea = A[:, 8:16].copy().view(np.int64).ravel()
    rng = np.random.default_rng(seed)
    X = np.concatenate([orc.from_double(prec, rng.uniform(-8, 8, M)), A[(ea <= 8) & (ea >= -300)][: M // 2]])
    Y = A.copy()
    Y[:, 0:4] = np.array([1], np.int32).view(np.uint8)
    Y = np.concatenate([Y, orc.from_double(prec, 1 + rng.uniform(-1e-3, 1e-3, 64))])
    return X, Y


@pytest.mark.parametrize("prec", PRECS)
def test_exp_log_faithful(orc, mpb, prec):
    """cu_exp / cu_log: within 1 ULP of MPFR (the reference's contract); with
    128 guard bits they are in practice correctly rounded, so the results must
    also equal mpfr_exp / mpfr_log on nearly every argument."""
    H = mpb.host_lib()
    X, Y = exp_log_cases(orc, prec, 400 if prec <= 1056 else 100, 0xE1 + prec)
    pref = min(4 * prec, orc.lib().orc_max_prec())
    for name, f, A, ref in (("exp", H.mpbh_exp, X, orc.exp), ("log", H.mpbh_log, Y, orc.log)):
        R = orc.empty(prec, A.shape[0])
        assert f(prec, A.shape[0], _p(A), _p(R)) == 0
        ulp = orc.ulp_errors(prec, R, pref, ref(prec, A, pref))
        assert ulp.max() <= 1.0, f"{name} PB={prec}: {ulp.max():.3f} ULP"
        assert orc.mismatches(prec, R, ref(prec, A))[0] <= A.shape[0] // 100, name


def _negate_complex(orc, prec, Z):
    """-Z for complex AoS elements (flip both components' sign words)."""
    es = orc.elem_bytes(prec)
    out = Z.copy()
    for off in (0, es):
        sgn = out[:, off:off + 4].copy().view(np.int32)
        out[:, off:off + 4] = (-sgn).view(np.uint8)
    return out


@pytest.mark.parametrize("prec", PRECS)
def test_cfma_single_rounding(orc, mpb, prec):
    """cu_cfma: a*b + c with one rounding per component, against the system
    mpc_fma and, independently, mpc_dot over ([a, c], [b, 1]).  Cases: the
    reference generator's wide exponent spreads (terms far apart: the
    round-to-odd branch), c = -round(a*b) (cancellation down to the rounding
    error of the product: the exact branch), a = (x, x) and b = (y, y)
    (the two products cancel exactly in the real part), and zeros."""
    H = mpb.host_lib()
    M = 2000 if prec <= 1056 else 500
    A, B = orc.gen_pairs(prec, M, 0x2222 + prec, cplx=True)
    Cc, _ = orc.gen_pairs(prec, M, 0x3333 + prec, cplx=True)
    es = orc.elem_bytes(prec)
    # near-cancelling addend: -round(a*b)
    AB = orc.empty(prec, M, True)
    assert H.mpbh_cbinop(prec, 0, M, _p(A), _p(B), _p(AB)) == 0
    Cn = _negate_complex(orc, prec, AB)
    # a = (x, x), b = (y, y): re = x*y - x*y = 0 exactly, so re = round(c.re)
    Ax, By = A.copy(), B.copy()
    Ax[:, es:] = Ax[:, :es]
    By[:, es:] = By[:, :es]
    # zeros: every third a, b or c is 0 + 0i
    zero = orc.binop("csub", prec, A[:1], A[:1], "mp")
    Az, Bz, Cz = A.copy(), B.copy(), Cc.copy()
    Az[0::3] = zero
    Bz[1::3] = zero
    Cz[2::3] = zero
    for name, (a, b, c) in {"spread": (A, B, Cc), "cancel": (A, B, Cn), "products cancel": (Ax, By, Cc),
                            "zeros": (Az, Bz, Cz)}.items():
        R = orc.empty(prec, M, True)
        assert H.mpbh_cfma(prec, M, _p(a), _p(b), _p(c), _p(R)) == 0
        want = orc.fma(prec, a, b, c, impl="mp", cplx=True)
        want2 = orc.fma(prec, a, b, c, impl="mpdot", cplx=True)
        assert orc.mismatches(prec, want, want2, True)[0] == 0, f"{name}: mpc_fma and mpc_dot disagree"
        bad, first = orc.mismatches(prec, R, want, True)
        assert bad == 0, f"cfma {name} PB={prec}: {bad} mismatches, first at {first}"


@pytest.mark.parametrize("cplx", (False, True))
@pytest.mark.parametrize("prec", (64, 256, 1024))
def test_axpy_host(orc, mpb, prec, cplx):
    H = mpb.host_lib()
    X, Y = orc.gen_pairs(prec, 2000, 0x99 + prec, cplx)
    a = X[:1].copy()
    Z = orc.empty(prec, 2000, cplx)
    f = H.mpbh_axpy_c if cplx else H.mpbh_axpy_r
    assert f(prec, 2000, _p(a), _p(X), _p(Y), _p(Z)) == 0
    assert orc.mismatches(prec, Z, orc.axpy(prec, a, X, Y, cplx, impl="mp"), cplx)[0] == 0


def test_sample_fixed_known_values(mpb):
    """Known values printed by the reference's sample (demos/sample_fixed.cu:59-67):
    1.5*(1/3)+1.5 and (1.5-0.25i)*(1+0.5i)+(2-1i) at 256 bits."""
    H = mpb.host_lib()
    prec = 256
    es = 16 + prec // 8
    d = np.array([1.5, 1.0 / 3.0], dtype=np.float64)
    v = np.zeros((2, es), dtype=np.uint8)
    assert H.mpbh_from_double(prec, 2, _p(d), _p(v)) == 0
    t = np.zeros((1, es), dtype=np.uint8)
    r = np.zeros((1, es), dtype=np.uint8)
    H.mpbh_binop(prec, 0, 1, _p(v[0:1].copy()), _p(v[1:2].copy()), _p(t))
    H.mpbh_binop(prec, 1, 1, _p(t), _p(v[0:1].copy()), _p(r))
    out = np.zeros(1)
    H.mpbh_to_double(prec, 1, _p(r), _p(out))
    assert out[0] == 1.5 * (1.0 / 3.0) + 1.5
    zd = np.array([1.5, -0.25, 1.0, 0.5, 2.0, -1.0])
    zz = np.zeros((6, es), dtype=np.uint8)
    H.mpbh_from_double(prec, 6, _p(zd), _p(zz))
    za, zx, zy = (zz[0:2].reshape(1, -1).copy(), zz[2:4].reshape(1, -1).copy(), zz[4:6].reshape(1, -1).copy())
    t = np.zeros((1, 2 * es), dtype=np.uint8)
    r = np.zeros((1, 2 * es), dtype=np.uint8)
    H.mpbh_cbinop(prec, 0, 1, _p(za), _p(zx), _p(t))
    H.mpbh_cbinop(prec, 1, 1, _p(t), _p(zy), _p(r))
    out = np.zeros(2)
    H.mpbh_to_double(prec, 2, _p(r.reshape(2, es).copy()), _p(out))
    assert tuple(out) == (3.625, -0.5)


# ---------------------------------------------------------------- elementary functions
def _fmath_host(H, orc, name, prec, A, B=None):
    import fmath_cases as fc

    R = orc.empty(prec, A.shape[0])
    rc = H.mpbh_fmath_r(fc.FN.index(name), prec, A.shape[0], _p(A), _p(B) if B is not None else None, _p(R))
    assert rc == 0
    return R


def _check_faithful(orc, prec, name, R, A, B=None, label="", cr=True):
    """at most 1 ULP from MPFR at 4 PB (the reference's contract); on random
    arguments (cr) also equal to MPFR's correctly rounded value on nearly
    every one -- structured arguments (the hard sets) can sit arbitrarily
    close to a rounding boundary, where a faithful result may differ"""
    pref = min(4 * prec, orc.lib().orc_max_prec())
    ulp = orc.ulp_errors(prec, R, pref, orc.fn(name, prec, A, B, pref))
    assert ulp.max() <= 1.0, f"{name}{label} PB={prec}: {ulp.max():.3g} ULP at {int(ulp.argmax())}"
    if cr:
        bad = orc.mismatches(prec, R, orc.fn(name, prec, A, B))[0]
        assert bad <= A.shape[0] // 100, f"{name}{label} PB={prec}: {bad} not correctly rounded"


@pytest.mark.parametrize("prec", PRECS)
def test_fmath_real_faithful(orc, mpb, prec):
    """cu_exp .. cu_pow (and atan2) on the reference's test ranges
    (tools/test_fmath.cu, test_fmath3.cu) and on the hard argument sets."""
    import fmath_cases as fc

    H = mpb.host_lib()
    M = 120 if prec <= 1056 else 40
    hard = fc.hard_args(orc, prec, 0xF0 + prec)
    for i, name in enumerate(fc.FN):
        A, B = fc.random_args(orc, name, prec, M, 0x3000 + 16 * prec + i)
        _check_faithful(orc, prec, name, _fmath_host(H, orc, name, prec, A, B), A, B)
        if name in hard:
            Hd = hard[name]
            _check_faithful(orc, prec, name, _fmath_host(H, orc, name, prec, Hd), Hd, label=" (hard set)", cr=False)


@pytest.mark.parametrize("prec", PRECS)
def test_fmath_complex_faithful(orc, mpb, prec):
    """cu_cexp .. cu_cdiv: each component within 1 ULP of MPC at 4 PB."""
    import fmath_cases as fc

    H = mpb.host_lib()
    M = 80 if prec <= 1056 else 24
    es, pref = orc.elem_bytes(prec), min(4 * prec, orc.lib().orc_max_prec())
    eo = orc.elem_bytes(pref)
    for i, name in enumerate(fc.CFN):
        A = orc.rand_elems(prec, M, 0x5000 + 16 * prec + i, -3, 3, cplx=True)
        B = orc.rand_elems(prec, M, 0x6000 + 16 * prec + i, -3, 3, cplx=True) if name == "div" else None
        R = orc.empty(prec, M, True)
        assert H.mpbh_fmath_c(i, prec, M, _p(A), _p(B) if B is not None else None, _p(R)) == 0
        ref = orc.cfn(name, prec, A, B, pref)
        for c in (0, 1):
            ulp = orc.ulp_errors(prec, R[:, c * es:(c + 1) * es], pref, ref[:, c * eo:(c + 1) * eo])
            assert ulp.max() <= 1.0, f"c{name} PB={prec} component {c}: {ulp.max():.3g} ULP"
        assert orc.mismatches(prec, R, orc.cfn(name, prec, A, B), True)[0] <= M // 50, f"c{name} PB={prec}"


@pytest.mark.parametrize("prec", (64, 256, 1056))
def test_fmath_special_values(orc, mpb, prec):
    """The documented edges: no value in the format gives 0; the reference's
    asin / acos clamps; exact cases (pow with an integer exponent, cbrt)."""
    import fmath_cases as fc

    H = mpb.host_lib()
    pi = orc.const("pi", prec)

    def scaled_pi(sign, shift):
        e = pi.copy()
        e[0, 0:4] = np.array([sign], np.int32).view(np.uint8)
        e[0, 8:16] = np.array([pi[0, 8:16].view(np.int64)[0] + shift], np.int64).view(np.uint8)
        return e

    named = {"pi": scaled_pi(1, 0), "pi/2": scaled_pi(1, -1), "-pi/2": scaled_pi(-1, -1), "pi/4": scaled_pi(1, -2)}
    for name, args, want in fc.special_args():
        A = orc.from_double(prec, [args[0]])
        B = orc.from_double(prec, [args[1]]) if len(args) > 1 else None
        got = _fmath_host(H, orc, name, prec, A, B)
        exp = named[want] if isinstance(want, str) else orc.from_double(prec, [want])
        assert orc.mismatches(prec, got, exp)[0] == 0, f"{name}{args} PB={prec}"


@pytest.mark.parametrize("prec", PRECS)
def test_div_ui_and_constants(orc, mpb, prec):
    """cu_div_ui (32- and 64-bit divisors) bit-identical to mpfr_div_ui, and
    cu_pi / cu_ln2 to mpfr_const_pi / mpfr_const_log2."""
    H = mpb.host_lib()
    A, _ = orc.gen_pairs(prec, 400, 0xD1 + prec)
    for u in (1, 3, 7, 10, 2 ** 31 + 11, 2 ** 32 - 1, 2 ** 32 + 15, 12345678901234567, 2 ** 64 - 1):
        R = orc.empty(prec, A.shape[0])
        assert H.mpbh_div_ui(prec, A.shape[0], _p(A), u, _p(R)) == 0
        assert orc.mismatches(prec, R, orc.div_ui(prec, A, u))[0] == 0, f"u={u}"
    for k, which in enumerate(("pi", "ln2")):
        R = orc.empty(prec, 1)
        assert H.mpbh_const(k, prec, _p(R)) == 0
        assert orc.mismatches(prec, R, orc.const(which, prec))[0] == 0, which


# ---------------------------------------------------------------- runtime precision
RP_PRECS = (1, 2, 24, 53, 62, 63, 100, 113, 126, 127, 200, 254, 255, 300, 510, 511, 1000, 1022, 1023, 1500, 2046)


def rp_storage(p):
    return next(q for q in (64, 128, 256, 512, 1024, 2048) if q >= p + 2)


def rp_operands(orc, p, n, seed):
    """operands in the storage format: the reference's pairs (exponent spreads
    40 and PB+200) plus a third operand; sqrt gets |a|"""
    pb = rp_storage(p)
    A, B = orc.gen_pairs(pb, n, seed)
    Cc, _ = orc.gen_pairs(pb, n, seed + 1)
    Apos = A.copy()
    Apos[:, 0:4] = np.array([1], np.int32).view(np.uint8)
    return pb, A, Apos, B, Cc


@pytest.mark.parametrize("p", RP_PRECS)
def test_runtime_precision_ops(orc, mpb, p):
    """mul / add / sub / fma / div / sqrt at any precision p (rounded to odd
    at the storage PB, then to nearest at p): bit-identical to MPFR with a
    p-bit destination (the reference's runtime layer, mpfr_cuda/mpfr.h:582-589)."""
    H = mpb.host_lib()
    n = 1500 if p <= 1023 else 400
    pb, A, Apos, B, Cc = rp_operands(orc, p, n, 0x9000 + p)
    for k, op in enumerate(("mul", "add", "sub", "fma", "div", "sqrt")):
        X = Apos if op == "sqrt" else A
        R = orc.empty(pb, n)
        assert H.mpbh_op_rp(k, p, n, _p(X), _p(B), _p(Cc), _p(R)) == 0
        bad, first = orc.mismatches(pb, R, orc.op_rp(op, p, pb, X, B, Cc))
        assert bad == 0, f"{op} p={p}: {bad} mismatches, first at {first}"
