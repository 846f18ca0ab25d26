"""GPU parity: every engine entry point, called through the C ABI, against the
CPU oracle -- bit for bit (integer arithmetic: no tolerance).

Operands follow the reference's test method (seeded xorshift pairs with
exponent spreads 40 / PB+200, tools/test_freal.cu:17-27,55) and the
benchmark workloads' value distributions; expected results come from the
system MPFR/MPC (``mp_*``) or the oracle's restatement (``orc_*``), which
tests/test_oracle.py pins to each other and to the reference headers.
"""
import numpy as np
import pytest

from conftest import to_dev, to_host
from mpc_cuda_b200 import layout, synth

pytestmark = pytest.mark.gpu
PRECS = layout.SUPPORTED


def dvec(prec, aos, cplx=False):
    return to_dev(layout.aos_to_vec(prec, aos, cplx))


def hvec(prec, t, n, cplx=False):
    return layout.vec_to_aos(prec, to_host(t), n, cplx)


def zero_aos(prec, n, cplx=False):
    z = np.zeros((n, layout.aos_bytes(prec)), np.uint8)
    z[:, 0:4] = np.array([1], np.int32).view(np.uint8)
    z[:, 8:16] = np.array([layout.AOS_ZERO_EXP], np.int64).view(np.uint8)
    return np.concatenate([z, z], axis=1) if cplx else z


def pad_rows(prec, A, rows, cols, ld, cplx=False):
    """AoS rows x cols -> AoS rows x ld with zero elements in the padding."""
    es = A.shape[1]
    out = np.repeat(zero_aos(prec, 1, cplx), rows * ld, axis=0).reshape(rows, ld, es)
    out[:, :cols] = A.reshape(rows, cols, es)
    return out.reshape(rows * ld, es)


def unpad_rows(A, rows, cols, ld):
    es = A.shape[1]
    return A.reshape(rows, ld, es)[:, :cols].reshape(rows * cols, es)


@pytest.mark.parametrize("prec", PRECS)
def test_binops_real(orc, mpb, prec):
    M = 100000 if prec <= 1024 else 30000  # 100k pairs as in tools/test_freal.cu:89
    A, B = orc.gen_pairs(prec, M, 0xBEEF + prec)
    a, b, r = dvec(prec, A), dvec(prec, B), mpb.empty(prec, M)
    for op, kind in enumerate(("mul", "add", "sub")):
        mpb.binop(prec, op, M, a, b, r)
        bad, first = orc.mismatches(prec, hvec(prec, r, M), orc.binop(kind, prec, A, B, "mp"))
        assert bad == 0, f"{kind} PB={prec}: {bad} mismatches, first at {first}"
    Cc, _ = orc.gen_pairs(prec, M, 0xFACE + prec)
    mpb.fma(prec, M, a, b, dvec(prec, Cc), r)
    bad, first = orc.mismatches(prec, hvec(prec, r, M), orc.fma(prec, A, B, Cc, "mp"))
    assert bad == 0, f"fma PB={prec}: {bad} mismatches, first at {first}"


@pytest.mark.parametrize("prec", (128, 256, 512, 1024, 2048))
def test_mul_uncertain_window(orc, mpb, prec):
    """Products next to a rounding midpoint (exact ties included): the kernel
    must fall back from the upper-column product to the full one."""
    from test_host_dropin import window_aos

    A, B = window_aos(prec, 2000, prec + 1)
    M = A.shape[0]
    r = mpb.empty(prec, M)
    mpb.binop(prec, 0, M, dvec(prec, A), dvec(prec, B), r)
    bad, first = orc.mismatches(prec, hvec(prec, r, M), orc.binop("mul", prec, A, B, "mp"))
    assert bad == 0, f"PB={prec}: {bad} mismatches, first at {first}"


@pytest.mark.parametrize("prec", (128, 256, 512, 1024, 2048))
def test_cmul_cancellation(orc, mpb, prec):
    """Complex products whose real part cancels exactly or down to ~2^-PB:
    the kernel must fall back from upper-column products to exact ones."""
    from test_host_dropin import cancelling_complex_pairs

    A, B = cancelling_complex_pairs(orc, prec, 4000, 0x7171 + prec)
    M = A.shape[0]
    r = mpb.empty(prec, M, True)
    mpb.binop(prec, 0, M, dvec(prec, A, True), dvec(prec, B, True), r, cplx=True)
    bad, first = orc.mismatches(prec, hvec(prec, r, M, True), orc.binop("cmul", prec, A, B, "mp"), True)
    assert bad == 0, f"PB={prec}: {bad} mismatches, first at {first}"


@pytest.mark.parametrize("prec", PRECS)
def test_div_sqrt(orc, mpb, prec):
    """mpb_div_r / mpb_sqrt_r (the drop-in cu_fdiv / cu_sqrt): one rounding,
    bit-exact with mpfr_div / mpfr_sqrt, on wide-spread pairs and exact cases."""
    from test_host_dropin import div_sqrt_cases

    A, B, S = div_sqrt_cases(orc, prec, 20000 if prec <= 1024 else 4000, 0xD5 + prec)
    M = A.shape[0]
    r = mpb.empty(prec, M)
    mpb.div(prec, M, dvec(prec, A), dvec(prec, B), r)
    bad, first = orc.mismatches(prec, hvec(prec, r, M), orc.div(prec, A, B))
    assert bad == 0, f"div PB={prec}: {bad} mismatches, first at {first}"
    M = S.shape[0]
    r = mpb.empty(prec, M)
    mpb.sqrt(prec, M, dvec(prec, S), r)
    bad, first = orc.mismatches(prec, hvec(prec, r, M), orc.sqrt(prec, S))
    assert bad == 0, f"sqrt PB={prec}: {bad} mismatches, first at {first}"


@pytest.mark.parametrize("prec", PRECS)
def test_exp_log(orc, mpb, prec):
    """mpb_exp_r / mpb_log_r: within 1 ULP of MPFR, and bit-identical to the
    host build of the same drop-in functions."""
    import ctypes as C

    from test_host_dropin import exp_log_cases

    H = mpb.host_lib()
    X, Y = exp_log_cases(orc, prec, 2000 if prec <= 512 else 400, 0xE5 + prec)
    pref = min(4 * prec, orc.lib().orc_max_prec())
    for name, f, hf, A, ref in (("exp", mpb.exp, H.mpbh_exp, X, orc.exp), ("log", mpb.log, H.mpbh_log, Y, orc.log)):
        M = A.shape[0]
        r = mpb.empty(prec, M)
        f(prec, M, dvec(prec, A), r)
        got = hvec(prec, r, M)
        ulp = orc.ulp_errors(prec, got, pref, ref(prec, A, pref))
        assert ulp.max() <= 1.0, f"{name} PB={prec}: {ulp.max():.3f} ULP"
        host = orc.empty(prec, M)
        hf(prec, M, A.ctypes.data_as(C.c_void_p), host.ctypes.data_as(C.c_void_p))
        assert orc.mismatches(prec, got, host)[0] == 0, f"{name} PB={prec}: device differs from host build"


@pytest.mark.parametrize("prec", PRECS)
def test_binops_complex(orc, mpb, prec):
    M = 30000 if prec <= 1024 else 6000
    A, B = orc.gen_pairs(prec, M, 0xC0DE + prec, cplx=True)
    a, b, r = dvec(prec, A, True), dvec(prec, B, True), mpb.empty(prec, M, True)
    for op, kind in enumerate(("cmul", "cadd", "csub")):
        mpb.binop(prec, op, M, a, b, r, cplx=True)
        bad, first = orc.mismatches(prec, hvec(prec, r, M, True), orc.binop(kind, prec, A, B, "mp"), True)
        assert bad == 0, f"{kind} PB={prec}: {bad} mismatches, first at {first}"


@pytest.mark.parametrize("prec", PRECS)
def test_fma_complex(orc, mpb, prec):
    """mpb_fma_c (the drop-in cu_cfma): one rounding per component, against the
    system mpc_fma, on the reference generator's wide-spread pairs and on
    c = -round(a*b), whose sums cancel down to the product's rounding error."""
    M = 20000 if prec <= 1024 else 4000
    A, B = orc.gen_pairs(prec, M, 0xCF + prec, cplx=True)
    Cc, _ = orc.gen_pairs(prec, M, 0xFC + prec, cplx=True)
    a, b, r = dvec(prec, A, True), dvec(prec, B, True), mpb.empty(prec, M, True)
    AB = orc.binop("cmul", prec, A, B, "mp")
    es = layout.aos_bytes(prec)
    Cn = AB.copy()
    for off in (0, es):
        Cn[:, off:off + 4] = (-Cn[:, off:off + 4].copy().view(np.int32)).view(np.uint8)
    for name, C in (("spread", Cc), ("cancel", Cn)):
        mpb.fma(prec, M, a, b, dvec(prec, C, True), r, cplx=True)
        bad, first = orc.mismatches(prec, hvec(prec, r, M, True), orc.fma(prec, A, B, C, "mp", cplx=True), True)
        assert bad == 0, f"cfma {name} PB={prec}: {bad} mismatches, first at {first}"


@pytest.mark.parametrize("cplx", (False, True))
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("n", (1, 31, 33, 1000))
def test_pack_unpack_and_ragged_sizes(orc, mpb, prec, n, cplx):
    import torch

    A, _ = orc.gen_pairs(prec, n, 0x51 + n, cplx)
    aos = torch.from_numpy(A.reshape(-1).copy()).cuda()
    v = mpb.empty(prec, n, cplx)
    mpb.pack_aos(prec, n, aos, v, cplx)
    assert np.array_equal(to_host(v)[: layout.vec_bytes(prec, n, cplx)], layout.aos_to_vec(prec, A, cplx))
    back = torch.zeros_like(aos)
    mpb.unpack_aos(prec, n, v, back, cplx)
    assert np.array_equal(to_host(back).reshape(A.shape), A)


@pytest.mark.parametrize("prec", PRECS)
def test_double_conversions(orc, mpb, prec):
    import torch

    rng = np.random.default_rng(prec)
    d = np.concatenate([rng.uniform(-1, 1, 5000), [0.0, 1.5, -1e-300, 3e300, 2.0**-1022]])
    n = d.size
    td = torch.from_numpy(d).cuda()
    v = mpb.empty(prec, n)
    mpb.from_double(prec, n, td, v)
    ref = orc.empty(prec, n)
    orc.lib().orc_from_double(prec, n, d.ctypes.data, ref.ctypes.data)
    assert orc.mismatches(prec, hvec(prec, v, n), ref)[0] == 0
    # to_double of random full-width values (overflow/underflow included):
    # same rounding as the host build of the drop-in surface and the reference
    A, _ = orc.gen_pairs(prec, 4000, 3 + prec)
    out = torch.zeros(4000, dtype=torch.float64, device="cuda")
    mpb.to_double(prec, 4000, dvec(prec, A), out)
    exp = np.zeros(4000)
    mpb.host_lib().mpbh_to_double(prec, 4000, A.ctypes.data, exp.ctypes.data)
    assert np.array_equal(out.cpu().numpy(), exp)
    if orc.ref_available():
        exp2 = np.zeros(4000)
        orc.ref().ref_to_double(prec, 4000, A.ctypes.data, exp2.ctypes.data)
        assert np.array_equal(exp, exp2)


@pytest.mark.parametrize("cplx", (False, True))
@pytest.mark.parametrize("prec", PRECS)
def test_axpy_reference_pairs(orc, mpb, prec, cplx):
    n = 20000 if prec <= 1024 else 4000
    X, Y = orc.gen_pairs(prec, n, 0xA0 + prec, cplx)
    a = X[7:8].copy()
    z = mpb.empty(prec, n, cplx)
    mpb.axpy(prec, n, dvec(prec, a, cplx), dvec(prec, X, cplx), dvec(prec, Y, cplx), z, cplx)
    bad, first = orc.mismatches(prec, hvec(prec, z, n, cplx), orc.axpy(prec, a, X, Y, cplx, impl="mp"), cplx)
    assert bad == 0, f"axpy PB={prec} cplx={cplx}: first mismatch {first}"


def test_axpy_real_pb256_full_size(orc, mpb):
    """The real AXPY workload at full size (PB=256, n=2^20, a=1.5, FP64 inputs)."""
    prec, n = 256, 1 << 20
    a, x, y = synth.axpy_r256(n=n)
    A, X, Y = (layout.aos_from_parts(prec, *p) for p in (a, x, y))
    z = mpb.empty(prec, n)
    mpb.axpy(prec, n, to_dev(layout.vec_from_parts(prec, *a)), to_dev(layout.vec_from_parts(prec, *x)),
             to_dev(layout.vec_from_parts(prec, *y)), z)
    bad, first = orc.mismatches(prec, hvec(prec, z, n), orc.axpy(prec, A, X, Y))
    assert bad == 0, f"first mismatch {first}"


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("scalar", (1.5, 3.0, -0.1, 2.0 ** -700, 1e300, -7.0 / 3.0, 0.0))
def test_axpy_short_scalar(orc, mpb, prec, scalar):
    """Scalars with one or two nonzero limbs (small integers, doubles) take the
    exact short product in the real AXPY; x and y are full random operands.
    With a = 1.5 or 3 a quarter of the products drop exactly half an ULP, so
    the ties-to-even path is exercised too."""
    n = 20000 if prec <= 1024 else 4000
    X, Y = orc.gen_pairs(prec, n, 0xA5 + prec)
    a = orc.from_double(prec, [scalar])
    z = mpb.empty(prec, n)
    mpb.axpy(prec, n, dvec(prec, a), dvec(prec, X), dvec(prec, Y), z)
    bad, first = orc.mismatches(prec, hvec(prec, z, n), orc.axpy(prec, a, X, Y, impl="mp"))
    assert bad == 0, f"axpy PB={prec} a={scalar}: first mismatch {first}"


def test_axpy_complex_pb1024_full_size(orc, mpb):
    """The complex AXPY workload at full size (PB=1024, n=2^18, 1% zeros)."""
    prec, n = 1024, 1 << 18
    a, x, y = synth.axpy_c1024(n=n)
    A, X, Y = (synth.interleave_complex(prec, *p) for p in (a, x, y))
    z = mpb.empty(prec, n, True)
    mpb.axpy(prec, n, dvec(prec, A, True), dvec(prec, X, True), dvec(prec, Y, True), z, cplx=True)
    bad, first = orc.mismatches(prec, hvec(prec, z, n, True), orc.axpy(prec, A, X, Y, True), True)
    assert bad == 0, f"first mismatch {first}"


@pytest.mark.parametrize("cplx", (False, True))
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("warps", (4, 16))
def test_gemm_plain_block_shapes(orc, mpb, prec, warps, cplx):
    """every block shape of the plain GEMM (mpb_set_gemm_warps) gives the MPFR/MPC result"""
    m, n, k = (37, 70, 19) if prec <= 1024 else (9, 33, 7)
    A, _ = orc.gen_pairs(prec, m * k, 0x63 + warps + prec, cplx)
    B, _ = orc.gen_pairs(prec, k * n, 0x64 + warps + prec, cplx)
    lda, ldb, ldc = (-(-k // 32) * 32, -(-n // 32) * 32, -(-n // 32) * 32)
    Cd = mpb.empty(prec, m * ldc, cplx)
    old = mpb.get_gemm_warps(prec, cplx)
    try:
        mpb.set_gemm_warps(prec, warps, cplx)
        mpb.gemm(prec, m, n, k, dvec(prec, pad_rows(prec, A, m, k, lda, cplx), cplx), lda,
                 dvec(prec, pad_rows(prec, B, k, n, ldb, cplx), cplx), ldb, Cd, ldc, cplx)
    finally:
        mpb.set_gemm_warps(prec, old, cplx)
    got = unpad_rows(hvec(prec, Cd, m * ldc, cplx), m, n, ldc)
    exp = orc.gemm(prec, m, n, k, A, k, B, n, cplx, impl="mp")
    bad, first = orc.mismatches(prec, got, exp, cplx)
    assert bad == 0, f"gemm PB={prec} warps={warps}: first mismatch {first}"


@pytest.mark.parametrize("cplx", (False, True))
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("shape", ((1, 1, 1), (5, 7, 33), (33, 40, 17), (64, 64, 64)))
def test_gemm_plain(orc, mpb, prec, shape, cplx):
    m, n, k = shape
    if prec == 2048 and m * n * k > 40000:
        pytest.skip("covered at smaller shapes")
    A, _ = orc.gen_pairs(prec, m * k, 0x61 + m + prec, cplx)
    B, _ = orc.gen_pairs(prec, k * n, 0x62 + n + prec, cplx)
    lda, ldb, ldc = (-(-k // 32) * 32, -(-n // 32) * 32, -(-n // 32) * 32)
    Cd = mpb.empty(prec, m * ldc, cplx)
    mpb.gemm(prec, m, n, k, dvec(prec, pad_rows(prec, A, m, k, lda, cplx), cplx), lda,
             dvec(prec, pad_rows(prec, B, k, n, ldb, cplx), cplx), ldb, Cd, ldc, cplx)
    got = unpad_rows(hvec(prec, Cd, m * ldc, cplx), m, n, ldc)
    exp = orc.gemm(prec, m, n, k, A, k, B, n, cplx, impl="mp")
    bad, first = orc.mismatches(prec, got, exp, cplx)
    assert bad == 0, f"gemm PB={prec} {shape}: first mismatch {first}"


@pytest.mark.parametrize("cplx", (False, True))
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("shape", ((1, 1), (16, 17), (37, 70), (130, 33)))
def test_gemv_plain(orc, mpb, prec, shape, cplx):
    m, n = shape
    A, _ = orc.gen_pairs(prec, m * n, 0x71 + m + prec, cplx)
    x, _ = orc.gen_pairs(prec, n, 0x72 + n, cplx)
    y, _ = orc.gen_pairs(prec, m, 0x73 + m, cplx)
    lda = -(-n // 32) * 32
    yo = mpb.empty(prec, m, cplx)
    mpb.gemv(prec, m, n, dvec(prec, pad_rows(prec, A, m, n, lda, cplx), cplx), lda, dvec(prec, x, cplx),
             dvec(prec, y, cplx), yo, cplx)
    exp = orc.gemv(prec, m, n, A, n, x, y, cplx, impl="mp")
    bad, first = orc.mismatches(prec, hvec(prec, yo, m, cplx), exp, cplx)
    assert bad == 0, f"gemv PB={prec} {shape}: first mismatch {first}"


def test_gemm_real_pb512_rows_sample(orc, mpb):
    """The 1024^3 PB=512 matmul workload at full size; a row sample is checked
    against the oracle (the whole product is ~1e9 MPFR multiply-adds)."""
    prec, m, n, k = 512, 1024, 1024, 1024
    (al, ah), (bl, bh) = synth.gemm_r512()
    Cd = mpb.empty(prec, m * n)
    mpb.gemm(prec, m, n, k, to_dev(layout.vec_from_parts(prec, al, ah)), k,
             to_dev(layout.vec_from_parts(prec, bl, bh)), n, Cd, n)
    got = hvec(prec, Cd, m * n)
    A, B = layout.aos_from_parts(prec, al, ah), layout.aos_from_parts(prec, bl, bh)
    rows = (0, 4)
    exp = orc.gemm(prec, m, n, k, A, k, B, n, rows=rows)
    es = got.shape[1]
    sel = slice(rows[0] * n, rows[1] * n)
    assert orc.mismatches(prec, got[sel], exp[sel])[0] == 0
    last = orc.gemm(prec, m, n, k, A, k, B, n, rows=(m - 2, m))
    assert orc.mismatches(prec, got[(m - 2) * n:], last[(m - 2) * n:])[0] == 0
    assert es == layout.aos_bytes(prec)


# ---------------------------------------------------------------- elementary functions
def _fmath_args(orc, prec, seed):
    """per function: random arguments in the reference's ranges plus the hard set"""
    import fmath_cases as fc

    M = 600 if prec <= 512 else 160
    hard = fc.hard_args(orc, prec, seed)
    out = {}
    for i, name in enumerate(fc.FN):
        A, B = fc.random_args(orc, name, prec, M, seed + 7 * i)
        if name in hard:
            A = np.concatenate([A, hard[name]])
        elif B is not None:
            A2, B2 = fc.random_args(orc, name, prec, 64, seed + 7 * i + 3)
            A, B = np.concatenate([A, A2]), np.concatenate([B, B2])
        out[name] = (A, B)
    return out


@pytest.mark.parametrize("prec", PRECS)
def test_fmath_real(orc, mpb, prec):
    """mpb_fmath_r, every function: bit-identical to the host build of the
    same drop-in functions (which tests/test_host_dropin.py holds to MPFR),
    and within 1 ULP of MPFR at 4 PB."""
    import ctypes as C

    import fmath_cases as fc

    H = mpb.host_lib()
    pref = min(4 * prec, orc.lib().orc_max_prec())
    for name, (A, B) in _fmath_args(orc, prec, 0x7100 + prec).items():
        M = A.shape[0]
        r = mpb.empty(prec, M)
        mpb.fmath(name, prec, M, dvec(prec, A), r, b=dvec(prec, B) if B is not None else None)
        got = hvec(prec, r, M)
        host = orc.empty(prec, M)
        H.mpbh_fmath_r(fc.FN.index(name), prec, M, A.ctypes.data_as(C.c_void_p),
                       B.ctypes.data_as(C.c_void_p) if B is not None else None, host.ctypes.data_as(C.c_void_p))
        bad, first = orc.mismatches(prec, got, host)
        assert bad == 0, f"{name} PB={prec}: device differs from host build at {first}"
        ulp = orc.ulp_errors(prec, got, pref, orc.fn(name, prec, A, B, pref))
        assert ulp.max() <= 1.0, f"{name} PB={prec}: {ulp.max():.3g} ULP"


@pytest.mark.parametrize("prec", PRECS)
def test_fmath_complex(orc, mpb, prec):
    """mpb_fmath_c, every function: bit-identical to the host build, each
    component within 1 ULP of MPC at 4 PB."""
    import ctypes as C

    import fmath_cases as fc

    H = mpb.host_lib()
    M = 300 if prec <= 512 else 80
    es, pref = orc.elem_bytes(prec), min(4 * prec, orc.lib().orc_max_prec())
    eo = orc.elem_bytes(pref)
    for i, name in enumerate(fc.CFN):
        A = orc.rand_elems(prec, M, 0x7300 + 16 * prec + i, -3, 3, cplx=True)
        B = orc.rand_elems(prec, M, 0x7400 + 16 * prec + i, -3, 3, cplx=True) if name == "div" else None
        r = mpb.empty(prec, M, True)
        mpb.cfmath(name, prec, M, dvec(prec, A, True), r, b=dvec(prec, B, True) if B is not None else None)
        got = hvec(prec, r, M, True)
        host = orc.empty(prec, M, True)
        H.mpbh_fmath_c(i, prec, M, A.ctypes.data_as(C.c_void_p), B.ctypes.data_as(C.c_void_p) if B is not None else None,
                       host.ctypes.data_as(C.c_void_p))
        assert orc.mismatches(prec, got, host, True)[0] == 0, f"c{name} PB={prec}: device differs from host build"
        ref = orc.cfn(name, prec, A, B, pref)
        for c in (0, 1):
            ulp = orc.ulp_errors(prec, got[:, c * es:(c + 1) * es], pref, ref[:, c * eo:(c + 1) * eo])
            assert ulp.max() <= 1.0, f"c{name} PB={prec} component {c}: {ulp.max():.3g} ULP"


@pytest.mark.parametrize("prec", PRECS)
def test_div_ui_and_constants(orc, mpb, prec):
    """mpb_div_ui_r and mpb_const_r bit-identical to mpfr_div_ui and
    mpfr_const_pi / mpfr_const_log2."""
    A, _ = orc.gen_pairs(prec, 3000, 0xD7 + prec)
    a = dvec(prec, A)
    for u in (3, 10, 2 ** 32 - 1, 2 ** 40 + 3, 2 ** 64 - 1):
        r = mpb.empty(prec, A.shape[0])
        mpb.div_ui(prec, A.shape[0], a, u, r)
        assert orc.mismatches(prec, hvec(prec, r, A.shape[0]), orc.div_ui(prec, A, u))[0] == 0, f"u={u}"
    for which in ("pi", "ln2"):
        r = mpb.empty(prec, 40)
        mpb.const(which, prec, 40, r)
        want = np.repeat(orc.const(which, prec), 40, axis=0)
        assert orc.mismatches(prec, hvec(prec, r, 40), want)[0] == 0, which


@pytest.mark.parametrize("p", (2, 53, 63, 113, 200, 255, 300, 511, 1000, 1023, 2046))
def test_runtime_precision_ops(orc, mpb, p):
    """mpb_op_rp: every operation at precision p bit-identical to MPFR with a
    p-bit destination (storage format PB = mpb_storage_prec(p))."""
    from test_host_dropin import rp_operands

    n = 4000 if p <= 1023 else 1000
    pb, A, Apos, B, Cc = rp_operands(orc, p, n, 0x9100 + p)
    assert mpb.storage_prec(p) == pb
    b, c = dvec(pb, B), dvec(pb, Cc)
    for op in mpb.RP_OPS:
        X = Apos if op == "sqrt" else A
        r = mpb.empty(pb, n)
        mpb.op_rp(op, p, n, dvec(pb, X), r, b=b, c=c)
        bad, first = orc.mismatches(pb, hvec(pb, r, n), orc.op_rp(op, p, pb, X, B, Cc))
        assert bad == 0, f"{op} p={p}: {bad} mismatches, first at {first}"
