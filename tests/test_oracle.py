"""Pin the CPU oracle before trusting it.

The oracle's C restatement of the reference arithmetic (``orc_*``) must agree
bit for bit with

* the system MPFR 4.2.1 / MPC 1.3.1 (``mp_*``), on the reference's own seeded
  property tests (tools/test_freal.cu:86-105, tools/test_fcomplex.cu:82-101:
  xorshift seeds per precision, exponent spread 40 / PB+200, 100k pairs there,
  fewer here to keep the CPU suite short);
* the reference's own headers compiled for the host (``ref_*``,
  oracle/_ref/libref_host.so) when that build is present;

and the correctly rounded dot (``orc_gemm_exact_*``) must equal mpfr_dot /
mpc_dot.  The reference commits no golden vectors; tests/golden holds vectors
produced by its own headers (see tests/golden/make_golden.py).
"""
import numpy as np
import pytest

PRECS = (32, 64, 96, 128, 160, 256, 288, 512, 1024, 1056, 2048)
# seeds of tools/test_freal.cu:92-102 and tools/test_fcomplex.cu:92-101
REAL_SEEDS = dict(zip(PRECS, (0x1111, 0x2222, 0x3333, 0x4444, 0x5555, 0x6666, 0x7777, 0x8888, 0x9999, 0xAAAA, 0xBBBB)))
CPLX_SEEDS = {32: 0x11, 96: 0x33, 128: 0x44, 160: 0x55, 256: 0x66, 288: 0x77, 512: 0x88, 1024: 0x99, 1056: 0xAA,
              2048: 0xBB, 64: 0x22}


def test_versions(orc):
    mpfr, mpc = orc.versions()
    assert mpfr.startswith("4.2") and mpc.startswith("1.3")


@pytest.mark.parametrize("prec", PRECS)
def test_real_ops_vs_mpfr(orc, prec):
    M = 20000 if prec <= 1056 else 6000
    A, B = orc.gen_pairs(prec, M, REAL_SEEDS[prec])
    for kind in ("mul", "add", "sub"):
        bad, first = orc.mismatches(prec, orc.binop(kind, prec, A, B, "orc"), orc.binop(kind, prec, A, B, "mp"))
        assert bad == 0, f"{kind} PB={prec}: {bad} mismatches, first at {first}"


@pytest.mark.parametrize("prec", PRECS)
def test_complex_ops_vs_mpc(orc, prec):
    M = 5000 if prec <= 1056 else 1500
    A, B = orc.gen_pairs(prec, M, CPLX_SEEDS[prec], cplx=True)
    for kind in ("cmul", "cadd", "csub"):
        bad, first = orc.mismatches(prec, orc.binop(kind, prec, A, B, "orc"), orc.binop(kind, prec, A, B, "mp"), True)
        assert bad == 0, f"{kind} PB={prec}: {bad} mismatches, first at {first}"


@pytest.mark.parametrize("prec", (64, 256, 512, 1024, 2048))
def test_fma_vs_mpfr(orc, prec):
    A, B = orc.gen_pairs(prec, 8000, 0xF00 + prec)
    Cc, _ = orc.gen_pairs(prec, 8000, 0xF11 + prec)
    bad, first = orc.mismatches(prec, orc.fma(prec, A, B, Cc, "orc"), orc.fma(prec, A, B, Cc, "mp"))
    assert bad == 0, f"fma PB={prec}: first mismatch {first}"


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference host build not present")
@pytest.mark.parametrize("prec", PRECS)
def test_restatement_vs_reference_headers(orc, prec):
    M = 10000 if prec <= 1056 else 3000
    A, B = orc.gen_pairs(prec, M, REAL_SEEDS[prec] ^ 0x5A5A)
    for kind in ("mul", "add", "sub"):
        bad, first = orc.mismatches(prec, orc.binop(kind, prec, A, B, "orc"), orc.binop(kind, prec, A, B, "ref"))
        assert bad == 0, f"{kind} PB={prec} vs reference: first mismatch {first}"
    Ac, Bc = orc.gen_pairs(prec, M // 4, CPLX_SEEDS[prec] ^ 0x5A, cplx=True)
    for kind in ("cmul", "cadd", "csub"):
        bad, first = orc.mismatches(prec, orc.binop(kind, prec, Ac, Bc, "orc"), orc.binop(kind, prec, Ac, Bc, "ref"),
                                    True)
        assert bad == 0, f"{kind} PB={prec} vs reference: first mismatch {first}"


@pytest.mark.parametrize("cplx", (False, True))
@pytest.mark.parametrize("prec", (64, 256, 512, 1024))
def test_loops_vs_mpfr_and_reference(orc, prec, cplx):
    n = 1500
    X, Y = orc.gen_pairs(prec, n, 0x77 + prec, cplx)
    a = X[:1].copy()
    z = orc.axpy(prec, a, X, Y, cplx)
    assert orc.mismatches(prec, z, orc.axpy(prec, a, X, Y, cplx, impl="mp"), cplx)[0] == 0
    m, k, nn = 9, 33, 7
    A, _ = orc.gen_pairs(prec, m * k, 11, cplx)
    B, _ = orc.gen_pairs(prec, k * nn, 12, cplx)
    x, _ = orc.gen_pairs(prec, k, 13, cplx)
    y0, _ = orc.gen_pairs(prec, m, 14, cplx)
    g = orc.gemm(prec, m, nn, k, A, k, B, nn, cplx)
    assert orc.mismatches(prec, g, orc.gemm(prec, m, nn, k, A, k, B, nn, cplx, impl="mp"), cplx)[0] == 0
    v = orc.gemv(prec, m, k, A, k, x, y0, cplx)
    assert orc.mismatches(prec, v, orc.gemv(prec, m, k, A, k, x, y0, cplx, impl="mp"), cplx)[0] == 0
    e = orc.gemm_exact(prec, m, nn, k, A, k, B, nn, cplx)
    assert orc.mismatches(prec, e, orc.gemm_exact(prec, m, nn, k, A, k, B, nn, cplx, impl="mp"), cplx)[0] == 0
    if orc.ref_available():
        assert orc.mismatches(prec, z, orc.axpy(prec, a, X, Y, cplx, impl="ref"), cplx)[0] == 0
        assert orc.mismatches(prec, g, orc.gemm(prec, m, nn, k, A, k, B, nn, cplx, impl="ref"), cplx)[0] == 0
        assert orc.mismatches(prec, v, orc.gemv(prec, m, k, A, k, x, y0, cplx, impl="ref"), cplx)[0] == 0


@pytest.mark.parametrize("prec", (64, 512))
def test_exact_dot_ulp_bound(orc, prec):
    """One rounding of the exact dot: <= 0.5 ULP against a 4*PB oracle."""
    m, k, nn = 6, 40, 5
    A, _ = orc.gen_pairs(prec, m * k, 21)
    B, _ = orc.gen_pairs(prec, k * nn, 22)
    e = orc.gemm_exact(prec, m, nn, k, A, k, B, nn)
    e4 = orc.gemm_exact(prec, m, nn, k, A, k, B, nn, out_prec=4 * prec)
    u = orc.ulp_errors(prec, e, 4 * prec, e4)
    assert u.max() <= 0.5


def test_planted_mistake_is_caught(orc):
    """A single flipped bit in an oracle result must be reported."""
    prec = 256
    A, B = orc.gen_pairs(prec, 100, 5)
    r = orc.binop("mul", prec, A, B, "orc")
    r2 = r.copy()
    r2[37, 16] ^= 1  # lowest limb bit of element 37
    assert orc.mismatches(prec, r, r2) == (1, 37)
