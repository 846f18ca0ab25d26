"""The drop-in cu_fp surface on the GPU: user kernels compiled through the
drop-in headers (tests/dropin/user_kernels.cu, written as the reference's
callers write them: demos/bench_3way.cu:44-59, tools/linalg_fast.cu:54-68,
tools/axpy_fast_complex.cu:32-40, tools/test_freal.cu:42-48) run on the B200
at the reference's test precisions, including the ones whose last 64-bit limb
is half used (96, 160, 288, 1056 bits; tools/test_freal.cu:86-105).

Checked against the system MPFR / MPC, bit for bit (integer arithmetic, no
tolerance): real and complex AXPY, the sequential-k real and complex matmul
(one rounding per operation, in k order), the correctly rounded division; the
faithful exponential within 1 ULP of MPFR and bit-identical to the host build
of the same header.  The same kernels built against the reference's own
headers (oracle/_ref/libref_user_kernels.so) run beside them on the same data,
as a second check of both and as the timing baseline of the bench.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
PRECS = (64, 96, 128, 160, 256, 288, 512, 1024, 1056, 2048)
FN_PRECS = PRECS[:-1]
UK_PATH = os.path.join(ROOT, "tests", "dropin", "libuser_kernels.so")
REF_UK_PATH = os.path.join(ROOT, "oracle", "_ref", "libref_user_kernels.so")

_I, _L, _V, _D = C.c_int, C.c_long, C.c_void_p, C.c_double


def _bind(path, pre):
    L = C.CDLL(path)
    getattr(L, pre + "axpy_r").argtypes = [_I, _L, _V, _V, _V, _V, _I, _I, _V]
    getattr(L, pre + "axpy_c").argtypes = [_I, _L, _V, _V, _V, _V, _I, _I, _V]
    getattr(L, pre + "axpy_d").argtypes = [_I, _L, _D, _V, _V, _V, _I, _I, _V]
    getattr(L, pre + "caxpy_d").argtypes = [_I, _L, _D, _D] + [_V] * 6 + [_I, _I, _V]
    for f in ("matmul_r", "matmul_c"):
        getattr(L, pre + f).argtypes = [_I, _I, _I, _I, _V, _I, _V, _I, _V, _I, _I, _I, _V]
    getattr(L, pre + "exp").argtypes = [_I, _L, _V, _V, _I, _I, _V]
    getattr(L, pre + "div").argtypes = [_I, _L, _V, _V, _V, _I, _I, _V]
    return L


@pytest.fixture(scope="module")
def uk():
    if not os.path.exists(UK_PATH):
        raise RuntimeError(f"{UK_PATH} is missing: run __graft_entry__.build()")
    return _bind(UK_PATH, "uk_")


@pytest.fixture(scope="module")
def refuk():
    if not os.path.exists(REF_UK_PATH):
        pytest.skip("the reference headers' user-kernel build (oracle/_ref) is not present")
    return _bind(REF_UK_PATH, "refuk_")


class _Dev:
    """AoS arrays on the device (torch memory), copied back as numpy uint8 rows."""

    def __init__(self):
        import torch

        self.torch = torch
        self.keep = []

    def put(self, a):
        t = self.torch.from_numpy(np.ascontiguousarray(a).reshape(-1).view(np.uint8).copy()).cuda()
        self.keep.append(t)
        return t.data_ptr()

    def out(self, nbytes):
        t = self.torch.zeros(max(nbytes, 16), dtype=self.torch.uint8, device="cuda")
        self.keep.append(t)
        return t

    def get(self, t, shape):
        self.torch.cuda.synchronize()
        return t.cpu().numpy()[: int(np.prod(shape))].reshape(shape)


def _call(L, name, *args):
    rc = getattr(L, name)(*args)
    assert rc == 0, f"{name} returned {rc}"


@pytest.mark.parametrize("prec", PRECS)
def test_user_axpy_real_and_complex(orc, uk, prec):
    d = _Dev()
    n = 4000 if prec <= 1056 else 1500
    X, Y = orc.gen_pairs(prec, n, 0xA1 + prec)
    a = orc.gen_pairs(prec, 1, 0xA2 + prec)[0]
    es = orc.elem_bytes(prec)
    z = d.out(n * es)
    _call(uk, "uk_axpy_r", prec, n, d.put(a), d.put(X), d.put(Y), z.data_ptr(), 0, 128, None)
    bad, first = orc.mismatches(prec, d.get(z, (n, es)), orc.axpy(prec, a, X, Y, impl="mp"))
    assert bad == 0, f"real AXPY PB={prec}: {bad} differ from MPFR (first {first})"
    nc = n // 2
    Xc, Yc = orc.gen_pairs(prec, nc, 0xA3 + prec, cplx=True)
    ac = orc.gen_pairs(prec, 1, 0xA4 + prec, cplx=True)[0]
    zc = d.out(nc * 2 * es)
    _call(uk, "uk_axpy_c", prec, nc, d.put(ac), d.put(Xc), d.put(Yc), zc.data_ptr(), 0, 128, None)
    bad, first = orc.mismatches(prec, d.get(zc, (nc, 2 * es)), orc.axpy(prec, ac, Xc, Yc, True, impl="mp"), True)
    assert bad == 0, f"complex AXPY PB={prec}: {bad} differ from MPC (first {first})"


@pytest.mark.parametrize("prec", PRECS)
def test_user_matmul_sequential_k(orc, uk, prec):
    """C = A B with acc = cu_fadd(acc, cu_fmul(a, b)) in k order (real) and
    acc = acc + a * b (complex), against MPFR / MPC in the same order."""
    d = _Dev()
    m, n, k = (12, 20, 33) if prec <= 1056 else (6, 10, 17)
    es = orc.elem_bytes(prec)
    A, _ = orc.gen_pairs(prec, m * k, 0xB1 + prec)
    B, _ = orc.gen_pairs(prec, k * n, 0xB2 + prec)
    c = d.out(m * n * es)
    _call(uk, "uk_matmul_r", prec, m, n, k, d.put(A), k, d.put(B), n, c.data_ptr(), n, 0, 64, None)
    bad, first = orc.mismatches(prec, d.get(c, (m * n, es)), orc.gemm(prec, m, n, k, A, k, B, n, impl="mp"))
    assert bad == 0, f"real matmul PB={prec}: {bad} differ (first {first})"
    Ac, _ = orc.gen_pairs(prec, m * k, 0xB3 + prec, cplx=True)
    Bc, _ = orc.gen_pairs(prec, k * n, 0xB4 + prec, cplx=True)
    cc = d.out(m * n * 2 * es)
    _call(uk, "uk_matmul_c", prec, m, n, k, d.put(Ac), k, d.put(Bc), n, cc.data_ptr(), n, 0, 64, None)
    bad, first = orc.mismatches(prec, d.get(cc, (m * n, 2 * es)),
                                orc.gemm(prec, m, n, k, Ac, k, Bc, n, cplx=True, impl="mp"), True)
    assert bad == 0, f"complex matmul PB={prec}: {bad} differ (first {first})"


def test_user_real_kernels_at_4096_bits(orc, uk, refuk):
    """Above 2048 bits (the reference benchmarks 4096 bits and up,
    demos/bench_3way.cu:167-169): the real AXPY and the sequential-k real
    matmul through the drop-in header at 4096 bits, bit for bit against MPFR,
    and the same source built against the reference's header agreeing."""
    prec = 4096
    d = _Dev()
    es = orc.elem_bytes(prec)
    n = 600
    X, Y = orc.gen_pairs(prec, n, 0xA1 + prec)
    a = orc.gen_pairs(prec, 1, 0xA2 + prec)[0]
    want = orc.axpy(prec, a, X, Y, impl="mp")
    for L, pre in ((uk, "uk_"), (refuk, "refuk_")):
        z = d.out(n * es)
        _call(L, pre + "axpy_r", prec, n, d.put(a), d.put(X), d.put(Y), z.data_ptr(), 0, 128, None)
        bad, first = orc.mismatches(prec, d.get(z, (n, es)), want)
        assert bad == 0, f"{pre}axpy_r PB={prec}: {bad} differ from MPFR (first {first})"
    m, nn, k = 4, 8, 9
    A, _ = orc.gen_pairs(prec, m * k, 0xB1 + prec)
    B, _ = orc.gen_pairs(prec, k * nn, 0xB2 + prec)
    c = d.out(m * nn * es)
    _call(uk, "uk_matmul_r", prec, m, nn, k, d.put(A), k, d.put(B), nn, c.data_ptr(), nn, 0, 64, None)
    bad, first = orc.mismatches(prec, d.get(c, (m * nn, es)), orc.gemm(prec, m, nn, k, A, k, B, nn, impl="mp"))
    assert bad == 0, f"real matmul PB={prec}: {bad} differ (first {first})"


@pytest.mark.parametrize("prec", FN_PRECS)
def test_user_exp_and_div(orc, mpb, uk, prec):
    d = _Dev()
    es = orc.elem_bytes(prec)
    n = 600 if prec <= 512 else 200
    X = orc.rand_elems(prec, n, 0xC1 + prec, -6, 6)
    Y = orc.rand_elems(prec, n, 0xC2 + prec, -40, 40)
    q = d.out(n * es)
    _call(uk, "uk_div", prec, n, d.put(X), d.put(Y), q.data_ptr(), 0, 128, None)
    bad, first = orc.mismatches(prec, d.get(q, (n, es)), orc.div(prec, X, Y, impl="mp"))
    assert bad == 0, f"cu_fdiv PB={prec}: {bad} differ from mpfr_div (first {first})"
    r = d.out(n * es)
    _call(uk, "uk_exp", prec, n, d.put(X), r.data_ptr(), 0, 128, None)
    got = d.get(r, (n, es))
    host = orc.empty(prec, n)
    mpb.host_lib().mpbh_exp(prec, n, X.ctypes.data_as(_V), host.ctypes.data_as(_V))
    assert orc.mismatches(prec, got, host)[0] == 0, f"cu_exp PB={prec}: device differs from the host build"
    pref = min(4 * prec, orc.lib().orc_max_prec())
    ulp = orc.ulp_errors(prec, got, pref, orc.exp(prec, X, pref))
    assert ulp.max() <= 1.0, f"cu_exp PB={prec}: {ulp.max():.3g} ULP"


@pytest.mark.parametrize("prec", PRECS)
def test_bench3way_axpy_fp64_io(orc, mpb, uk, prec):
    """The benchmark kernels of demos/bench_3way.cu:44-59 (FP64 operands in,
    the PB-bit result rounded to FP64 out) against MPFR / MPC, whose results
    are rounded to FP64 by the host build of to_double (held to the
    reference's to_double by tests/test_dropin_util.py)."""
    import torch

    to_d = mpb.host_lib().mpbh_to_double

    rng = np.random.default_rng(prec)
    n = 4096
    x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    a = 1.5
    X, Y, O = (torch.from_numpy(v).cuda() for v in (x, y, np.zeros(n)))
    _call(uk, "uk_axpy_d", prec, n, a, X.data_ptr(), Y.data_ptr(), O.data_ptr(), 128, 32, None)
    torch.cuda.synchronize()
    want = orc.axpy(prec, orc.from_double(prec, [a]), orc.from_double(prec, x), orc.from_double(prec, y),
                    impl="mp")
    wd = np.zeros(n)
    to_d(prec, n, want.ctypes.data_as(_V), wd.ctypes.data_as(_V))
    assert np.array_equal(O.cpu().numpy(), wd)
    xr, xi, yr, yi = (rng.uniform(-1, 1, n) for _ in range(4))
    T = [torch.from_numpy(v).cuda() for v in (xr, xi, yr, yi, np.zeros(n), np.zeros(n))]
    _call(uk, "uk_caxpy_d", prec, n, 1.5, -0.25, *[t.data_ptr() for t in T], 128, 32, None)
    torch.cuda.synchronize()

    def cvec(re, im):
        R, I = orc.from_double(prec, re), orc.from_double(prec, im)
        return np.concatenate([R, I], axis=1)

    wc = orc.axpy(prec, cvec([1.5], [-0.25]), cvec(xr, xi), cvec(yr, yi), True, impl="mp")
    es = orc.elem_bytes(prec)
    for comp, t in ((0, T[4]), (1, T[5])):
        part = np.ascontiguousarray(wc[:, comp * es:(comp + 1) * es])
        dd = np.zeros(n)
        to_d(prec, n, part.ctypes.data_as(_V), dd.ctypes.data_as(_V))
        assert np.array_equal(t.cpu().numpy(), dd), f"complex component {comp}"


@pytest.mark.parametrize("prec", PRECS)
def test_reference_headers_on_the_gpu_agree(orc, uk, refuk, prec):
    """The same user kernels built against the reference's own headers give the
    same AXPY and matmul results on the B200 (both are bit-exact with MPFR /
    MPC for + - *)."""
    d = _Dev()
    es = orc.elem_bytes(prec)
    n = 2000 if prec <= 1056 else 600
    X, Y = orc.gen_pairs(prec, n, 0xD1 + prec)
    a = orc.gen_pairs(prec, 1, 0xD2 + prec)[0]
    outs = []
    for L, pre in ((uk, "uk_"), (refuk, "refuk_")):
        z = d.out(n * es)
        _call(L, pre + "axpy_r", prec, n, d.put(a), d.put(X), d.put(Y), z.data_ptr(), 0, 128, None)
        outs.append(d.get(z, (n, es)))
    assert orc.mismatches(prec, outs[0], outs[1])[0] == 0
    m, nn, k = 6, 9, 14
    A, _ = orc.gen_pairs(prec, m * k, 0xD3 + prec, cplx=True)
    B, _ = orc.gen_pairs(prec, k * nn, 0xD4 + prec, cplx=True)
    outs = []
    for L, pre in ((uk, "uk_"), (refuk, "refuk_")):
        c = d.out(m * nn * 2 * es)
        _call(L, pre + "matmul_c", prec, m, nn, k, d.put(A), k, d.put(B), nn, c.data_ptr(), nn, 0, 64, None)
        outs.append(d.get(c, (m * nn, 2 * es)))
    assert orc.mismatches(prec, outs[0], outs[1], True)[0] == 0
