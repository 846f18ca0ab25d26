"""Golden vectors produced by the reference's own cu_freal/cu_fcomplex headers
(tests/golden/make_golden.py): the oracle's restatement, the host build of
the drop-in surface and (on a GPU) the engine must reproduce them bit for bit."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import to_dev, to_host
from mpc_cuda_b200 import layout

GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_vectors.npz"))
PRECS = (64, 96, 128, 256, 512, 1024, 2048)
GM, GN, GK = 3, 4, 5


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.mark.parametrize("prec", PRECS)
def test_oracle_restatement_matches_reference_vectors(orc, prec):
    g = lambda k: np.ascontiguousarray(GOLD[f"{k}"])  # noqa: E731
    A, B = g(f"r{prec}_a"), g(f"r{prec}_b")
    for kind in ("mul", "add", "sub"):
        assert orc.mismatches(prec, orc.binop(kind, prec, A, B), g(f"r{prec}_{kind}"))[0] == 0, kind
    Ac, Bc = g(f"c{prec}_a"), g(f"c{prec}_b")
    for kind in ("cmul", "cadd", "csub"):
        assert orc.mismatches(prec, orc.binop(kind, prec, Ac, Bc), g(f"c{prec}_{kind}"), True)[0] == 0, kind
    assert orc.mismatches(prec, orc.axpy(prec, A[:1].copy(), A, B), g(f"r{prec}_axpy"))[0] == 0
    assert orc.mismatches(prec, orc.axpy(prec, Ac[:1].copy(), Ac, Bc, True), g(f"c{prec}_axpy"), True)[0] == 0
    got = orc.gemm(prec, GM, GN, GK, g(f"r{prec}_ga"), GK, g(f"r{prec}_gb"), GN)
    assert orc.mismatches(prec, got, g(f"r{prec}_gemm"))[0] == 0
    got = orc.gemm(prec, GM, GN, GK, g(f"c{prec}_ga"), GK, g(f"c{prec}_gb"), GN, True)
    assert orc.mismatches(prec, got, g(f"c{prec}_gemm"), True)[0] == 0


@pytest.mark.parametrize("prec", PRECS)
def test_host_dropin_matches_reference_vectors(orc, mpb, prec):
    H = mpb.host_lib()
    g = lambda k: np.ascontiguousarray(GOLD[f"{k}"])  # noqa: E731
    A, B = g(f"r{prec}_a"), g(f"r{prec}_b")
    for op, kind in enumerate(("mul", "add", "sub")):
        R = np.zeros_like(A)
        H.mpbh_binop(prec, op, A.shape[0], _p(A), _p(B), _p(R))
        assert orc.mismatches(prec, R, g(f"r{prec}_{kind}"))[0] == 0, kind
    Ac, Bc = g(f"c{prec}_a"), g(f"c{prec}_b")
    for op, kind in enumerate(("cmul", "cadd", "csub")):
        R = np.zeros_like(Ac)
        H.mpbh_cbinop(prec, op, Ac.shape[0], _p(Ac), _p(Bc), _p(R))
        assert orc.mismatches(prec, R, g(f"c{prec}_{kind}"), True)[0] == 0, kind


@pytest.mark.gpu
@pytest.mark.parametrize("prec", tuple(p for p in PRECS if p in layout.SUPPORTED))
def test_engine_matches_reference_vectors(orc, mpb, prec):
    g = lambda k: np.ascontiguousarray(GOLD[f"{k}"])  # noqa: E731
    A, B = g(f"r{prec}_a"), g(f"r{prec}_b")
    n = A.shape[0]
    dA, dB = to_dev(layout.aos_to_vec(prec, A)), to_dev(layout.aos_to_vec(prec, B))
    r = mpb.empty(prec, n)
    for op, kind in enumerate(("mul", "add", "sub")):
        mpb.binop(prec, op, n, dA, dB, r)
        assert orc.mismatches(prec, layout.vec_to_aos(prec, to_host(r), n), g(f"r{prec}_{kind}"))[0] == 0, kind
    mpb.axpy(prec, n, dA, dA, dB, r)
    assert orc.mismatches(prec, layout.vec_to_aos(prec, to_host(r), n), g(f"r{prec}_axpy"))[0] == 0
    Ac, Bc = g(f"c{prec}_a"), g(f"c{prec}_b")
    nc = Ac.shape[0]
    dA, dB = to_dev(layout.aos_to_vec(prec, Ac, True)), to_dev(layout.aos_to_vec(prec, Bc, True))
    rc = mpb.empty(prec, nc, True)
    for op, kind in enumerate(("cmul", "cadd", "csub")):
        mpb.binop(prec, op, nc, dA, dB, rc, cplx=True)
        got = layout.vec_to_aos(prec, to_host(rc), nc, True)
        assert orc.mismatches(prec, got, g(f"c{prec}_{kind}"), True)[0] == 0, kind
    mpb.axpy(prec, nc, dA, dA, dB, rc, cplx=True)
    got = layout.vec_to_aos(prec, to_host(rc), nc, True)
    assert orc.mismatches(prec, got, g(f"c{prec}_axpy"), True)[0] == 0
