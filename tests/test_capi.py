"""The C ABI library: loads without a GPU, exports every symbol mpb.h declares,
and rejects bad arguments on the host with the documented status codes
(no kernel is launched by any call here)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"\b(mpb_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_exports_every_declared_symbol(mpb):
    lib = C.CDLL(mpb.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"declared but not exported: {missing}"
    assert set(declared_symbols()) <= set(mpb.exported_symbols())


def test_info_calls(mpb):
    L = mpb.lib()
    assert L.mpb_version() >= 100
    for p in (64, 128, 256, 512, 1024, 2048):
        assert L.mpb_prec_supported(p) == 1
        assert L.mpb_vec_bytes(p, 33) == mpb.vec_bytes(p, 33)
        assert L.mpb_cvec_bytes(p, 33) == mpb.vec_bytes(p, 33, True)
        assert L.mpb_aos_bytes(p) == 16 + p // 8
    for p in (0, 32, 96, 100, 4096, -64):
        assert L.mpb_prec_supported(p) == 0
        assert L.mpb_vec_bytes(p, 10) == 0
    assert b"precision" in L.mpb_status_string(-1)


def test_bad_arguments_rejected_on_host(mpb):
    L = mpb.lib()
    good = 4096  # a fake, 16-byte aligned "device" address: never dereferenced here
    # unsupported precision
    assert L.mpb_axpy_r(96, 10, good, good, good, good, None) == -1
    assert L.mpb_gemm_r(100, 4, 4, 4, good, 32, good, 32, good, 32, None) == -1
    # null and misaligned buffers
    assert L.mpb_axpy_r(256, 10, None, good, good, good, None) == -3
    assert L.mpb_axpy_c(256, 10, good, good, good + 8, good, None) == -4
    assert L.mpb_binop_r(256, 0, 10, good, None, good, None) == -3
    # bad op code
    assert L.mpb_binop_r(256, 7, 10, good, good, good, None) == -7
    # leading dimensions: not a multiple of 32, or shorter than a row
    assert L.mpb_gemm_r(256, 4, 4, 4, good, 33, good, 32, good, 32, None) == -5
    assert L.mpb_gemm_r(256, 4, 40, 4, good, 32, good, 32, good, 32, None) == -5
    assert L.mpb_gemv_r(256, 4, 50, good, 32, good, good, good, None) == -5
    # size overflow
    assert L.mpb_axpy_r(256, 1 << 62, good, good, good, good, None) == -2
    # elementary functions: unknown function, missing second operand
    assert L.mpb_fmath_r(16, 256, 10, good, None, good, None) == -7
    assert L.mpb_fmath_r(14, 256, 10, good, None, good, None) == -3  # pow needs b
    assert L.mpb_fmath_c(9, 256, 10, good, good, good, None) == -7
    assert L.mpb_fmath_c(8, 256, 10, good, None, good, None) == -3  # division needs b
    assert L.mpb_const_r(2, 256, 10, good, None) == -7
    assert L.mpb_div_ui_r(100, 10, good, 3, good, None) == -1
    # runtime precision: storage formats and bad arguments
    assert [L.mpb_storage_prec(p) for p in (1, 62, 63, 126, 127, 2046, 2047, 0)] == [64, 64, 128, 128, 256, 2048, -1, -1]
    assert L.mpb_op_rp(6, 100, 10, good, good, good, good, None) == -7
    assert L.mpb_op_rp(0, 2047, 10, good, good, good, good, None) == -1
    assert L.mpb_op_rp(3, 100, 10, good, good, None, good, None) == -3  # fma needs c


def test_empty_inputs_are_noops(mpb):
    L = mpb.lib()
    assert L.mpb_axpy_r(256, 0, None, None, None, None, None) == 0
    assert L.mpb_axpy_c(1024, 0, None, None, None, None, None) == 0
    assert L.mpb_gemm_r(512, 0, 8, 8, None, 32, None, 32, None, 32, None) == 0
    assert L.mpb_gemv_c(256, 0, 5, None, 32, None, None, None, None) == 0
    assert L.mpb_pack_aos(256, 0, None, None, None) == 0
    assert L.mpb_fmath_r(0, 256, 0, None, None, None, None) == 0
    assert L.mpb_op_rp(0, 100, 0, None, None, None, None, None) == 0


def test_exact_gemm_workspace_and_checks(mpb):
    L = mpb.lib()
    # PB=512, 1024^3, 32-bit spread: S = 69 digit planes, 137 diagonals (each
    # padded by 1056 entries), plus one certification flag byte per entry
    S, m = 69, 1024
    need = L.mpb_gemm_exact_workspace(512, m, m, m, 32)
    planes = S * 2 * m * m + 137 * (m * m + 1056) * 4 + m * m
    assert planes <= need <= planes + 64 * 1024
    # the tensor cores skip the low diagonals 0..64: 2616 of the 69^2 slice pairs
    assert mpb.gemm_exact_info(512, m, m, m, 32) == (69, 65, 2616)
    assert mpb.gemm_exact_info(256, 512, 512, 512, 16, cplx=True) == (35, 29, 790)
    assert L.mpb_gemm_exact_workspace(96, 8, 8, 8, 32) == 0
    good = 4096
    # missing workspace, misaligned workspace, bad leading dimension
    assert L.mpb_gemm_exact_r(512, 8, 8, 8, good, 32, good, 32, good, 32, 32, None, 0, None, None) == -8
    assert L.mpb_gemm_exact_r(512, 8, 8, 8, good, 32, good, 32, good, 32, 32, good + 16, 1 << 30, None, None) == -4
    assert L.mpb_gemm_exact_r(512, 8, 8, 8, good, 40, good, 32, good, 32, 32, good, 1 << 30, None, None) == -5
    assert L.mpb_gemm_exact_r(512, 0, 8, 8, None, 32, None, 32, None, 32, 32, None, 0, None, None) == 0


def test_exact_gemm_complex_workspace(mpb):
    L = mpb.lib()
    # PB=256, 512^3 complex, 16-bit spread: S = ceil((256+16+3)/8) = 35, 3 products
    S, m = 35, 512
    need = L.mpb_gemm_exact_c_workspace(256, m, m, m, 16)
    planes = 3 * S * 2 * m * m + 3 * (2 * S - 1) * (m * m + 1056) * 4 + m * m
    assert planes <= need <= planes + 64 * 1024
    assert L.mpb_gemm_exact_c(256, 8, 8, 8, 4096, 32, 4096, 32, 4096, 32, 16, None, 0, None, None) == -8


def test_batch_gemv_plan_validation(mpb):
    import ctypes as C

    L = mpb.lib()
    assert L.mpb_batch_gemv_workspace(4096) >= 4096 * 48
    assert L.mpb_batch_gemv_workspace(0) == 0
    good = 4096
    ws = 1 << 20  # fake, 256-aligned; validation fails before it is used

    def one(**kw):
        d = dict(prec=256, m=4, n=5, lda=32, A=good, x=good, y=good, y_out=good)
        d.update(kw)
        arr = (mpb.GemvProblem * 1)(mpb.GemvProblem(**d))
        h = C.c_void_p()
        return L.mpb_batch_gemv_plan(1, C.cast(arr, C.c_void_p), ws, 1 << 20, C.byref(h))

    assert one(prec=96) == -1
    assert one(lda=40) == -5
    assert one(lda=0) == -5
    assert one(x=None) == -3
    assert one(y_out=good + 8) == -4
    assert one(m=-1) == -2
    h = C.c_void_p()
    assert L.mpb_batch_gemv_plan(1, None, ws, 1 << 20, C.byref(h)) == -3
