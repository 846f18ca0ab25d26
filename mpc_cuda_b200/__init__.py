"""mpc_cuda_b200 -- Python host side of the mpb B200 fixed-precision engine.

The engine is ``libmpb.so`` (CUDA, sm_100a) behind the C ABI of
``include/mpb.h``.  This module binds that ABI with ctypes and accepts torch
CUDA tensors (any dtype; the bytes are used) as device buffers; torch supplies
device memory and streams only.  There is no CPU implementation: if the
library is missing or no GPU is present every compute call raises.

Buffers hold the tiled layout (``mpc_cuda_b200.layout``):
``vec_bytes(prec, n)`` bytes for a real vector, ``cvec_bytes`` for complex,
row-major matrices with a leading dimension that is a multiple of 32.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from . import layout
from .layout import SUPPORTED, aos_bytes, tile_bytes

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmpb.so")
HOST_LIB_PATH = os.path.join(HERE, "libmpb_host.so")

MPB_OP_MUL, MPB_OP_ADD, MPB_OP_SUB = 0, 1, 2

_STATUS = {
    0: "MPB_OK", -1: "MPB_ERR_PREC", -2: "MPB_ERR_SIZE", -3: "MPB_ERR_NULL", -4: "MPB_ERR_ALIGN",
    -5: "MPB_ERR_LD", -6: "MPB_ERR_CUDA", -7: "MPB_ERR_ARG", -8: "MPB_ERR_WORKSPACE",
}


class MpbError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        super().__init__(f"{where}: {_STATUS.get(status, status)} ({status_string(status)})")


_lib = None
_host = None

# name -> argument types (after the leading int prec where present)
_V, _S, _I, _L = C.c_void_p, C.c_size_t, C.c_int, C.c_long
_SIGS = {
    "mpb_version": ([], C.c_int),
    "mpb_status_string": ([_I], C.c_char_p),
    "mpb_prec_supported": ([_I], C.c_int),
    "mpb_vec_bytes": ([_I, _S], C.c_size_t),
    "mpb_cvec_bytes": ([_I, _S], C.c_size_t),
    "mpb_aos_bytes": ([_I], C.c_size_t),
    "mpb_pack_aos": ([_I, _S, _V, _V, _V], C.c_int),
    "mpb_unpack_aos": ([_I, _S, _V, _V, _V], C.c_int),
    "mpb_cpack_aos": ([_I, _S, _V, _V, _V], C.c_int),
    "mpb_cunpack_aos": ([_I, _S, _V, _V, _V], C.c_int),
    "mpb_from_double": ([_I, _S, _V, _V, _V], C.c_int),
    "mpb_to_double": ([_I, _S, _V, _V, _V], C.c_int),
    "mpb_binop_r": ([_I, _I, _S, _V, _V, _V, _V], C.c_int),
    "mpb_fma_r": ([_I, _S, _V, _V, _V, _V, _V], C.c_int),
    "mpb_fma_c": ([_I, _S, _V, _V, _V, _V, _V], C.c_int),
    "mpb_div_r": ([_I, _S, _V, _V, _V, _V], C.c_int),
    "mpb_sqrt_r": ([_I, _S, _V, _V, _V], C.c_int),
    "mpb_exp_r": ([_I, _S, _V, _V, _V], C.c_int),
    "mpb_log_r": ([_I, _S, _V, _V, _V], C.c_int),
    "mpb_fmath_r": ([_I, _I, _S, _V, _V, _V, _V], C.c_int),
    "mpb_fmath_c": ([_I, _I, _S, _V, _V, _V, _V], C.c_int),
    "mpb_div_ui_r": ([_I, _S, _V, C.c_uint64, _V, _V], C.c_int),
    "mpb_const_r": ([_I, _I, _S, _V, _V], C.c_int),
    "mpb_storage_prec": ([_I], C.c_int),
    "mpb_op_rp": ([_I, _I, _S, _V, _V, _V, _V, _V], C.c_int),
    "mpb_aos_to_mpfr": ([_I, _S, _V, _V], C.c_int),
    "mpb_aos_from_mpfr": ([_I, _S, _V, _V], C.c_int),
    "mpb_caos_to_mpc": ([_I, _S, _V, _V], C.c_int),
    "mpb_caos_from_mpc": ([_I, _S, _V, _V], C.c_int),
    "mpb_binop_c": ([_I, _I, _S, _V, _V, _V, _V], C.c_int),
    "mpb_axpy_r": ([_I, _S, _V, _V, _V, _V, _V], C.c_int),
    "mpb_axpy_c": ([_I, _S, _V, _V, _V, _V, _V], C.c_int),
    "mpb_gemv_r": ([_I, _S, _S, _V, _S, _V, _V, _V, _V], C.c_int),
    "mpb_gemv_c": ([_I, _S, _S, _V, _S, _V, _V, _V, _V], C.c_int),
    "mpb_gemm_r": ([_I, _S, _S, _S, _V, _S, _V, _S, _V, _S, _V], C.c_int),
    "mpb_gemm_c": ([_I, _S, _S, _S, _V, _S, _V, _S, _V, _S, _V], C.c_int),
    "mpb_gemm_exact_plan_info": ([_I, _S, _S, _S, _I, _I, C.POINTER(_I), C.POINTER(_I), C.POINTER(C.c_longlong)],
                                 C.c_int),
    "mpb_batch_gemv_workspace": ([_I], C.c_size_t),
    "mpb_batch_gemv_plan": ([_I, _V, _V, _S, C.POINTER(_V)], C.c_int),
    "mpb_batch_gemv_run": ([_V, _V], C.c_int),
    "mpb_batch_gemv_autotune": ([_V, _V], C.c_int),
    "mpb_batch_gemv_get_tuning": ([_V, _I, C.POINTER(_I), C.POINTER(_I)], C.c_int),
    "mpb_batch_gemv_set_tuning": ([_V, _I, _I, _I], C.c_int),
    "mpb_batch_gemv_tuned_ms": ([_V, _I, C.POINTER(C.c_float)], C.c_int),
    "mpb_batch_gemv_get_split": ([_V, _I, C.POINTER(_I)], C.c_int),
    "mpb_batch_gemv_set_split": ([_V, _I, _I], C.c_int),
    "mpb_set_split": ([_I, _I, _I], C.c_int),
    "mpb_get_split": ([_I, _I, C.POINTER(_I)], C.c_int),
    "mpb_set_gemm_warps": ([_I, _I, _I], C.c_int),
    "mpb_get_gemm_warps": ([_I, _I, C.POINTER(_I)], C.c_int),
    "mpb_batch_gemv_destroy": ([_V], None),
    "mpb_gemm_exact_workspace": ([_I, _S, _S, _S, _I], C.c_size_t),
    "mpb_profile_enable": ([_I], None),
    "mpb_profile_phases": ([C.c_uint], None),
    "mpb_profile_phase_ms": ([_I], C.c_float),
    "mpb_profile_phase_count": ([_I], C.c_int),
    "mpb_gemm_exact_r": ([_I, _S, _S, _S, _V, _S, _V, _S, _V, _S, _I, _V, _S, _V, _V], C.c_int),
    "mpb_gemm_exact_c_workspace": ([_I, _S, _S, _S, _I], C.c_size_t),
    "mpb_gemm_exact_c": ([_I, _S, _S, _S, _V, _S, _V, _S, _V, _S, _I, _V, _S, _V, _V], C.c_int),
    "mpb_gemm_exact_r_static": ([_I, _S, _S, _S, _V, _S, _V, _S, _V, _S, _I, _V, _V], C.c_int),
    "mpb_gemm_exact_test_inject": ([_I, C.c_longlong], C.c_int),
    "mpb_axpy_r_rp": ([_I, _S, _V, _V, _V, _V, _V], C.c_int),
    "mpb_gemv_r_rp": ([_I, _S, _S, _V, _S, _V, _V, _V, _V], C.c_int),
    "mpb_gemm_r_rp": ([_I, _S, _S, _S, _V, _S, _V, _S, _V, _S, _V], C.c_int),
    "mpb_fmath_r_rp": ([_I, _I, _S, _V, _V, _V, _V], C.c_int),
}


def build(verbose: bool = False) -> None:
    """Compile libmpb.so / libmpb_host.so in-tree (nvcc, sm_100a)."""
    out = subprocess.run(["make", "-C", os.path.join(HERE, "csrc"), "-j8"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("mpb build failed:\n" + out.stdout[-4000:] + out.stderr[-4000:])
    if verbose:
        print(out.stdout)


def lib():
    """The loaded CUDA engine.  Raises if libmpb.so was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run mpc_cuda_b200.build() (nvcc, sm_100a)")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def host_lib():
    """The drop-in cu_fp surface built for the host CPU (AoS arrays)."""
    global _host
    if _host is None:
        if not os.path.exists(HOST_LIB_PATH):
            raise RuntimeError(f"{HOST_LIB_PATH} is missing: run mpc_cuda_b200.build()")
        H = C.CDLL(HOST_LIB_PATH)
        for name in ("mpbh_binop", "mpbh_cbinop"):
            getattr(H, name).argtypes = [_I, _I, _L, _V, _V, _V]
        H.mpbh_fma.argtypes = [_I, _L, _V, _V, _V, _V]
        H.mpbh_cfma.argtypes = [_I, _L, _V, _V, _V, _V]
        H.mpbh_div.argtypes = [_I, _L, _V, _V, _V]
        H.mpbh_sqrt.argtypes = [_I, _L, _V, _V]
        H.mpbh_exp.argtypes = [_I, _L, _V, _V]
        H.mpbh_log.argtypes = [_I, _L, _V, _V]
        for name in ("mpbh_fmath_r", "mpbh_fmath_c"):
            getattr(H, name).argtypes = [_I, _I, _L, _V, _V, _V]
        H.mpbh_div_ui.argtypes = [_I, _L, _V, C.c_ulonglong, _V]
        H.mpbh_const.argtypes = [_I, _I, _V]
        H.mpbh_op_rp.argtypes = [_I, _I, _L, _V, _V, _V, _V]
        for name in ("mpbh_axpy_r", "mpbh_axpy_c"):
            getattr(H, name).argtypes = [_I, _L, _V, _V, _V, _V]
        H.mpbh_from_double.argtypes = [_I, _L, _V, _V]
        H.mpbh_to_double.argtypes = [_I, _L, _V, _V]
        _host = H
    return _host


def exported_symbols():
    return list(_SIGS)


def status_string(status: int) -> str:
    try:
        return lib().mpb_status_string(status).decode()
    except Exception:  # library missing: still describe the code
        return _STATUS.get(status, "unknown")


def vec_bytes(prec: int, n: int, cplx: bool = False) -> int:
    return layout.vec_bytes(prec, n, cplx)


# ---------------------------------------------------------------- buffers
def _ptr(t):
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


def _stream(stream):
    if stream is None:
        import torch

        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def empty(prec: int, n: int, cplx: bool = False, device="cuda"):
    """Uninitialised device vector of n elements (torch uint8 tensor)."""
    import torch

    return torch.empty(max(vec_bytes(prec, n, cplx), 16), dtype=torch.uint8, device=device)


def empty_matrix(prec: int, rows: int, ld: int, cplx: bool = False, device="cuda"):
    return empty(prec, rows * ld, cplx, device)


def _call(name, *args):
    rc = getattr(lib(), name)(*args)
    if rc != 0:
        raise MpbError(rc, name)


# ---------------------------------------------------------------- operations
def pack_aos(prec, n, aos, vec, cplx=False, stream=None):
    _call("mpb_cpack_aos" if cplx else "mpb_pack_aos", prec, n, _ptr(aos), _ptr(vec), _stream(stream))


def unpack_aos(prec, n, vec, aos, cplx=False, stream=None):
    _call("mpb_cunpack_aos" if cplx else "mpb_unpack_aos", prec, n, _ptr(vec), _ptr(aos), _stream(stream))


def from_double(prec, n, d, vec, stream=None):
    _call("mpb_from_double", prec, n, _ptr(d), _ptr(vec), _stream(stream))


def to_double(prec, n, vec, d, stream=None):
    _call("mpb_to_double", prec, n, _ptr(vec), _ptr(d), _stream(stream))


def binop(prec, op, n, a, b, r, cplx=False, stream=None):
    _call("mpb_binop_c" if cplx else "mpb_binop_r", prec, op, n, _ptr(a), _ptr(b), _ptr(r), _stream(stream))


def div(prec, n, a, b, r, stream=None):
    """r = round(a / b), one rounding (0 where b is 0)."""
    _call("mpb_div_r", prec, n, _ptr(a), _ptr(b), _ptr(r), _stream(stream))


def sqrt(prec, n, a, r, stream=None):
    """r = round(sqrt(a)), one rounding (0 where a < 0)."""
    _call("mpb_sqrt_r", prec, n, _ptr(a), _ptr(r), _stream(stream))


def exp(prec, n, a, r, stream=None):
    """r = exp(a), faithful (0 where |a| >= 2^29)."""
    _call("mpb_exp_r", prec, n, _ptr(a), _ptr(r), _stream(stream))


def log(prec, n, a, r, stream=None):
    """r = log(a), faithful (0 where a <= 0)."""
    _call("mpb_log_r", prec, n, _ptr(a), _ptr(r), _stream(stream))


# elementary functions, in the order of mpb.h's MPB_FN_* / MPB_CFN_*
FN = ("exp", "log", "expm1", "log1p", "sin", "cos", "tan", "atan", "sinh", "cosh",
      "atanh", "asin", "acos", "cbrt", "pow", "atan2")
CFN = ("exp", "log", "sqrt", "sin", "cos", "tan", "sinh", "cosh", "div")


def fmath(name, prec, n, a, r, b=None, stream=None):
    """r = name(a) (pow / atan2: name(a, b)), faithful; the drop-in cu_<name>."""
    _call("mpb_fmath_r", FN.index(name), prec, n, _ptr(a), _ptr(b) if b is not None else None, _ptr(r),
          _stream(stream))


def cfmath(name, prec, n, a, r, b=None, stream=None):
    """complex r = name(a) (div: a / b), each component faithful; cu_c<name>."""
    _call("mpb_fmath_c", CFN.index(name), prec, n, _ptr(a), _ptr(b) if b is not None else None, _ptr(r),
          _stream(stream))


def div_ui(prec, n, a, u, r, stream=None):
    """r = round(a / u) for an unsigned 64-bit integer u (cu_div_ui)."""
    _call("mpb_div_ui_r", prec, n, _ptr(a), u, _ptr(r), _stream(stream))


def const(which, prec, n, r, stream=None):
    """r[0 .. n) = pi ('pi') or ln 2 ('ln2'), correctly rounded (cu_pi / cu_ln2)."""
    _call("mpb_const_r", 0 if which == "pi" else 1, prec, n, _ptr(r), _stream(stream))


RP_OPS = ("mul", "add", "sub", "fma", "div", "sqrt")


def storage_prec(prec):
    """the supported PB whose vectors hold precision prec (PB >= prec + 2)"""
    pb = lib().mpb_storage_prec(prec)
    if pb < 0:
        raise MpbError(pb, "mpb_storage_prec")
    return pb


def op_rp(op, prec, n, a, r, b=None, c=None, stream=None):
    """r = op(a, b, c) correctly rounded at a runtime precision prec (vectors in
    the storage_prec(prec) format); op in RP_OPS."""
    _call("mpb_op_rp", RP_OPS.index(op), prec, n, _ptr(a), _ptr(b), _ptr(c), _ptr(r), _stream(stream))


def axpy_rp(prec, n, a, x, y, z, stream=None):
    """z = round(round(a*x) + y) at a runtime precision prec (storage_prec layout)."""
    _call("mpb_axpy_r_rp", prec, n, _ptr(a), _ptr(x), _ptr(y), _ptr(z), _stream(stream))


def gemv_rp(prec, m, n, A, lda, x, y, y_out, stream=None):
    _call("mpb_gemv_r_rp", prec, m, n, _ptr(A), lda, _ptr(x), _ptr(y), _ptr(y_out), _stream(stream))


def gemm_rp(prec, m, n, k, A, lda, B, ldb, C, ldc, stream=None):
    _call("mpb_gemm_r_rp", prec, m, n, k, _ptr(A), lda, _ptr(B), ldb, _ptr(C), ldc, _stream(stream))


def fmath_rp(name, prec, n, a, r, b=None, stream=None):
    """elementary function `name` (FN) at a runtime precision prec, within 1 ULP of prec bits."""
    _call("mpb_fmath_r_rp", FN.index(name), prec, n, _ptr(a), _ptr(b), _ptr(r), _stream(stream))


def fma(prec, n, a, b, c, r, cplx=False, stream=None):
    """r = a*b + c with one rounding (per component when complex)."""
    _call("mpb_fma_c" if cplx else "mpb_fma_r", prec, n, _ptr(a), _ptr(b), _ptr(c), _ptr(r), _stream(stream))


def axpy(prec, n, a, x, y, z, cplx=False, stream=None):
    """z = a*x + y (a: element 0 of a vector), one rounding per operation."""
    _call("mpb_axpy_c" if cplx else "mpb_axpy_r", prec, n, _ptr(a), _ptr(x), _ptr(y), _ptr(z), _stream(stream))


def gemv(prec, m, n, A, lda, x, y, y_out, cplx=False, stream=None):
    """y_out = A.x + y, sequential-k per-operation rounding, then + y."""
    _call("mpb_gemv_c" if cplx else "mpb_gemv_r", prec, m, n, _ptr(A), lda, _ptr(x), _ptr(y), _ptr(y_out),
          _stream(stream))


def gemm(prec, m, n, k, A, lda, B, ldb, Cm, ldc, cplx=False, stream=None):
    """C = A.B, sequential-k per-operation rounding (plain kernel)."""
    _call("mpb_gemm_c" if cplx else "mpb_gemm_r", prec, m, n, k, _ptr(A), lda, _ptr(B), ldb, _ptr(Cm), ldc,
          _stream(stream))


def gemm_exact_workspace(prec, m, n, k, sp_bits=32, cplx=False):
    f = lib().mpb_gemm_exact_c_workspace if cplx else lib().mpb_gemm_exact_workspace
    return int(f(prec, m, n, k, sp_bits))


def gemm_exact_info(prec, m, n, k, sp_bits=32, cplx=False):
    """(slices S, lowest tensor-core diagonal d0, slice pairs per real product)."""
    S, d0, pairs = C.c_int(), C.c_int(), C.c_longlong()
    _call("mpb_gemm_exact_plan_info", prec, m, n, k, sp_bits, 1 if cplx else 0, C.byref(S), C.byref(d0),
          C.byref(pairs))
    return S.value, d0.value, pairs.value


def gemm_exact(prec, m, n, k, A, lda, B, ldb, Cm, ldc, sp_bits=32, workspace=None, status=None,
               cplx=False, stream=None):
    """C = A.B with one rounding per entry (exact accumulation on the INT8
    tensor cores).  ``workspace``: device buffer of gemm_exact_workspace(...)
    bytes (allocated here when None); ``status``: optional device int32[2]
    receiving [fallback rows+cols, kernel error code]."""
    if workspace is None:
        import torch

        nbytes = gemm_exact_workspace(prec, m, n, k, sp_bits, cplx)
        workspace = torch.empty(max(nbytes, 256), dtype=torch.uint8, device="cuda")
    nbytes = workspace.numel() * workspace.element_size() if not isinstance(workspace, int) else (1 << 62)
    _call("mpb_gemm_exact_c" if cplx else "mpb_gemm_exact_r", prec, m, n, k, _ptr(A), lda, _ptr(B), ldb, _ptr(Cm),
          ldc, sp_bits, _ptr(workspace), nbytes, _ptr(status), _stream(stream))
    return workspace


# thread-vs-warp split of the kernels with a warp-cooperative form (mpb.h)
SPLIT_AXPY_C, SPLIT_GEMV_R = 0, 1


def set_split(kind, prec, lanes):
    """Lanes per element for `kind` at `prec` (1 = one thread per element)."""
    _call("mpb_set_split", int(kind), int(prec), int(lanes))


def get_split(kind, prec):
    v = C.c_int()
    _call("mpb_get_split", int(kind), int(prec), C.byref(v))
    return v.value


def set_gemm_warps(prec, warps, cplx=False):
    """Warps (rows of C) per block of the plain GEMM at `prec`: 4, 8 or 16."""
    _call("mpb_set_gemm_warps", 1 if cplx else 0, int(prec), int(warps))


def get_gemm_warps(prec, cplx=False):
    v = C.c_int()
    _call("mpb_get_gemm_warps", 1 if cplx else 0, int(prec), C.byref(v))
    return v.value


class GemvProblem(C.Structure):
    """mpb_gemv_problem: y_out = A.x + y at precision prec (device pointers)."""
    _fields_ = [("prec", C.c_int), ("m", C.c_int), ("n", C.c_int), ("lda", C.c_size_t), ("A", C.c_void_p),
                ("x", C.c_void_p), ("y", C.c_void_p), ("y_out", C.c_void_p)]


class BatchGemv:
    """A planned batch of independent GEMV problems (mixed sizes and precisions).

    ``problems``: iterable of (prec, m, n, lda, A, x, y, y_out) with torch CUDA
    tensors (or raw device addresses).  ``run()`` launches every problem (no
    host synchronisation, capturable in a CUDA graph); ``autotune()`` picks the
    launch shape per precision on this batch; ``tuning``/``set_tuning`` read
    and install cached choices."""

    def __init__(self, problems, device="cuda"):
        import torch

        probs = [GemvProblem(p, m, n, lda, _ptr(A), _ptr(x), _ptr(y), _ptr(yo))
                 for (p, m, n, lda, A, x, y, yo) in problems]
        self.count = len(probs)
        arr = (GemvProblem * self.count)(*probs)
        nbytes = int(lib().mpb_batch_gemv_workspace(self.count))
        self.workspace = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=device)
        h = C.c_void_p()
        _call("mpb_batch_gemv_plan", self.count, C.cast(arr, C.c_void_p), _ptr(self.workspace), nbytes, C.byref(h))
        self._plan = h

    def run(self, stream=None):
        _call("mpb_batch_gemv_run", self._plan, _stream(stream))

    def autotune(self, stream=None):
        _call("mpb_batch_gemv_autotune", self._plan, _stream(stream))

    def tuning(self):
        out = {}
        for p in SUPPORTED:
            b, s = C.c_int(), C.c_int()
            _call("mpb_batch_gemv_get_tuning", self._plan, p, C.byref(b), C.byref(s))
            out[p] = (b.value, s.value)
        return out

    def tuned_ms(self):
        """{prec: ms of one solo run of that precision's problems} from the last autotune."""
        out = {}
        for p in SUPPORTED:
            v = C.c_float()
            _call("mpb_batch_gemv_tuned_ms", self._plan, p, C.byref(v))
            out[p] = v.value
        return out

    def set_tuning(self, table):
        for p, (b, s) in table.items():
            _call("mpb_batch_gemv_set_tuning", self._plan, int(p), int(b), int(s))

    def splits(self):
        """{prec: lanes per row} (1 = one thread per row, else a warp-cooperative group)."""
        out = {}
        for p in SUPPORTED:
            v = C.c_int()
            _call("mpb_batch_gemv_get_split", self._plan, p, C.byref(v))
            out[p] = v.value
        return out

    def set_split(self, prec, lanes):
        _call("mpb_batch_gemv_set_split", self._plan, int(prec), int(lanes))

    def close(self):
        if getattr(self, "_plan", None):
            lib().mpb_batch_gemv_destroy(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = [
    "SUPPORTED", "MpbError", "aos_bytes", "tile_bytes", "vec_bytes", "build", "lib", "host_lib", "empty",
    "empty_matrix", "pack_aos", "unpack_aos", "from_double", "to_double", "binop", "fma", "div", "sqrt", "exp", "log",
    "axpy",
    "gemv", "gemm",
    "layout", "MPB_OP_MUL", "MPB_OP_ADD", "MPB_OP_SUB", "gemm_exact", "gemm_exact_workspace", "gemm_exact_info",
    "BatchGemv",
    "GemvProblem",
]
