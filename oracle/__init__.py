"""CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loaded only by ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py``, as the checker or as the timed CPU baseline.  The product
(``mpc_cuda_b200``) never imports this package.

Three libraries are wrapped:

* ``liboracle.so`` -- ``mpb_oracle.c``: a C restatement of the reference's
  ``cu_freal``/``cu_fcomplex`` arithmetic and kernel loops (``orc_*``) and the
  same operations through the system MPFR 4.2.1 / MPC 1.3.1 (``mp_*``).
* ``_ref/libref_host.so`` -- the reference's own headers compiled for the host
  (``ref_*``); present only where the reference tree was available at build
  time (it travels as a prebuilt file).

Every buffer is a numpy ``uint8`` array holding the reference's AoS element
layout ``cu_freal<PB>`` = ``{int32 sign; int32 pad; int64 exp; uint64 m[N64]}``
(complex: ``{re, im}``), see ``mpc_cuda_b200.layout``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None


# where the reference tree is mounted in the build container (read-only); the
# GPU machines have no copy and use the libraries built here
REFERENCE_TREE = os.environ.get("MPB_REFERENCE_TREE", "/root/reference")


def build(quiet: bool = True) -> None:
    """Compile liboracle.so, and _ref/libref_host.so when the reference tree exists."""
    cmd = ["make", "-C", HERE]
    inc = os.path.join(REFERENCE_TREE, "include")
    if os.path.isfile(os.path.join(inc, "mpc_cuda", "cu_freal.cuh")):
        cmd.append("REF_INCLUDE=" + inc)
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp, lg, it = C.c_void_p, C.c_long, C.c_int
        for name in ("orc_mul", "orc_add", "orc_sub", "orc_cmul", "orc_cadd", "orc_csub",
                     "mp_mul", "mp_add", "mp_sub", "mp_cmul", "mp_cadd", "mp_csub"):
            getattr(L, name).argtypes = [it, lg, vp, vp, vp]
        L.mp_div.argtypes = [it, lg, vp, vp, vp]
        L.mp_sqrt.argtypes = [it, lg, vp, vp]
        L.mp_exp.argtypes = [it, it, lg, vp, vp]
        L.mp_log.argtypes = [it, it, lg, vp, vp]
        for name in ("mp_fn", "mp_cfn"):
            getattr(L, name).argtypes = [it, it, it, lg, vp, vp, vp]
        L.mp_div_ui.argtypes = [it, lg, vp, C.c_ulong, vp]
        L.mp_const.argtypes = [it, it, vp]
        L.mp_op_rp.argtypes = [it, it, it, lg, vp, vp, vp, vp]
        for name in ("orc_fma", "mp_fma", "mp_cfma", "mp_cfma_dot"):
            getattr(L, name).argtypes = [it, lg, vp, vp, vp, vp]
        for name in ("orc_axpy_r", "orc_axpy_c", "mp_axpy_r", "mp_axpy_c"):
            getattr(L, name).argtypes = [it, lg, vp, vp, vp, vp]
        for name in ("orc_gemv_r", "orc_gemv_c", "mp_gemv_r", "mp_gemv_c"):
            getattr(L, name).argtypes = [it, lg, lg, vp, lg, vp, vp, vp]
        for name in ("orc_gemm_r", "orc_gemm_c", "mp_gemm_r", "mp_gemm_c"):
            getattr(L, name).argtypes = [it, lg, lg, lg, vp, lg, vp, lg, vp, lg, lg, lg]
        for name in ("orc_gemm_exact_r", "orc_gemm_exact_c", "mp_gemm_exact_r", "mp_gemm_exact_c"):
            getattr(L, name).argtypes = [it, it, lg, lg, lg, vp, lg, vp, lg, vp, lg, lg, lg]
        L.orc_convert.argtypes = [it, it, lg, vp, vp]
        L.orc_from_double.argtypes = [it, lg, vp, vp]
        L.orc_count_mismatch.argtypes = [it, lg, vp, vp, C.POINTER(C.c_long)]
        L.orc_count_mismatch.restype = C.c_long
        L.orc_ulp_err.argtypes = [it, vp, it, vp]
        L.orc_ulp_err.restype = C.c_double
        for name in ("orc_gen_pairs_r", "orc_gen_pairs_c"):
            getattr(L, name).argtypes = [it, lg, C.c_uint64, vp, vp]
            getattr(L, name).restype = C.c_uint64
        L.orc_elem_bytes.argtypes = [it]
        L.orc_elem_bytes.restype = C.c_size_t
        L.orc_mpfr_version.restype = C.c_char_p
        L.orc_mpc_version.restype = C.c_char_p
        L.orc_num_threads.restype = C.c_int
        _LIB = L
    return _LIB


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libref_host.so"))


def ref():
    """The reference's own headers compiled for the host (None if not built)."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libref_host.so")
        if not os.path.exists(path):
            return None
        R = C.CDLL(path)
        vp, lg, it = C.c_void_p, C.c_long, C.c_int
        for name in ("ref_mul", "ref_add", "ref_sub", "ref_cmul", "ref_cadd", "ref_csub"):
            getattr(R, name).argtypes = [it, lg, vp, vp, vp]
        for name in ("ref_axpy_r", "ref_axpy_c"):
            getattr(R, name).argtypes = [it, lg, vp, vp, vp, vp]
        for name in ("ref_gemv_r", "ref_gemv_c"):
            getattr(R, name).argtypes = [it, lg, lg, vp, lg, vp, vp, vp]
        for name in ("ref_gemm_r", "ref_gemm_c"):
            getattr(R, name).argtypes = [it, lg, lg, lg, vp, lg, vp, lg, vp, lg, lg, lg]
        R.ref_div.argtypes = [it, lg, vp, vp, vp]
        R.ref_sqrt.argtypes = [it, lg, vp, vp]
        R.ref_exp.argtypes = [it, lg, vp, vp]
        R.ref_log.argtypes = [it, lg, vp, vp]
        for name in ("ref_fn", "ref_cfn"):
            getattr(R, name).argtypes = [it, it, lg, vp, vp, vp]
        R.ref_from_double.argtypes = [it, lg, vp, vp]
        R.ref_to_double.argtypes = [it, lg, vp, vp]
        R.ref_elem_bytes.argtypes = [it]
        _REF = R
    return _REF


# ---------------------------------------------------------------- helpers
def elem_bytes(prec: int) -> int:
    return 16 + 8 * ((prec + 63) // 64)


def empty(prec: int, n: int, cplx: bool = False) -> np.ndarray:
    return np.zeros((n, (2 if cplx else 1) * elem_bytes(prec)), dtype=np.uint8)


def gen_pairs(prec: int, n: int, seed: int, cplx: bool = False):
    """The reference's seeded random operand pairs (tools/test_freal.cu:55,
    tools/test_fcomplex.cu:55-57): xorshift64 stream, exponent spread 40 for
    three of every four pairs and PB+200 for the fourth."""
    A, B = empty(prec, n, cplx), empty(prec, n, cplx)
    f = lib().orc_gen_pairs_c if cplx else lib().orc_gen_pairs_r
    f(prec, n, seed, _p(A), _p(B))
    return A, B


def rand_elems(prec: int, n: int, seed: int, elo: int, ehi: int, positive: bool = False,
               cplx: bool = False) -> np.ndarray:
    """n random elements in the reference's test layout (tools/test_fmath.cu:
    14-20 randf): full-width random significands (top bit set, the bits below
    PB clear), exponents uniform in [elo, ehi], random signs unless positive."""
    rng = np.random.default_rng(seed)
    n64, es = (prec + 63) // 64, elem_bytes(prec)
    parts = []
    for _ in range(2 if cplx else 1):
        m = rng.integers(0, 1 << 63, size=(n, n64), dtype=np.uint64) * np.uint64(2) + \
            rng.integers(0, 2, size=(n, n64), dtype=np.uint64)
        m[:, -1] |= np.uint64(1 << 63)
        sb = 64 * n64 - prec
        if sb:
            m[:, 0] &= ~np.uint64((1 << sb) - 1)
        E = np.zeros((n, es), np.uint8)
        sign = np.ones(n, np.int32) if positive else rng.choice(np.array([-1, 1], np.int32), n)
        E[:, 0:4] = sign.view(np.uint8).reshape(n, 4)
        E[:, 8:16] = rng.integers(elo, ehi + 1, n).astype(np.int64).view(np.uint8).reshape(n, 8)
        E[:, 16:] = m.view(np.uint8).reshape(n, 8 * n64)
        parts.append(E)
    return np.concatenate(parts, axis=1) if cplx else parts[0]


def mismatches(prec: int, X: np.ndarray, Y: np.ndarray, cplx: bool = False):
    """(count, first index) of entries that differ as values (+0 == -0)."""
    n = X.shape[0] * (2 if cplx else 1)
    first = C.c_long(-1)
    cnt = lib().orc_count_mismatch(prec, n, _p(np.ascontiguousarray(X)),
                                   _p(np.ascontiguousarray(Y)), C.byref(first))
    return int(cnt), int(first.value)


def binop(kind: str, prec: int, A: np.ndarray, B: np.ndarray, impl: str = "orc") -> np.ndarray:
    """kind in mul/add/sub/cmul/cadd/csub; impl 'orc' (restatement), 'mp' (MPFR/MPC), 'ref'."""
    cplx = kind.startswith("c")
    R = empty(prec, A.shape[0], cplx)
    if impl == "ref":
        rc = getattr(ref(), "ref_" + kind)(prec, A.shape[0], _p(A), _p(B), _p(R))
        if rc != 0:
            raise ValueError(f"reference host build has no PB={prec}")
    else:
        getattr(lib(), f"{impl}_{kind}")(prec, A.shape[0], _p(A), _p(B), _p(R))
    return R


def from_double(prec: int, d) -> np.ndarray:
    """Exact conversion of doubles to AoS elements (the restatement's from_double)."""
    d = np.ascontiguousarray(d, dtype=np.float64)
    R = empty(prec, d.shape[0])
    lib().orc_from_double(prec, d.shape[0], _p(d), _p(R))
    return R


def div(prec: int, A, B, impl: str = "mp") -> np.ndarray:
    """a / b: 'mp' = round(a / b) by the system MPFR (mpfr_div, RNDN); 'ref' =
    the reference's own faithful cu_fdiv built for the host."""
    R = empty(prec, A.shape[0])
    f = ref().ref_div if impl == "ref" else lib().mp_div
    f(prec, A.shape[0], _p(A), _p(B), _p(R))
    return R


def sqrt(prec: int, A, impl: str = "mp") -> np.ndarray:
    """sqrt(a): 'mp' = mpfr_sqrt (RNDN); 'ref' = the reference's cu_sqrt."""
    R = empty(prec, A.shape[0])
    f = ref().ref_sqrt if impl == "ref" else lib().mp_sqrt
    f(prec, A.shape[0], _p(A), _p(R))
    return R


def exp(prec: int, A, out_prec: int | None = None, impl: str = "mp") -> np.ndarray:
    """exp(a): 'mp' = mpfr_exp rounded at out_prec bits (default prec); 'ref' =
    the reference's own faithful cu_exp built for the host."""
    po = out_prec or prec
    R = empty(po, A.shape[0])
    if impl == "ref":
        ref().ref_exp(prec, A.shape[0], _p(A), _p(R))
    else:
        lib().mp_exp(prec, po, A.shape[0], _p(A), _p(R))
    return R


def log(prec: int, A, out_prec: int | None = None, impl: str = "mp") -> np.ndarray:
    """log(a): 'mp' = mpfr_log at out_prec bits; 'ref' = the reference's cu_log."""
    po = out_prec or prec
    R = empty(po, A.shape[0])
    if impl == "ref":
        ref().ref_log(prec, A.shape[0], _p(A), _p(R))
    else:
        lib().mp_log(prec, po, A.shape[0], _p(A), _p(R))
    return R


# elementary functions, numbered as the engine's MPB_FN_* / MPB_CFN_*
FN = ("exp", "log", "expm1", "log1p", "sin", "cos", "tan", "atan", "sinh", "cosh",
      "atanh", "asin", "acos", "cbrt", "pow", "atan2")
CFN = ("exp", "log", "sqrt", "sin", "cos", "tan", "sinh", "cosh", "div")


def fn(name: str, prec: int, A, B=None, out_prec: int | None = None, impl: str = "mp") -> np.ndarray:
    """Real function ``name`` (FN; pow / atan2 take B): 'mp' = MPFR rounded at
    out_prec bits (default prec); 'ref' = the reference's own cu_fmath
    function built for the host (at prec)."""
    f = FN.index(name)
    n = A.shape[0]
    po = prec if impl == "ref" else (out_prec or prec)
    R = empty(po, n)
    pb = _p(B) if B is not None else None
    if impl == "ref":
        ref().ref_fn(f, prec, n, _p(A), pb, _p(R))
    else:
        lib().mp_fn(f, prec, po, n, _p(A), pb, _p(R))
    return R


def cfn(name: str, prec: int, A, B=None, out_prec: int | None = None, impl: str = "mp") -> np.ndarray:
    """Complex function ``name`` (CFN; div takes B): 'mp' = MPC (each component
    rounded to nearest at out_prec bits); 'ref' = the reference's cu_fcmath."""
    f = CFN.index(name)
    n = A.shape[0]
    po = prec if impl == "ref" else (out_prec or prec)
    R = empty(po, n, True)
    pb = _p(B) if B is not None else None
    if impl == "ref":
        ref().ref_cfn(f, prec, n, _p(A), pb, _p(R))
    else:
        lib().mp_cfn(f, prec, po, n, _p(A), pb, _p(R))
    return R


def div_ui(prec: int, A, u: int) -> np.ndarray:
    """round(a / u), mpfr_div_ui (RNDN)."""
    R = empty(prec, A.shape[0])
    lib().mp_div_ui(prec, A.shape[0], _p(A), u, _p(R))
    return R


def op_rp(op: str, p: int, P: int, A, B=None, Cc=None) -> np.ndarray:
    """op (mul, add, sub, fma, div, sqrt) rounded to nearest at p bits by the
    system MPFR, operands and results in the P-bit element format."""
    R = empty(P, A.shape[0])
    lib().mp_op_rp(("mul", "add", "sub", "fma", "div", "sqrt").index(op), p, P, A.shape[0], _p(A), _p(B), _p(Cc),
                   _p(R))
    return R


def const(which: str, prec: int) -> np.ndarray:
    """pi or ln2 rounded to nearest at prec bits (mpfr_const_pi / _log2)."""
    R = empty(prec, 1)
    lib().mp_const(0 if which == "pi" else 1, prec, _p(R))
    return R


def fma(prec: int, A, B, Cc, impl: str = "orc", cplx: bool = False) -> np.ndarray:
    """a*b + c, one rounding (per component).  Complex: impl 'mp' = mpc_fma,
    'mpdot' = mpc_dot over ([a, c], [b, 1]); the reference has no fma."""
    R = empty(prec, A.shape[0], cplx)
    if cplx:
        if impl not in ("mp", "mpdot"):
            raise ValueError("complex fma: impl 'mp' or 'mpdot'")
        name = "mp_cfma_dot" if impl == "mpdot" else "mp_cfma"
    else:
        name = f"{impl}_fma"
    getattr(lib(), name)(prec, A.shape[0], _p(A), _p(B), _p(Cc), _p(R))
    return R


def axpy(prec: int, a, X, Y, cplx: bool = False, impl: str = "orc") -> np.ndarray:
    n = X.shape[0]
    Z = empty(prec, n, cplx)
    suffix = "c" if cplx else "r"
    if impl == "ref":
        getattr(ref(), "ref_axpy_" + suffix)(prec, n, _p(a), _p(X), _p(Y), _p(Z))
    else:
        getattr(lib(), f"{impl}_axpy_{suffix}")(prec, n, _p(a), _p(X), _p(Y), _p(Z))
    return Z


def gemv(prec: int, m, n, A, lda, x, y, cplx: bool = False, impl: str = "orc") -> np.ndarray:
    Y = empty(prec, m, cplx)
    suffix = "c" if cplx else "r"
    f = getattr(ref(), "ref_gemv_" + suffix) if impl == "ref" else getattr(lib(), f"{impl}_gemv_{suffix}")
    f(prec, m, n, _p(A), lda, _p(x), _p(y), _p(Y))
    return Y


def gemm(prec: int, m, n, k, A, lda, B, ldb, cplx: bool = False, impl: str = "orc",
         rows=None) -> np.ndarray:
    """Sequential-k, per-operation-rounded C = A.B; ``rows=(r0, r1)`` limits the
    rows computed (others stay zero)."""
    Cm = empty(prec, m * n, cplx)
    r0, r1 = rows if rows else (0, m)
    suffix = "c" if cplx else "r"
    f = getattr(ref(), "ref_gemm_" + suffix) if impl == "ref" else getattr(lib(), f"{impl}_gemm_{suffix}")
    f(prec, m, n, k, _p(A), lda, _p(B), ldb, _p(Cm), n, r0, r1)
    return Cm


def gemm_exact(prec: int, m, n, k, A, lda, B, ldb, cplx: bool = False, impl: str = "orc",
               out_prec: int | None = None, rows=None) -> np.ndarray:
    """Correctly rounded C = A.B (one rounding per entry) at ``out_prec`` bits."""
    po = out_prec or prec
    Cm = empty(po, m * n, cplx)
    r0, r1 = rows if rows else (0, m)
    suffix = "c" if cplx else "r"
    getattr(lib(), f"{impl}_gemm_exact_{suffix}")(prec, po, m, n, k, _p(A), lda, _p(B), ldb,
                                                  _p(Cm), n, r0, r1)
    return Cm


def ulp_errors(prec: int, X: np.ndarray, ref_prec: int, Y: np.ndarray) -> np.ndarray:
    """Per-entry |x - y| in ULPs of a ``prec``-bit number with y's exponent."""
    ex, ey = elem_bytes(prec), elem_bytes(ref_prec)
    Xf = np.ascontiguousarray(X).reshape(-1, ex)
    Yf = np.ascontiguousarray(Y).reshape(-1, ey)
    L = lib()
    out = np.empty(Xf.shape[0])
    bx, by = Xf.ctypes.data, Yf.ctypes.data
    for i in range(Xf.shape[0]):
        out[i] = L.orc_ulp_err(prec, C.c_void_p(bx + i * ex), ref_prec, C.c_void_p(by + i * ey))
    return out


def convert(to_prec: int, from_prec: int, X: np.ndarray) -> np.ndarray:
    n = X.size // elem_bytes(from_prec)
    R = empty(to_prec, n)
    lib().orc_convert(to_prec, from_prec, n, _p(np.ascontiguousarray(X)), _p(R))
    return R


def versions():
    L = lib()
    return L.orc_mpfr_version().decode(), L.orc_mpc_version().decode()


def num_threads() -> int:
    return int(lib().orc_num_threads())
