"""Arguments for the elementary-function tests (host build and GPU).

Random arguments follow the reference's accuracy tests: full-width random
significands with the exponent ranges of tools/test_fmath.cu:57-59 (exp,
expm1, log1p, atan, sinh, cosh: spread 3, expm1 / log1p shifted down by 6;
log: 20, positive; sin / cos / tan: 5) and tools/test_fmath3.cu:44-50
(asin / acos / atanh: |x| < 1, exponent in [-4, 0]; pow: x > 0 with exponent
in [-3, 3], y in [-2, 2]).  The hard sets add what those tests do not reach:
arguments next to multiples of pi/2, logarithms next to 1, tiny and huge
magnitudes, the ends of the asin / acos / atanh domains.  They are exact
roundings of high-precision values (mpmath).
"""
import mpmath
import numpy as np

FN = ("exp", "log", "expm1", "log1p", "sin", "cos", "tan", "atan", "sinh", "cosh",
      "atanh", "asin", "acos", "cbrt", "pow", "atan2")
CFN = ("exp", "log", "sqrt", "sin", "cos", "tan", "sinh", "cosh", "div")

# (exponent lo, exponent hi, positive)
RANGES = {
    "exp": (-3, 3, False), "log": (-20, 20, True), "expm1": (-12, 0, False), "log1p": (-12, 0, False),
    "sin": (-5, 5, False), "cos": (-5, 5, False), "tan": (-5, 5, False), "atan": (-3, 3, False),
    "sinh": (-3, 3, False), "cosh": (-3, 3, False), "atanh": (-4, 0, False), "asin": (-4, 0, False),
    "acos": (-4, 0, False), "cbrt": (-20, 20, False), "pow": (-3, 3, True), "atan2": (-5, 5, False),
}


def random_args(orc, name, prec, n, seed):
    """(A, B) in the reference's test ranges; B only for pow / atan2."""
    lo, hi, pos = RANGES[name]
    A = orc.rand_elems(prec, n, seed, lo, hi, pos)
    B = orc.rand_elems(prec, n, seed + 1, -2, 2) if name in ("pow", "atan2") else None
    return A, B


def mp_elems(orc, prec, vals):
    """AoS elements: each value rounded to nearest at prec bits."""
    n64 = (prec + 63) // 64
    sb = 64 * n64 - prec
    out = orc.empty(prec, len(vals))
    for i, v in enumerate(vals):
        v = mpmath.mpf(v)
        if v == 0:
            out[i] = orc.from_double(prec, [0.0])[0]
            continue
        a = abs(v)
        e = int(mpmath.floor(mpmath.log(a, 2))) + 1
        M = int(mpmath.nint(mpmath.ldexp(a, prec - e)))
        while M >> prec:
            M >>= 1
            e += 1
        while M < (1 << (prec - 1)):
            M <<= 1
            e -= 1
        out[i, 0:4] = np.array([-1 if v < 0 else 1], np.int32).view(np.uint8)
        out[i, 8:16] = np.array([e], np.int64).view(np.uint8)
        out[i, 16:] = np.frombuffer((M << sb).to_bytes(8 * n64, "little"), np.uint8)
    return out


def hard_args(orc, prec, seed):
    """name -> AoS arguments for that function's hard regions (full-width
    significands: the random factors carry 2 PB + 64 random bits)."""
    rng = np.random.default_rng(seed)
    nbytes = (2 * prec + 64) // 8

    def uni(lo, hi):
        f = mpmath.mpf(int.from_bytes(rng.bytes(nbytes), "little")) / mpmath.mpf(2) ** (8 * nbytes)
        return lo + (hi - lo) * f

    def p2(lo, hi):
        return mpmath.mpf(2) ** int(rng.integers(lo, hi))

    with mpmath.workprec(4 * prec + 64):
        ks = list(range(1, 41)) + [1000003, 2 ** 20 + 7, 123456789]
        kpi2 = [k * mpmath.pi / 2 for k in ks] + [-k * mpmath.pi / 2 for k in ks[:10]]
        big = [uni(1, 2) * p2(10, 29) * (1 if i % 2 else -1) for i in range(20)]
        near1 = [1 + uni(-1, 1) / p2(1, prec + 8) for _ in range(30)]
        tiny = [uni(-1, 1) / p2(20, 3000) for _ in range(20)]
        ends = [(1 - 1 / p2(1, prec + 1)) * (1 if i % 2 else -1) for i in range(24)]
        wide = [uni(-1, 1) * p2(0, 26) for _ in range(20)]
        huge = [uni(-1, 1) * p2(30, 3000) for _ in range(20)]
        sets = {
            "sin": kpi2 + big + tiny, "cos": kpi2 + big, "tan": kpi2 + big + tiny,
            "log": near1 + [abs(v) for v in huge + tiny], "log1p": tiny + ends,
            "expm1": tiny + wide, "exp": wide + tiny, "sinh": tiny + wide, "cosh": wide,
            "atan": tiny + huge, "asin": tiny + ends, "acos": ends + tiny, "atanh": tiny + ends,
            "cbrt": huge + tiny + [mpmath.mpf(27), mpmath.mpf(-8), mpmath.mpf(1) / 64],
        }
        return {k: mp_elems(orc, prec, v) for k, v in sets.items()}


def special_args():
    """(function, argument(s), expected value) for the documented edges, as
    doubles: values with no representation give 0, the reference's clamps."""
    return [
        ("log", (-1.5,), 0.0), ("log", (0.0,), 0.0), ("log", (1.0,), 0.0), ("log1p", (-1.0,), 0.0),
        ("log1p", (-3.0,), 0.0), ("atanh", (1.0,), 0.0), ("atanh", (-2.0,), 0.0), ("asin", (1.0,), "pi/2"),
        ("asin", (-3.0,), "-pi/2"), ("acos", (1.0,), 0.0), ("acos", (2.0,), 0.0), ("acos", (-1.0,), "pi"),
        ("pow", (-2.0, 0.5), 0.0), ("pow", (-2.0, 3.0), -8.0), ("pow", (-2.0, 2.0), 4.0), ("pow", (0.0, 2.5), 0.0),
        ("pow", (5.0, 0.0), 1.0), ("pow", (0.0, 0.0), 1.0), ("exp", (0.0,), 1.0), ("cos", (0.0,), 1.0),
        ("cosh", (0.0,), 1.0), ("sin", (0.0,), 0.0), ("tan", (0.0,), 0.0), ("atan", (0.0,), 0.0),
        ("expm1", (0.0,), 0.0), ("cbrt", (0.0,), 0.0), ("cbrt", (-27.0,), -3.0), ("exp", (2.0 ** 30,), 0.0),
        ("sinh", (-(2.0 ** 29),), 0.0), ("expm1", (-(2.0 ** 30),), -1.0), ("sin", (2.0 ** 31,), 0.0),
        ("atan2", (0.0, 0.0), 0.0), ("atan2", (1.0, 0.0), "pi/2"), ("atan2", (-1.0, 0.0), "-pi/2"),
        ("atan2", (0.0, -1.0), "pi"), ("atan", (1.0,), "pi/4"),
    ]
