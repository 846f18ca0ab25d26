#!/usr/bin/env python3
"""Writes consts.cuh: ln 2 and pi as little-endian 32-bit words, truncated.

  ln 2: 72 words of floor(ln2 * 2^2304) (the working precision of the largest
        supported PB, 2048, plus 128 guard bits, plus margin), from
        ln 2 = sum_{k>=1} 1 / (k 2^k).
  pi:   136 words of floor(pi / 4 * 2^4352): the argument reduction of sin /
        cos / tan works at 2 N + 4 limbs (132 at PB = 2048), from Machin's
        formula pi / 4 = 4 atan(1/5) - atan(1/239).

Every series term is floored 64 bits below the last kept bit, so each sum is
below the true value by less than one unit of the kept precision.  The script
checks the top words against the float constants, and that rounding the
truncated words at every supported PB from N + 4 words -- what the engine's
pi() and ln2() do -- gives the correctly rounded constant (the bits below
position PB are never within one unit of the halfway point).

    python include/mpb/make_consts.py > include/mpb/consts.cuh
"""
import math

G = 64


def ln2_fixed(P):
    s, k = 0, 1
    while True:
        t = (1 << (P + G)) // (k << k)
        if t == 0:
            return s >> G
        s += t
        k += 1


def atan_inv_fixed(x, P):
    """atan(1/x) * 2^(P+G), terms floored"""
    one = 1 << (P + G)
    s, t, k, x2 = 0, one // x, 0, x * x
    while t:
        s += t // (2 * k + 1) if k % 2 == 0 else -(t // (2 * k + 1))
        t //= x2
        k += 1
    return s


def pi4_fixed(P):
    return (4 * atan_inv_fixed(5, P) - atan_inv_fixed(239, P)) >> G


def words_of(v, n):
    w = [(v >> (32 * i)) & 0xFFFFFFFF for i in range(n)]
    assert w[-1] >> 31 == 1
    return w


def check_rounding(words, name):
    n = len(words)
    v = sum(w << (32 * i) for i, w in enumerate(words))
    for pb in (64, 128, 256, 512, 1024, 2048):
        nw = pb // 32 + 4
        t = v >> (32 * (n - nw))  # top nw words
        tail = t & ((1 << 128) - 1)
        half = 1 << 127
        assert abs(tail - half) > 1, f"{name}: rounding at PB={pb} is within one unit of halfway"


LN2_WORDS, PI_WORDS = 72, 136
ln2 = ln2_fixed(32 * LN2_WORDS)
pi4 = pi4_fixed(32 * PI_WORDS)
assert abs((ln2 >> (32 * LN2_WORDS - 60)) / 2.0 ** 60 - math.log(2.0)) < 1e-15
assert abs((pi4 >> (32 * PI_WORDS - 60)) / 2.0 ** 60 - math.pi / 4) < 1e-15
wl, wp = words_of(ln2, LN2_WORDS), words_of(pi4, PI_WORDS)
check_rounding(wl, "ln2")
check_rounding(wp, "pi")


def table(name, words):
    print("#if defined(__CUDACC__)")
    print("__host__ __device__")
    print("#endif")
    print(f"inline uint32_t {name}(int i) {{")
    print(f"  constexpr uint32_t w[{len(words)}] = {{")
    for i in range(0, len(words), 6):
        print("      " + ", ".join(f"0x{x:08x}u" for x in words[i:i + 6]) + ",")
    print("  };")
    print("  return w[i];")
    print("}")


print("/* consts.cuh -- generated by make_consts.py; do not edit.")
print(f" * ln 2 = sum(ln2_word(i) 2^(32 i)) / 2^(32 * {LN2_WORDS}) and")
print(f" * pi / 4 = sum(pi_word(i) 2^(32 i)) / 2^(32 * {PI_WORDS}), both truncated. */")
print("#ifndef MPB_CONSTS_CUH")
print("#define MPB_CONSTS_CUH")
print("namespace mpb {")
print(f"constexpr int kLn2WordCount = {LN2_WORDS};")
print(f"constexpr int kPiWordCount = {PI_WORDS};")
table("ln2_word", wl)
table("pi_word", wp)
print("}  // namespace mpb")
print("#endif")
