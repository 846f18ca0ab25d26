#!/usr/bin/env python3
"""Writes consts.cuh: ln 2 as 72 little-endian 32-bit words of
floor(ln2 * 2^2304) (2304 bits: the working precision of the largest supported
PB, 2048, plus 128 guard bits, plus margin).

ln 2 = sum_{k>=1} 1 / (k 2^k); each term is floored at 2304 + 64 bits, so the
sum is below the true value by less than 2400 units of 2^-(2304+64), far below
the last kept bit; the script also checks the top words against float ln 2.

    python include/mpb/make_consts.py > include/mpb/consts.cuh
"""
import math

WORDS = 72
P = 32 * WORDS
G = 64
s = 0
k = 1
while True:
    t = (1 << (P + G)) // (k << k)
    if t == 0:
        break
    s += t
    k += 1
ln2 = s >> G
assert abs((ln2 >> (P - 60)) / 2.0 ** 60 - math.log(2.0)) < 1e-15
words = [(ln2 >> (32 * i)) & 0xFFFFFFFF for i in range(WORDS)]
assert words[-1] >> 31 == 1
print("/* consts.cuh -- generated by make_consts.py; do not edit.")
print(" * ln 2 = sum(ln2_word(i) 2^(32 i)) / 2^(32 * 72), truncated. */")
print("#ifndef MPB_CONSTS_CUH")
print("#define MPB_CONSTS_CUH")
print("namespace mpb {")
print(f"constexpr int kLn2WordCount = {WORDS};")
print("#if defined(__CUDACC__)")
print("__host__ __device__")
print("#endif")
print("inline uint32_t ln2_word(int i) {")
print("  constexpr uint32_t w[72] = {")
for i in range(0, WORDS, 6):
    print("      " + ", ".join(f"0x{x:08x}u" for x in words[i:i + 6]) + ",")
print("  };")
print("  return w[i];")
print("}")
print("}  // namespace mpb")
print("#endif")
