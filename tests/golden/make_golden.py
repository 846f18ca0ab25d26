"""Generate tests/golden/ref_vectors.npz from the reference's OWN arithmetic.

The reference (tkouya/mpc_cuda) commits no golden vectors; its tests
regenerate expectations from seeds and MPFR at run time.  This script runs
the reference's include/mpc_cuda/cu_freal.cuh and cu_fcomplex.cuh, compiled
for the host into oracle/_ref/libref_host.so (make -C oracle, which needs the
reference tree), on seeded operands from the reference's own generator
(xorshift64 randf, tools/test_freal.cu:15-27,55) and stores inputs and
outputs, so the pin holds on machines without the reference tree.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402

PRECS = (64, 96, 128, 256, 512, 1024, 2048)
NREAL, NCPLX = 40, 12
GM, GN, GK = 3, 4, 5


def main():
    if not O.ref_available():
        sys.exit("oracle/_ref/libref_host.so missing: build it with make -C oracle where the reference tree exists")
    out = {}
    for P in PRECS:
        A, B = O.gen_pairs(P, NREAL, 0xC0FFEE + P)
        out[f"r{P}_a"], out[f"r{P}_b"] = A, B
        for kind in ("mul", "add", "sub"):
            out[f"r{P}_{kind}"] = O.binop(kind, P, A, B, "ref")
        Ac, Bc = O.gen_pairs(P, NCPLX, 0xFACADE + P, cplx=True)
        out[f"c{P}_a"], out[f"c{P}_b"] = Ac, Bc
        for kind in ("cmul", "cadd", "csub"):
            out[f"c{P}_{kind}"] = O.binop(kind, P, Ac, Bc, "ref")
        out[f"r{P}_axpy"] = O.axpy(P, A[:1].copy(), A, B, impl="ref")
        out[f"c{P}_axpy"] = O.axpy(P, Ac[:1].copy(), Ac, Bc, True, impl="ref")
        Ga, _ = O.gen_pairs(P, GM * GK, 0xABBA + P)
        Gb, _ = O.gen_pairs(P, GK * GN, 0xBAAB + P)
        out[f"r{P}_ga"], out[f"r{P}_gb"] = Ga, Gb
        out[f"r{P}_gemm"] = O.gemm(P, GM, GN, GK, Ga, GK, Gb, GN, impl="ref")
        Gca, _ = O.gen_pairs(P, GM * GK, 0xCAFE + P, cplx=True)
        Gcb, _ = O.gen_pairs(P, GK * GN, 0xDEAF + P, cplx=True)
        out[f"c{P}_ga"], out[f"c{P}_gb"] = Gca, Gcb
        out[f"c{P}_gemm"] = O.gemm(P, GM, GN, GK, Gca, GK, Gcb, GN, True, impl="ref")
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_vectors.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
