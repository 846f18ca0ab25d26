"""Batched GEMV: thousands of independent problems y = A.x + y of uneven sizes
and mixed precisions, planned once and run as one fork/join of persistent
kernels (capturable in a CUDA graph).  Every result must be bit-exact with
MPFR at its own precision, in mpb_gemv_r's order (sequential k, one rounding
per operation, then + y)."""
import numpy as np
import pytest

from conftest import to_dev, to_host
from mpc_cuda_b200 import layout, synth

pytestmark = pytest.mark.gpu


def make_batch(count, seed, lo=1, hi=130, exps=24, precs=layout.SUPPORTED, empties=True):
    rng = np.random.default_rng(seed)
    m = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).round().astype(int)
    n = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).round().astype(int)
    p = rng.choice(precs, size=count)
    if empties:
        m[0], n[1] = 0, 0
    probs = []
    for i in range(count):
        prec, mi, ni = int(p[i]), int(m[i]), int(n[i])
        lda = max(32, -(-ni // 32) * 32)
        A = synth.random_elems(rng, prec, mi * ni, -exps, exps)
        x = synth.random_elems(rng, prec, ni, -exps, exps)
        y = synth.random_elems(rng, prec, mi, -exps, exps)
        L = np.zeros((mi, lda, prec // 32), np.uint32)
        H = np.full((mi, lda), layout.HEAD_ZERO, np.uint32)
        L[:, :ni] = A[0].reshape(mi, ni, prec // 32)
        H[:, :ni] = A[1].reshape(mi, ni)
        probs.append(dict(prec=prec, m=mi, n=ni, lda=lda, A=(A[0], A[1]), x=x, y=y,
                          dA=to_dev(layout.vec_from_parts(prec, L.reshape(mi * lda, -1), H.reshape(-1)))
                          if mi * ni else to_dev(np.zeros(16, np.uint8)),
                          dx=to_dev(layout.vec_from_parts(prec, *x)) if ni else to_dev(np.zeros(16, np.uint8)),
                          dy=to_dev(layout.vec_from_parts(prec, *y)) if mi else to_dev(np.zeros(16, np.uint8))))
    for pr in probs:
        import torch

        pr["dyo"] = torch.zeros(max(16, layout.vec_bytes(pr["prec"], pr["m"])), dtype=torch.uint8, device="cuda")
    return probs


def plan(mpb, probs):
    return mpb.BatchGemv([(p["prec"], p["m"], p["n"], p["lda"], p["dA"], p["dx"], p["dy"], p["dyo"]) for p in probs])


def expected(orc, p):
    prec, m, n = p["prec"], p["m"], p["n"]
    A = layout.aos_from_parts(prec, *p["A"])
    return orc.gemv(prec, m, n, A, n, layout.aos_from_parts(prec, *p["x"]),
                    layout.aos_from_parts(prec, *p["y"]), impl="mp")


def got(p):
    return layout.vec_to_aos(p["prec"], to_host(p["dyo"]), p["m"])


def test_batch_matches_mpfr_per_problem(orc, mpb):
    probs = make_batch(240, 7)
    b = plan(mpb, probs)
    b.run()
    for i, p in enumerate(probs):
        if p["m"] == 0:
            continue
        bad, first = orc.mismatches(p["prec"], got(p), expected(orc, p))
        assert bad == 0, f"problem {i} PB={p['prec']} {p['m']}x{p['n']}: first mismatch {first}"
    b.close()


def test_batch_graph_capture_autotune_and_replay(orc, mpb):
    import torch

    probs = make_batch(90, 11, hi=70)
    b = plan(mpb, probs)
    b.autotune()
    tune = b.tuning()
    assert all(blk % 32 == 0 and 32 <= blk <= 256 for blk, _ in tune.values())
    for p in probs:
        p["dyo"].zero_()
    s = torch.cuda.Stream()
    b.run(stream=s)  # plan-side set-up outside the capture
    torch.cuda.synchronize()
    for p in probs:
        p["dyo"].zero_()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        b.run(stream=s)
    for _ in range(2):
        for p in probs:
            p["dyo"].zero_()
        g.replay()
        torch.cuda.synchronize()
        for i, p in enumerate(probs):
            if p["m"]:
                assert orc.mismatches(p["prec"], got(p), expected(orc, p))[0] == 0, i
    del g
    b.close()


def upload_batch(probs, pools):
    """Device pools (one tiled buffer per precision and operand) and the
    BatchGemv problem tuples pointing into them."""
    import torch

    dev = {}
    for prec, P in pools.items():
        dev[prec] = {k: to_dev(layout.vec_from_parts(prec, *P[k])) for k in ("A", "x", "y")}
        dev[prec]["yo"] = torch.zeros_like(dev[prec]["y"])
    tup = []
    for pr in probs:
        d, vb = dev[pr["prec"]], (lambda off, p=pr["prec"]: layout.vec_bytes(p, off))
        tup.append((pr["prec"], pr["m"], pr["n"], pr["lda"], d["A"].data_ptr() + vb(pr["a_off"]),
                    d["x"].data_ptr() + vb(pr["x_off"]), d["y"].data_ptr() + vb(pr["y_off"]),
                    d["yo"].data_ptr() + vb(pr["y_off"])))
    return dev, tup


def test_batch_full_size_4096_problems(orc, mpb):
    """The batched workload at full size: 4096 problems, m, n log-uniform in
    [16, 512], PB uniform over the six precisions, exponents in [-24, 24].
    Every result equals the single-problem kernel's; a sample equals MPFR."""
    import torch

    probs, pools = synth.gemv_batch()
    dev, tup = upload_batch(probs, pools)
    b = mpb.BatchGemv(tup)
    b.autotune()
    for d in dev.values():
        d["yo"].zero_()
    b.run()
    torch.cuda.synchronize()
    batched = {p: to_host(d["yo"]) for p, d in dev.items()}
    for d in dev.values():
        d["yo"].zero_()
    for t in tup:
        mpb.gemv(t[0], t[1], t[2], t[4], t[3], t[5], t[6], t[7])
    torch.cuda.synchronize()
    for p, d in dev.items():
        assert np.array_equal(batched[p], to_host(d["yo"])), f"PB={p}: batched results differ from mpb_gemv_r"
    rng = np.random.default_rng(3)
    for i in rng.choice(len(probs), 24, replace=False):
        pr = probs[i]
        prec, m, n = pr["prec"], pr["m"], pr["n"]
        A, x, y = synth.gemv_batch_problem(pools, pr)
        want = orc.gemv(prec, m, n, layout.aos_from_parts(prec, *A), n, layout.aos_from_parts(prec, *x),
                        layout.aos_from_parts(prec, *y), impl="mp")
        tiles = batched[prec][layout.vec_bytes(prec, pr["y_off"]):]
        assert orc.mismatches(prec, layout.vec_to_aos(prec, tiles, m), want)[0] == 0, i
    b.close()
