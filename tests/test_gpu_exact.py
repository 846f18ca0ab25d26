"""Exact-accumulation GEMM on the INT8 tensor cores, through the C ABI.

Every entry is one rounding of the exact dot product, so it must equal the
system MPFR's mpfr_dot (the correctly rounded dot, pinned in test_oracle.py)
bit for bit, and lie within 0.5 ULP of a 4*PB oracle.  Rows/columns outside
the spread budget are computed by the plain per-operation kernel and must
equal the sequential-k MPFR oracle instead.
"""
import numpy as np
import pytest

from conftest import to_dev, to_host
from mpc_cuda_b200 import layout, synth

pytestmark = pytest.mark.gpu


def rand_aos(prec, count, seed, elo=-8, ehi=8, zero_frac=0.05):
    rng = np.random.default_rng(seed)
    return layout.aos_from_parts(prec, *synth.random_elems(rng, prec, count, elo, ehi, zero_frac))


def pad_rows(prec, A, rows, cols, ld):
    es = A.shape[1]
    z = layout.aos_from_parts(prec, np.zeros((1, prec // 32), np.uint32), np.array([layout.HEAD_ZERO], np.uint32))
    out = np.repeat(z, rows * ld, axis=0).reshape(rows, ld, es)
    out[:, :cols] = A.reshape(rows, cols, es)
    return out.reshape(rows * ld, es)


def run_exact(mpb, prec, m, n, k, A, B, sp_bits):
    import torch

    lda, ldb, ldc = (-(-k // 32) * 32, -(-n // 32) * 32, -(-n // 32) * 32)
    dA = to_dev(layout.aos_to_vec(prec, pad_rows(prec, A, m, k, lda)))
    dB = to_dev(layout.aos_to_vec(prec, pad_rows(prec, B, k, n, ldb)))
    Cd = mpb.empty(prec, m * ldc)
    st = torch.zeros(2, dtype=torch.int32, device="cuda")
    mpb.gemm_exact(prec, m, n, k, dA, lda, dB, ldb, Cd, ldc, sp_bits=sp_bits, status=st)
    C = layout.vec_to_aos(prec, to_host(Cd), m * ldc).reshape(m, ldc, -1)[:, :n].reshape(m * n, -1)
    return C, st.cpu().numpy()


@pytest.mark.parametrize("prec", (64, 256, 512, 1024, 2048))
@pytest.mark.parametrize("shape", ((1, 1, 1), (5, 7, 33), (33, 40, 17), (128, 256, 128), (130, 260, 300)))
def test_exact_vs_mpfr_dot(orc, mpb, prec, shape):
    m, n, k = shape
    if prec == 2048 and m * n * k > 200000:
        pytest.skip("covered at smaller shapes")
    A = rand_aos(prec, m * k, 100 + m + prec)
    B = rand_aos(prec, k * n, 200 + n + prec)
    C, st = run_exact(mpb, prec, m, n, k, A, B, sp_bits=16)
    assert st[1] == 0, f"kernel error code {st[1]}"
    assert st[0] == 0, "no row/column exceeds a 16-bit spread here"
    exp = orc.gemm_exact(prec, m, n, k, A, k, B, n, impl="mp")
    bad, first = orc.mismatches(prec, C, exp)
    assert bad == 0, f"PB={prec} {shape}: {bad} mismatches, first at {first}"


@pytest.mark.parametrize("prec", (128, 512))
def test_exact_cancellation_and_signs(orc, mpb, prec):
    """Columns of B that are exact negatives of each other give exact zeros and
    deep cancellation; the result must still be the correctly rounded sum."""
    m, n, k = 40, 64, 96
    A = rand_aos(prec, m * k, 7, -4, 4, 0.0)
    B = rand_aos(prec, k * n, 8, -4, 4, 0.0).reshape(k, n, -1)
    B[:, 1] = B[:, 0]
    B[:, 1, 0:4] = np.where(B[:, 0, 0:4].view(np.int32) > 0, -1, 1).astype(np.int32).view(np.uint8).reshape(k, 4)
    B[:, 3] = B[:, 2]
    B = B.reshape(k * n, -1)
    C, st = run_exact(mpb, prec, m, n, k, A, B, sp_bits=8)
    assert st[1] == 0
    exp = orc.gemm_exact(prec, m, n, k, A, k, B, n, impl="mp")
    assert orc.mismatches(prec, C, exp)[0] == 0


@pytest.mark.parametrize("prec", (128, 512))
def test_exact_uncertified_entries_are_recomputed(orc, mpb, prec):
    """Sums that cancel inside the dot product: the tensor cores skip the
    low-order slice pairs, so these entries cannot certify their rounding
    from the truncated sum and must be recomputed from the full sum.

    A = [H, H'] and, for the columns in J, B = [G; -G]: every such entry is
    exactly 0 (H' = H) or a residual ~2^-PB below its terms (rows in I, where
    H' differs from H in the last bit of one entry).  The other columns are
    ordinary random sums.  m, n span two output tiles each, so marked and
    unmarked tiles mix."""
    m, n, k = 130, 300, 96
    h = k // 2
    rng = np.random.default_rng(prec)
    H = rand_aos(prec, m * h, 31, -4, 4, 0.0).reshape(m, h, -1)
    H2 = H.copy()
    rows_i = rng.choice(m, 40, replace=False)
    H2[rows_i, 0, 16] ^= 1  # lowest limb byte of entry (i, h): last significand bit
    A = np.concatenate([H, H2], axis=1).reshape(m * k, -1)
    G = rand_aos(prec, h * n, 32, -4, 4, 0.0).reshape(h, n, -1)
    negG = G.copy()
    negG[:, :, 0:4] = (-negG[:, :, 0:4].view(np.int32)).view(np.uint8)
    B = np.concatenate([G, rand_aos(prec, h * n, 33, -4, 4, 0.0).reshape(h, n, -1)], axis=0)
    cols_j = rng.choice(n, 120, replace=False)
    B[h:, cols_j] = negG[:, cols_j]
    B = B.reshape(k * n, -1)
    C, st = run_exact(mpb, prec, m, n, k, A, B, sp_bits=16)
    assert st[1] == 0 and st[0] == 0
    exp = orc.gemm_exact(prec, m, n, k, A, k, B, n, impl="mp")
    bad, first = orc.mismatches(prec, C, exp)
    assert bad == 0, f"PB={prec}: {bad} mismatches, first at {first}"
    # the construction really produced exact zeros and deep cancellation
    Cm = C.reshape(m, n, -1)
    zero_exp = layout.AOS_ZERO_EXP
    ez = Cm[:, cols_j, 8:16].copy().view(np.int64).reshape(m, len(cols_j))
    others = np.setdiff1d(np.arange(m), rows_i)
    assert (ez[others] == zero_exp).all() and (ez[rows_i] != zero_exp).all()


def test_exact_fallback_rows_and_columns(orc, mpb):
    """Rows/columns whose exponent spread exceeds the budget take the plain
    per-operation-rounded kernel (never the CPU) and are counted."""
    prec, m, n, k = 256, 20, 40, 50
    A = rand_aos(prec, m * k, 31, -4, 4, 0.0).reshape(m, k, -1)
    B = rand_aos(prec, k * n, 32, -4, 4, 0.0).reshape(k, n, -1)
    for r in (3, 11):  # one tiny entry far below the row's top
        A[r, 5, 8:16] = np.array([-400], np.int64).view(np.uint8)
    B[7, 9, 8:16] = np.array([-400], np.int64).view(np.uint8)
    A, B = A.reshape(m * k, -1), B.reshape(k * n, -1)
    C, st = run_exact(mpb, prec, m, n, k, A, B, sp_bits=32)
    assert st[1] == 0 and st[0] == 3
    exact = orc.gemm_exact(prec, m, n, k, A, k, B, n, impl="mp").reshape(m, n, -1)
    plain = orc.gemm(prec, m, n, k, A, k, B, n, impl="mp").reshape(m, n, -1)
    C = C.reshape(m, n, -1)
    for i in range(m):
        for j in range(n):
            want = plain if (i in (3, 11) or j == 9) else exact
            assert orc.mismatches(prec, C[i, j:j + 1], want[i, j:j + 1])[0] == 0, (i, j)


def test_exact_real_pb512_full_size(orc, mpb):
    """The 1024^3 PB=512 workload: entries with 16 random limbs and exponents
    in [-16, 16]; a row sample must equal mpfr_dot and be <= 0.5 ULP from the
    exact sum at 2048 bits."""
    import torch

    prec, m, n, k = 512, 1024, 1024, 1024
    (al, ah), (bl, bh) = synth.gemm_r512()
    dA = to_dev(layout.vec_from_parts(prec, al, ah))
    dB = to_dev(layout.vec_from_parts(prec, bl, bh))
    Cd = mpb.empty(prec, m * n)
    st = torch.zeros(2, dtype=torch.int32, device="cuda")
    mpb.gemm_exact(prec, m, n, k, dA, k, dB, n, Cd, n, sp_bits=32, status=st)
    st = st.cpu().numpy()
    assert st[1] == 0 and st[0] == 0
    got = layout.vec_to_aos(prec, to_host(Cd), m * n)
    A, B = layout.aos_from_parts(prec, al, ah), layout.aos_from_parts(prec, bl, bh)
    for r0, r1 in ((0, 2), (517, 518), (m - 1, m)):
        exp = orc.gemm_exact(prec, m, n, k, A, k, B, n, impl="mp", rows=(r0, r1))
        sel = slice(r0 * n, r1 * n)
        assert orc.mismatches(prec, got[sel], exp[sel])[0] == 0
        e4 = orc.gemm_exact(prec, m, n, k, A, k, B, n, out_prec=4 * prec, rows=(r0, r1))
        ulp = orc.ulp_errors(prec, got[sel], 4 * prec, e4[r0 * n * 1:r1 * n])
        assert ulp.max() <= 0.5


def rand_caos(prec, count, seed, elo=-8, ehi=8, zero_frac=0.05):
    rng = np.random.default_rng(seed)
    re = synth.random_elems(rng, prec, count, elo, ehi, zero_frac)
    im = synth.random_elems(rng, prec, count, elo, ehi, zero_frac)
    return synth.interleave_complex(prec, re, im)


def pad_rows_c(prec, A, rows, cols, ld):
    z1 = layout.aos_from_parts(prec, np.zeros((1, prec // 32), np.uint32), np.array([layout.HEAD_ZERO], np.uint32))
    z = np.concatenate([z1, z1], axis=1)
    es = A.shape[1]
    out = np.repeat(z, rows * ld, axis=0).reshape(rows, ld, es)
    out[:, :cols] = A.reshape(rows, cols, es)
    return out.reshape(rows * ld, es)


def run_exact_c(mpb, prec, m, n, k, A, B, sp_bits):
    import torch

    lda, ldb, ldc = (-(-k // 32) * 32, -(-n // 32) * 32, -(-n // 32) * 32)
    dA = to_dev(layout.aos_to_vec(prec, pad_rows_c(prec, A, m, k, lda), True))
    dB = to_dev(layout.aos_to_vec(prec, pad_rows_c(prec, B, k, n, ldb), True))
    Cd = mpb.empty(prec, m * ldc, True)
    st = torch.zeros(2, dtype=torch.int32, device="cuda")
    mpb.gemm_exact(prec, m, n, k, dA, lda, dB, ldb, Cd, ldc, sp_bits=sp_bits, status=st, cplx=True)
    C = layout.vec_to_aos(prec, to_host(Cd), m * ldc, True).reshape(m, ldc, -1)[:, :n].reshape(m * n, -1)
    return C, st.cpu().numpy()


@pytest.mark.parametrize("prec", (64, 256, 512, 1024))
@pytest.mark.parametrize("shape", ((1, 1, 1), (5, 7, 33), (33, 40, 17), (130, 260, 300)))
def test_exact_complex_vs_mpc_dot(orc, mpb, prec, shape):
    """Each component is one rounding of the exact complex dot (mpc_dot),
    computed with three exact integer products (Gauss form)."""
    m, n, k = shape
    if prec == 1024 and m * n * k > 200000:
        pytest.skip("covered at smaller shapes")
    A = rand_caos(prec, m * k, 300 + m + prec)
    B = rand_caos(prec, k * n, 400 + n + prec)
    C, st = run_exact_c(mpb, prec, m, n, k, A, B, sp_bits=16)
    assert st[1] == 0 and st[0] == 0
    exp = orc.gemm_exact(prec, m, n, k, A, k, B, n, cplx=True, impl="mp")
    bad, first = orc.mismatches(prec, C, exp, True)
    assert bad == 0, f"PB={prec} {shape}: {bad} mismatches, first at {first}"


@pytest.mark.parametrize("cplx", (False, True))
@pytest.mark.parametrize("sp_bits", (16, 32, 100))
@pytest.mark.parametrize("prec", (64, 128, 256, 512, 1024, 2048))
def test_exact_every_slice_geometry(orc, mpb, prec, sp_bits, cplx):
    """Every (precision, spread budget) instantiation of the slicing and
    rounding kernels -- the budget picks 1, 2 or 4 extra words for the aligned
    integers -- against mpfr_dot / mpc_dot, on a shape with a ragged last tile."""
    if cplx and prec == 2048:
        pytest.skip("complex PB=2048 is covered by the plain kernels")
    m, n, k = 9, 37, 45
    if cplx:
        A, B = rand_caos(prec, m * k, 61 + sp_bits, -6, 6, 0.02), rand_caos(prec, k * n, 62 + sp_bits, -6, 6, 0.02)
        C, st = run_exact_c(mpb, prec, m, n, k, A, B, sp_bits=sp_bits)
    else:
        A, B = rand_aos(prec, m * k, 61 + sp_bits, -6, 6, 0.02), rand_aos(prec, k * n, 62 + sp_bits, -6, 6, 0.02)
        C, st = run_exact(mpb, prec, m, n, k, A, B, sp_bits=sp_bits)
    assert st[1] == 0 and st[0] == 0
    exp = orc.gemm_exact(prec, m, n, k, A, k, B, n, cplx=cplx, impl="mp")
    bad, first = orc.mismatches(prec, C, exp, cplx)
    assert bad == 0, f"PB={prec} sp={sp_bits} cplx={cplx}: {bad} mismatches, first at {first}"


def test_exact_complex_fallback(orc, mpb):
    prec, m, n, k = 256, 12, 40, 30
    A = rand_caos(prec, m * k, 41, -4, 4, 0.0).reshape(m, k, -1)
    B = rand_caos(prec, k * n, 42, -4, 4, 0.0)
    es = layout.aos_bytes(prec)
    A[4, 2, es + 8:es + 16] = np.array([-500], np.int64).view(np.uint8)  # imaginary part far below
    A = A.reshape(m * k, -1)
    C, st = run_exact_c(mpb, prec, m, n, k, A, B, sp_bits=32)
    assert st[1] == 0 and st[0] == 1
    exact = orc.gemm_exact(prec, m, n, k, A, k, B, n, cplx=True, impl="mp").reshape(m, n, -1)
    plain = orc.gemm(prec, m, n, k, A, k, B, n, cplx=True, impl="mp").reshape(m, n, -1)
    C = C.reshape(m, n, -1)
    assert orc.mismatches(prec, C[4], plain[4], True)[0] == 0
    for i in (0, 3, 5, 11):
        assert orc.mismatches(prec, C[i], exact[i], True)[0] == 0


@pytest.mark.parametrize("cplx", (False, True))
def test_exact_long_k_split_into_parts(orc, mpb, cplx):
    """k beyond 2^17/S splits every diagonal into k-parts (separate int32
    planes summed in the rounding): results must stay correctly rounded."""
    prec, m, n, k = 512, 9, 33, 2400
    if cplx:
        A, B = rand_caos(prec, m * k, 51), rand_caos(prec, k * n, 52)
        C, st = run_exact_c(mpb, prec, m, n, k, A, B, sp_bits=16)
    else:
        A, B = rand_aos(prec, m * k, 51), rand_aos(prec, k * n, 52)
        C, st = run_exact(mpb, prec, m, n, k, A, B, sp_bits=16)
    assert st[1] == 0 and st[0] == 0
    exp = orc.gemm_exact(prec, m, n, k, A, k, B, n, cplx=cplx, impl="mp")
    assert orc.mismatches(prec, C, exp, cplx)[0] == 0


def test_exact_complex_pb256_full_size(orc, mpb):
    """The 512^3 complex PB=256 workload: 8-limb entries, exponents in [-8, 8];
    a row sample must equal mpc_dot and be <= 0.5 ULP per component from the
    exact sum at 1024 bits."""
    import torch

    prec, m, n, k = 256, 512, 512, 512
    (ar, ai), (br, bi) = synth.gemm_c256()
    A, B = synth.interleave_complex(prec, ar, ai), synth.interleave_complex(prec, br, bi)
    dA = to_dev(layout.aos_to_vec(prec, A, True))
    dB = to_dev(layout.aos_to_vec(prec, B, True))
    Cd = mpb.empty(prec, m * n, True)
    st = torch.zeros(2, dtype=torch.int32, device="cuda")
    mpb.gemm_exact(prec, m, n, k, dA, k, dB, n, Cd, n, sp_bits=16, status=st, cplx=True)
    st = st.cpu().numpy()
    assert st[1] == 0 and st[0] == 0
    got = layout.vec_to_aos(prec, to_host(Cd), m * n, True)
    for r0, r1 in ((0, 1), (300, 301), (m - 1, m)):
        sel = slice(r0 * n, r1 * n)
        exp = orc.gemm_exact(prec, m, n, k, A, k, B, n, cplx=True, impl="mp", rows=(r0, r1))
        assert orc.mismatches(prec, got[sel], exp[sel], True)[0] == 0
        e4 = orc.gemm_exact(prec, m, n, k, A, k, B, n, cplx=True, out_prec=4 * prec, rows=(r0, r1))
        es, e4s = layout.aos_bytes(prec), layout.aos_bytes(4 * prec)
        for part in (0, 1):
            g = got[sel][:, part * es:(part + 1) * es]
            w = e4[sel][:, part * e4s:(part + 1) * e4s]
            assert orc.ulp_errors(prec, g, 4 * prec, w).max() <= 0.5


def test_plain_complex_pb256_full_size(orc, mpb):
    """The plain per-operation-rounded complex GEMM on the same 512^3 PB=256
    workload (the kernel the bench times beside the exact one): a row sample
    (first, middle, last rows) must equal MPC's mpc_mul + mpc_add in k order."""
    prec, m, n, k = 256, 512, 512, 512
    (ar, ai), (br, bi) = synth.gemm_c256()
    A, B = synth.interleave_complex(prec, ar, ai), synth.interleave_complex(prec, br, bi)
    dA = to_dev(layout.aos_to_vec(prec, A, True))
    dB = to_dev(layout.aos_to_vec(prec, B, True))
    Cd = mpb.empty(prec, m * n, True)
    mpb.gemm(prec, m, n, k, dA, k, dB, n, Cd, n, cplx=True)
    got = layout.vec_to_aos(prec, to_host(Cd), m * n, True)
    for r0, r1 in ((0, 2), (257, 258), (m - 1, m)):
        sel = slice(r0 * n, r1 * n)
        exp = orc.gemm(prec, m, n, k, A, k, B, n, cplx=True, impl="mp", rows=(r0, r1))
        bad, first = orc.mismatches(prec, got[sel], exp[sel], True)
        assert bad == 0, f"rows {r0}-{r1}: {bad} entries differ from MPC (first {first})"


def test_tensor_kernel_wait_runs_out_and_reports(orc, mpb):
    """The bounded-wait path of the tensor-core kernel: one launch runs with an
    accumulator commit withheld in its first CTA and 50 ms wait limits, so that
    CTA's epilogue wait runs out (nothing else sets the barrier).  The kernel
    must report an error code in status[1] instead of hanging or faulting,
    and the next call on the same stream must be correct again."""
    L = mpb.lib()
    assert L.mpb_gemm_exact_test_inject(2, 50_000_000) == -7  # MPB_ERR_ARG: no such injection
    assert L.mpb_gemm_exact_test_inject(1, 10) == -7  # limit out of range
    prec, m, n, k = 512, 256, 512, 64
    A = rand_aos(prec, m * k, 301)
    B = rand_aos(prec, k * n, 302)
    assert L.mpb_gemm_exact_test_inject(1, 50_000_000) == 0
    _, st = run_exact(mpb, prec, m, n, k, A, B, sp_bits=16)
    assert st[1] in (1, 2, 3, 4), f"status {st}: the withheld commit was not reported"
    C, st = run_exact(mpb, prec, m, n, k, A, B, sp_bits=16)
    assert st.tolist() == [0, 0]
    assert orc.mismatches(prec, C, orc.gemm_exact(prec, m, n, k, A, k, B, n, impl="mp"))[0] == 0


@pytest.mark.parametrize("cplx", (False, True))
def test_exact_gemm_graph_capture_replays_bit_exact(mpb, cplx):
    """The whole exact GEMM call (statistics, slicing, tensor-core passes,
    rounding, fallback; launched with programmatic stream serialisation) is
    captured into a CUDA graph and replayed: every replay must give the direct
    call's result and status, including a row outside the spread budget that
    the fallback computes inside the graph (real case)."""
    import torch

    prec = 256 if cplx else 512
    m, n, k = 70, 96, 96  # n, k multiples of 32: no padding
    if cplx:
        rng = np.random.default_rng(0xCA97)
        A = synth.interleave_complex(prec, synth.random_elems(rng, prec, m * k, -6, 6),
                                     synth.random_elems(rng, prec, m * k, -6, 6))
        B = synth.interleave_complex(prec, synth.random_elems(rng, prec, k * n, -6, 6),
                                     synth.random_elems(rng, prec, k * n, -6, 6))
    else:
        A = rand_aos(prec, m * k, 0xCA98, -6, 6).reshape(m, k, -1)
        A[3, 5] = rand_aos(prec, 1, 0xCA9A, -60, -60, 0.0)[0]  # row 3 spreads 54+ bits: fallback
        A = A.reshape(m * k, -1)
        B = rand_aos(prec, k * n, 0xCA99, -6, 6)
    dA = to_dev(layout.aos_to_vec(prec, A, cplx))
    dB = to_dev(layout.aos_to_vec(prec, B, cplx))
    ws = torch.empty(mpb.gemm_exact_workspace(prec, m, n, k, 16, cplx), dtype=torch.uint8, device="cuda")
    ref, refst = mpb.empty(prec, m * n, cplx), torch.zeros(2, dtype=torch.int32, device="cuda")
    out, outst = mpb.empty(prec, m * n, cplx), torch.zeros(2, dtype=torch.int32, device="cuda")
    s = torch.cuda.Stream()

    def call(C, st):
        mpb.gemm_exact(prec, m, n, k, dA, k, dB, n, C, n, sp_bits=16, workspace=ws, status=st, cplx=cplx, stream=s)

    with torch.cuda.stream(s):
        call(ref, refst)  # direct call (also the per-device set-up, outside the capture)
    torch.cuda.synchronize()
    L = mpb.lib()
    L.mpb_profile_enable(1)  # the phase events become nodes of the graph
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        call(out, outst)
    for _ in range(2):
        out.zero_()
        outst.fill_(-1)
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
        assert outst.tolist() == refst.tolist()
    # the tensor-core phase of the last replay, timed by the captured events
    assert L.mpb_profile_phase_count(2) == 1 and L.mpb_profile_phase_ms(2) > 0.0
    L.mpb_profile_enable(0)
    assert refst[1].item() == 0
    if not cplx:
        assert refst[0].item() >= 1  # the row outside the budget went to the fallback
    del g


@pytest.mark.parametrize("cplx", (False, True))
def test_exact_gemm_empty_dimensions(mpb, cplx):
    """k = 0: every entry is the empty sum +0; m = 0: nothing to do.  Both
    report a clean status (no fallback, no error) into a reused status word."""
    import torch

    prec, m, n, ldc = 256, 5, 40, 64
    rng = np.random.default_rng(0xE0)
    zero_parts = (np.zeros((1, prec // 32), np.uint32), np.array([layout.HEAD_ZERO], np.uint32))
    if cplx:
        C0 = synth.interleave_complex(prec, synth.random_elems(rng, prec, m * ldc, -4, 4),
                                      synth.random_elems(rng, prec, m * ldc, -4, 4))
        zero = synth.interleave_complex(prec, zero_parts, zero_parts)[0]
    else:
        C0 = layout.aos_from_parts(prec, *synth.random_elems(rng, prec, m * ldc, -4, 4))
        zero = layout.aos_from_parts(prec, *zero_parts)[0]
    C = to_dev(layout.aos_to_vec(prec, C0, cplx))
    st = torch.full((2,), -7, dtype=torch.int32, device="cuda")
    mpb.gemm_exact(prec, m, n, 0, None, 32, None, 64, C, ldc, sp_bits=16, status=st, cplx=cplx)
    torch.cuda.synchronize()
    assert st.tolist() == [0, 0]
    got = layout.vec_to_aos(prec, to_host(C), m * ldc, cplx).reshape(m, ldc, -1)[:, :n]
    assert (got == zero).all(), "k = 0 must give +0 in every entry"
    st.fill_(-7)
    mpb.gemm_exact(prec, 0, n, 8, None, 32, None, 64, C, ldc, sp_bits=16, status=st, cplx=cplx)
    torch.cuda.synchronize()
    assert st.tolist() == [0, 0]
