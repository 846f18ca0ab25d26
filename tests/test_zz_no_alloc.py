"""The allocation-free exact GEMM (mpb_gemm_exact_r_static), through the C ABI.

Some callers cannot allocate device memory: a latency-critical loop that must
not call cudaMalloc (nor take its implicit synchronisation) once it is
running, or code inside a framework that owns the whole device memory pool.
For them the exact GEMM has an entry point that takes no workspace and
allocates nothing: its scratch is a fixed 16 MiB area inside the library.

This test calls that entry point twice in a row on different problems (and
once more on the first problem, after the second has overwritten the shared
scratch), and checks every result bit for bit -- the exact GEMM is integer
arithmetic, the same tolerance as every other test here -- against the
entry point that takes a caller-provided workspace.  It also checks that a
problem needing more than the fixed area is refused with MPB_ERR_SIZE, that
once each kernel has been loaded a run of static calls leaves the device's
free memory unchanged (nothing is allocated), and that a first call whose
scratch-address lookup is refused -- made while a stream capture is in
progress -- does not stick: the next ordinary call succeeds.
This file is collected last so a failure here never hides other results.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from mpc_cuda_b200 import layout, synth

pytestmark = pytest.mark.gpu

MPB_ERR_SIZE = -2


def _problem(prec, m, n, k, seed):
    import torch

    rng = np.random.default_rng(seed)
    lda, ldb, ldc = -(-k // 32) * 32, -(-n // 32) * 32, -(-n // 32) * 32

    def mat(rows, cols, ld):
        limbs, heads = synth.random_elems(rng, prec, rows * cols, -12, 12, 0.03)
        L = np.zeros((rows, ld, prec // 32), np.uint32)
        H = np.full((rows, ld), layout.HEAD_ZERO, np.uint32)
        L[:, :cols] = limbs.reshape(rows, cols, -1)
        H[:, :cols] = heads.reshape(rows, cols)
        v = layout.vec_from_parts(prec, L.reshape(rows * ld, -1), H.reshape(-1))
        return torch.from_numpy(v.copy()).cuda()

    return dict(prec=prec, m=m, n=n, k=k, lda=lda, ldb=ldb, ldc=ldc, A=mat(m, k, lda), B=mat(k, n, ldb))


def _run(mpb, pr, static, sp_bits):
    import torch

    L = mpb.lib()
    C = torch.zeros(layout.vec_bytes(pr["prec"], pr["m"] * pr["ldc"]), dtype=torch.uint8, device="cuda")
    st = torch.zeros(2, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    args = (pr["prec"], pr["m"], pr["n"], pr["k"], pr["A"].data_ptr(), pr["lda"], pr["B"].data_ptr(), pr["ldb"],
            C.data_ptr(), pr["ldc"], sp_bits)
    if static:
        rc = L.mpb_gemm_exact_r_static(*args, st.data_ptr(), stream)
    else:
        nbytes = L.mpb_gemm_exact_workspace(pr["prec"], pr["m"], pr["n"], pr["k"], sp_bits)
        ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        rc = L.mpb_gemm_exact_r(*args, ws.data_ptr(), nbytes, st.data_ptr(), stream)
    assert rc == 0, mpb.status_string(rc)
    torch.cuda.synchronize()
    return C.cpu().numpy(), st.cpu().numpy()


def test_static_scratch_matches_workspace_entry_point(mpb):
    p1 = _problem(512, 70, 90, 100, 11)
    p2 = _problem(256, 40, 33, 64, 12)
    for pr, sp in ((p1, 32), (p2, 16), (p1, 32)):
        got, st_got = _run(mpb, pr, True, sp)
        want, st_want = _run(mpb, pr, False, sp)
        assert st_got.tolist() == st_want.tolist() and st_got[1] == 0
        assert np.array_equal(got, want), f"PB={pr['prec']}: static-scratch result differs"


def test_static_scratch_rejects_oversized_problem(mpb):
    L = mpb.lib()
    # 1024^3 at PB=512 needs ~730 MB of scratch, far beyond the fixed 16 MiB
    assert L.mpb_gemm_exact_workspace(512, 1024, 1024, 1024, 32) > 16 << 20
    rc = L.mpb_gemm_exact_r_static(512, 1024, 1024, 1024, 4096, 1024, 4096, 1024, 4096, 1024, 32, None, None)
    assert rc == MPB_ERR_SIZE


def test_static_calls_allocate_nothing(mpb):
    """After one call per shape (which loads each kernel the first time), more
    static calls at those shapes leave the device's free byte count as it was."""
    import torch

    L = mpb.lib()
    probs = [(_problem(512, 70, 90, 100, 21), 32), (_problem(256, 40, 33, 64, 22), 16),
             (_problem(128, 130, 64, 200, 23), 24)]
    outs = []
    for pr, _ in probs:  # every buffer the calls use exists before the count is taken
        outs.append((torch.zeros(layout.vec_bytes(pr["prec"], pr["m"] * pr["ldc"]), dtype=torch.uint8,
                                 device="cuda"), torch.zeros(2, dtype=torch.int32, device="cuda")))
    stream = torch.cuda.current_stream().cuda_stream

    def call(i):
        pr, sp = probs[i]
        C, st = outs[i]
        rc = L.mpb_gemm_exact_r_static(pr["prec"], pr["m"], pr["n"], pr["k"], pr["A"].data_ptr(), pr["lda"],
                                       pr["B"].data_ptr(), pr["ldb"], C.data_ptr(), pr["ldc"], sp, st.data_ptr(),
                                       stream)
        assert rc == 0, mpb.status_string(rc)

    for i in range(len(probs)):
        call(i)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        for i in range(len(probs)):
            call(i)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"static calls changed the device's free memory by {free0 - free1} bytes"
    for i, (pr, sp) in enumerate(probs):
        want, _ = _run(mpb, pr, False, sp)
        assert np.array_equal(outs[i][0].cpu().numpy(), want)


_FIRST_CALL_IN_CAPTURE = r"""
import sys
sys.path.insert(0, sys.argv[1])
import numpy as np
import torch
import mpc_cuda_b200 as M
from tests.test_zz_no_alloc import _problem, _run
torch.cuda.init()
pr = _problem(512, 70, 90, 100, 31)
L = M.lib()
s = torch.cuda.Stream()
C = torch.zeros(1 << 20, dtype=torch.uint8, device="cuda")
st = torch.zeros(2, dtype=torch.int32, device="cuda")
torch.cuda.synchronize()
g = torch.cuda.CUDAGraph()
rc_first = None
try:
    with torch.cuda.graph(g, stream=s):
        rc_first = L.mpb_gemm_exact_r_static(512, 70, 90, 100, pr["A"].data_ptr(), pr["lda"], pr["B"].data_ptr(),
                                             pr["ldb"], C.data_ptr(), pr["ldc"], 32, st.data_ptr(), s.cuda_stream)
except Exception as e:
    print("capture ended with:", type(e).__name__)
del g
torch.cuda.synchronize()
print("first call during capture returned", rc_first)
got, st_got = _run(M, pr, True, 32)
want, st_want = _run(M, pr, False, 32)
assert st_got.tolist() == st_want.tolist() and st_got[1] == 0
assert np.array_equal(got, want)
print("SECOND_CALL_OK")
"""


def test_first_call_during_capture_does_not_stick():
    """In a fresh process, the very first static call is made inside a stream
    capture (where the runtime may refuse the scratch-address lookup); the
    ordinary call after the capture must succeed and match the workspace entry
    point.  A fresh process is needed because the address, once found, is kept
    for the life of the process."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _FIRST_CALL_IN_CAPTURE, root], cwd=root, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0 and "SECOND_CALL_OK" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
