#!/usr/bin/env python3
"""bench.py -- throughput of the mpb engine on its benchmark workloads.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mpb|reference]
                    [--workload gemm_r512|gemm_c256|gemv_batch|axpy_c1024|axpy_r256|
                                div_r512|sqrt_r512|exp_r512|log_r512|sin_r512|cexp_c512]

One JSON line on stdout (rank 0).  A step is one pass of the hot path over
one batch of synthetic operands already resident in HBM; K steps are timed
with CUDA events on the launching stream between a barrier and a device
synchronize, the time is the max over ranks, and ``value`` is the units all
ranks processed divided by that time.  With N > 1 (torchrun, one process per
GPU) every rank runs its own independent shard of the same size (weak
scaling, no data-path collective: the problems are independent).

``e2e`` is the same metric measured through the C ABI starting from HOST
buffers of mpc_cuda AoS structs (pinned): per step the inputs are copied in,
packed into the engine layout, computed, unpacked and copied back.

``--impl reference`` times the reference's own implementation of the path on
the host cores (its cu_freal/cu_fcomplex headers compiled for the CPU with
OpenMP, oracle/_ref; the oracle's C restatement when that build is absent)
on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "mp-FMA/s at PB=256/1024: tensor-core exact GEMM vs plain kernel, ≤0.5 ULP"
L2_BYTES = 126 * 1024 * 1024


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


# ------------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during timing."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r for r in csv.reader(io.StringIO(self.f.read())) if len(r) >= 9]
        self.f.close()
        os.unlink(self.f.name)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


class NvmlClocks:
    """The same SM clock and clock-event reasons nvidia-smi reports, read
    through NVML by a thread every ~2 ms while the timed regions run (a timed
    region of 20 GEMM steps lasts ~40 ms, shorter than nvidia-smi's start-up
    and sampling period).  Read-only: no setting of the GPU is touched."""

    BITS = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
            "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
            "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
            "sw_power_cap": "nvmlClocksEventReasonSwPowerCap"}

    def __init__(self, cuda_index: int):
        import pynvml
        import torch

        self.nv = pynvml
        pynvml.nvmlInit()
        uuid = str(torch.cuda.get_device_properties(cuda_index).uuid)
        try:
            self.h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            self.h = pynvml.nvmlDeviceGetHandleByIndex(cuda_index)
        self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        self.samples, self.stop_flag, self.thread = [], False, None

    def _run(self):
        nv = self.nv
        while not self.stop_flag:
            try:
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)),
                                     int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))))
            except Exception:
                pass
            time.sleep(0.002)

    def start(self):
        import threading

        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def stop(self):
        self.stop_flag = True
        self.thread.join(timeout=5)
        reasons = set()
        for _, bits in self.samples:
            for nm, const in self.BITS.items():
                if bits & getattr(self.nv, const):
                    reasons.add(nm)
        sm = [mhz for mhz, _ in self.samples]
        try:
            self.nv.nvmlShutdown()
        except Exception:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(sm), "source": "NVML, every ~2 ms"}


def make_clocks(cuda_index: int):
    """NVML sampling when the bindings are importable, else nvidia-smi."""
    try:
        return NvmlClocks(cuda_index)
    except Exception:
        return Clocks(cuda_index)


# ------------------------------------------------------------------ helpers
def pinned_from(np_arr):
    import torch

    t = torch.from_numpy(np_arr.reshape(-1).copy())
    return t.pin_memory()


def dev_from(np_arr, device):
    import torch

    a = np_arr.reshape(-1)
    return torch.from_numpy(a.copy()).to(device)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "MEASURED_PEAKS.json"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def imad_peak(stream_ptr):
    """IMAD lane-ops/s of this GPU (libmpb_probe.so), or None."""
    import ctypes

    path = os.path.join(ROOT, "mpc_cuda_b200", "libmpb_probe.so")
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    L.mpb_probe_imad_ops_per_s.argtypes = [ctypes.c_void_p]
    L.mpb_probe_imad_ops_per_s.restype = ctypes.c_double
    v = L.mpb_probe_imad_ops_per_s(stream_ptr)
    return v if v > 0 else None


def rounded_product_imads(N):
    """32-bit multiply-adds (lo + hi per limb pair) of one N-limb product as the
    engine computes it for a rounded product or a certified fmms: from N = 4
    up only the columns N-2 .. 2N-2 of the limb product (the rare exact case
    aside)."""
    if N < 4:
        return 2 * N * N
    return 2 * ((N - 1) + N + N * (N - 1) // 2)


# ------------------------------------------------------------------ workloads
class AxpyWorkload:
    """z = a*x + y over n elements (real or complex), rotating input sets so
    consecutive steps never hit L2 (footprint > 126 MB)."""

    def __init__(self, name, cplx, prec, n, seed):
        self.name, self.cplx, self.prec, self.n, self.seed = name, cplx, prec, n, seed
        comp = 2 if cplx else 1
        self.elem_bytes = comp * 4 * (prec // 32 + 1)  # tiled layout, limbs + head
        # one complex mp-FMA = one complex multiply (4 exact products) + add
        self.products = 4 if cplx else 1
        self.nsets = max(2, -(-2 * L2_BYTES // (3 * n * self.elem_bytes)))
        self.desc = (f"{'complex' if cplx else 'real'} AXPY z=a*x+y, "
                     f"{'cu_fcomplex' if cplx else 'cu_freal'}<{prec}>, "
                     f"{'MPC_RNDNN' if cplx else 'RNDN'} per operation, n=2^{n.bit_length() - 1}")

    def make_host(self, rank):
        from mpc_cuda_b200 import layout, synth

        if self.cplx:
            a, x, y = synth.axpy_c1024(seed=shard_seed(self.seed, rank), n=self.n, prec=self.prec)
            conv = lambda p: synth.interleave_complex(self.prec, *p)  # noqa: E731
        else:
            a, x, y = synth.axpy_r256(seed=shard_seed(self.seed, rank), n=self.n, prec=self.prec)
            conv = lambda p: layout.aos_from_parts(self.prec, *p)  # noqa: E731
        return conv(a), conv(x), conv(y)

    def setup(self, rank, device):
        import mpc_cuda_b200 as M
        from mpc_cuda_b200 import layout

        self.M = M
        A, X, Y = self.make_host(rank)
        self.host = (A, X, Y)
        vec = lambda aos: dev_from(layout.aos_to_vec(self.prec, aos, self.cplx), device)  # noqa: E731
        self.a = vec(A)
        self.sets = []
        for s in range(self.nsets):
            xs = vec(X) if s == 0 else self.sets[0][0].clone()
            ys = vec(Y) if s == 0 else self.sets[0][1].clone()
            self.sets.append((xs, ys, M.empty(self.prec, self.n, self.cplx, device=device)))
        # e2e: pinned host AoS buffers and device staging
        import torch

        self.hx, self.hy = pinned_from(X), pinned_from(Y)
        self.hz = [torch.empty(X.size, dtype=torch.uint8).pin_memory() for _ in range(2)]
        dev2 = lambda nb: [torch.empty(nb, dtype=torch.uint8, device=device) for _ in range(2)]  # noqa: E731
        self.dx_aos, self.dy_aos, self.dz_aos = dev2(X.size), dev2(Y.size), dev2(X.size)
        self.ex, self.ey, self.ez = (M.empty(self.prec, self.n, self.cplx, device=device) for _ in range(3))

    def units(self):
        return self.n

    @property
    def default_steps(self):
        return 4000 if self.cplx else 40000

    def step(self, i, stream):
        x, y, z = self.sets[i % self.nsets]
        self.M.axpy(self.prec, self.n, self.a, x, y, z, self.cplx, stream=stream)

    launches_per_step = 1

    def e2e_h2d(self, s):
        self.dx_aos[s].copy_(self.hx, non_blocking=True)
        self.dy_aos[s].copy_(self.hy, non_blocking=True)

    def e2e_compute(self, s, stream):
        M = self.M
        M.pack_aos(self.prec, self.n, self.dx_aos[s], self.ex, self.cplx, stream=stream)
        M.pack_aos(self.prec, self.n, self.dy_aos[s], self.ey, self.cplx, stream=stream)
        M.axpy(self.prec, self.n, self.a, self.ex, self.ey, self.ez, self.cplx, stream=stream)
        M.unpack_aos(self.prec, self.n, self.ez, self.dz_aos[s], self.cplx, stream=stream)

    def e2e_d2h(self, s):
        self.hz[s].copy_(self.dz_aos[s], non_blocking=True)

    e2e_launches_per_step = 4

    def e2e_bytes(self):
        return 2 * self.host[1].size, self.host[1].size

    def roofline(self, kernel_s, peaks, imad_ops_s):
        N = self.prec // 32
        # complex: 4 upper-column products (two certified fmms); real: one rounded product
        imad_per_unit = (4 if self.cplx else 1) * rounded_product_imads(N)
        bytes_per_unit = 3 * self.elem_bytes
        imad = imad_per_unit * self.n / kernel_s
        gbs = bytes_per_unit * self.n / kernel_s / 1e9
        hbm_peak, hbm_src = peaks
        hbm = {"achieved": round(gbs, 1), "peak": hbm_peak["hbm_gbs"], "unit": "GB/s",
               "frac": round(gbs / hbm_peak["hbm_gbs"], 4), "bytes_per_unit": bytes_per_unit,
               "peak_source": hbm_src}
        if self.prec <= 256 and not self.cplx or imad_ops_s is None:
            out = {"bound": "hbm", **hbm, "traffic": None}
            out["imad"] = None if imad_ops_s is None else {
                "achieved": round(imad / 1e9, 1), "peak": round(imad_ops_s / 1e9, 1), "unit": "Gop/s",
                "frac": round(imad / imad_ops_s, 4), "ops_per_unit": imad_per_unit}
            return out
        return {"bound": "imad", "achieved": round(imad / 1e9, 1), "peak": round(imad_ops_s / 1e9, 1),
                "unit": "Gop/s", "frac": round(imad / imad_ops_s, 4), "ops_per_unit": imad_per_unit,
                "peak_source": "libmpb_probe.so mad.lo/mad.hi throughput, measured in this run",
                "traffic": None, "hbm": hbm}

    def cpu_run(self, impl, count):
        """AXPY over the first count elements; returns the units computed."""
        import oracle as O

        A, X, Y = self.host
        O.axpy(self.prec, A, X[:count], Y[:count], self.cplx, impl=impl)
        return count

    cpu_probe_units = 2048

    def config(self):
        return {"workload": self.desc, "prec": self.prec, "n": self.n,
                "units": "complex mp-FMA (one complex multiply + one complex add)" if self.cplx
                else "mp-FMA (one multiply + one add, each rounded)",
                "layout": "tiled SoL, 32-element tiles, 128-bit limb groups + 32-bit head",
                "l2": f"{self.nsets} rotating input sets, {self.nsets * 3 * self.n * self.elem_bytes >> 20} MiB > L2"}


def int8_peak_ops(device):
    """Dense int8 tensor-core throughput of this GPU: cuBLASLt int8 GEMM
    (torch._int_mm, 8192^3, int32 out), best of 5, ops = 2*M*N*K."""
    import torch

    try:
        M = 8192
        a = torch.randint(-128, 127, (M, M), dtype=torch.int8, device=device)
        b = torch.randint(-128, 127, (M, M), dtype=torch.int8, device=device).t()
        torch._int_mm(a, b)
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        del a, b
        return 2.0 * M**3 / (best / 1e3)
    except Exception:
        return None


class GemmWorkload:
    """C = A.B, m x n x k at precision prec: the exact-accumulation INT8
    tensor-core GEMM (one rounding per entry) is the timed step; the plain
    per-operation-rounded kernel on the same operands is timed beside it."""

    def __init__(self, name, prec, m, n, k, sp_bits, gen, cplx=False):
        self.name, self.prec, self.m, self.n, self.k, self.sp_bits, self.gen = name, prec, m, n, k, sp_bits, gen
        self.cplx = cplx
        self.nprod = 3 if cplx else 1  # complex: 3 exact real products (Gauss form)
        self.S = (prec + sp_bits + (3 if cplx else 2) + 7) // 8
        kind = f"complex matmul, cu_fcomplex<{prec}>" if cplx else f"real matmul, cu_freal<{prec}>"
        form = ", 3-product Gauss form, one rounding per component" if cplx else ", one rounding per entry"
        self.desc = (f"{kind} C=A.B, {m}x{n}x{k}: exact-accumulation GEMM on INT8 tensor cores "
                     f"({self.S} digit slices{form}) vs plain sequential-k kernel")

    @property
    def default_steps(self):
        return 2000 if self.cplx else 200  # ~1 s of GPU time: long enough for clock sampling

    @property
    def launches_per_step(self):
        # stats x2, slice x2, tensor-core GEMM, round, fallback; with truncated
        # diagonals also the (usually empty) low-diagonal GEMM and second round
        return 7 + (2 if getattr(self, "d0", 0) > 0 else 0)

    @property
    def e2e_launches_per_step(self):
        return self.launches_per_step + 3  # + pack A, pack B, unpack C

    def make_host(self, rank):
        from mpc_cuda_b200 import layout

        from mpc_cuda_b200 import synth

        a, b = self.gen(seed=shard_seed(0x5EED5 if self.cplx else 0x5EED3, rank))
        if self.cplx:
            return synth.interleave_complex(self.prec, *a), synth.interleave_complex(self.prec, *b)
        return layout.aos_from_parts(self.prec, *a), layout.aos_from_parts(self.prec, *b)

    def setup(self, rank, device):
        import torch

        import mpc_cuda_b200 as M
        from mpc_cuda_b200 import layout

        self.M = M
        A, B = self.make_host(rank)
        self.host = (A, B)
        c = self.cplx
        self.dA = dev_from(layout.aos_to_vec(self.prec, A, c), device)
        self.dB = dev_from(layout.aos_to_vec(self.prec, B, c), device)
        self.dC = M.empty(self.prec, self.m * self.n, c, device=device)
        self.dC2 = M.empty(self.prec, self.m * self.n, c, device=device)
        self.ws = torch.empty(M.gemm_exact_workspace(self.prec, self.m, self.n, self.k, self.sp_bits, c),
                              dtype=torch.uint8, device=device)
        S, self.d0, self.pairs = M.gemm_exact_info(self.prec, self.m, self.n, self.k, self.sp_bits, c)
        assert S == self.S, (S, self.S)
        self.status = torch.zeros(2, dtype=torch.int32, device=device)
        self.hA, self.hB = pinned_from(A), pinned_from(B)
        cbytes = self.m * self.n * A.shape[1]
        self.hC = [torch.empty(cbytes, dtype=torch.uint8).pin_memory() for _ in range(2)]
        dev2 = lambda nb: [torch.empty(nb, dtype=torch.uint8, device=device) for _ in range(2)]  # noqa: E731
        self.dA_aos, self.dB_aos, self.dC_aos = dev2(A.size), dev2(B.size), dev2(cbytes)
        self.eA = M.empty(self.prec, self.m * self.k, c, device=device)
        self.eB = M.empty(self.prec, self.k * self.n, c, device=device)

    def units(self):
        return self.m * self.n * self.k

    def step(self, i, stream):
        self.M.gemm_exact(self.prec, self.m, self.n, self.k, self.dA, self.k, self.dB, self.n, self.dC, self.n,
                          sp_bits=self.sp_bits, workspace=self.ws, status=self.status, cplx=self.cplx,
                          stream=stream)

    def e2e_h2d(self, s):
        self.dA_aos[s].copy_(self.hA, non_blocking=True)
        self.dB_aos[s].copy_(self.hB, non_blocking=True)

    def e2e_compute(self, s, stream):
        M = self.M
        c = self.cplx
        M.pack_aos(self.prec, self.m * self.k, self.dA_aos[s], self.eA, c, stream=stream)
        M.pack_aos(self.prec, self.k * self.n, self.dB_aos[s], self.eB, c, stream=stream)
        M.gemm_exact(self.prec, self.m, self.n, self.k, self.eA, self.k, self.eB, self.n, self.dC, self.n,
                     sp_bits=self.sp_bits, workspace=self.ws, status=self.status, cplx=c, stream=stream)
        M.unpack_aos(self.prec, self.m * self.n, self.dC, self.dC_aos[s], c, stream=stream)

    def e2e_d2h(self, s):
        self.hC[s].copy_(self.dC_aos[s], non_blocking=True)

    def e2e_bytes(self):
        return self.host[0].size + self.host[1].size, self.hC[0].numel()

    def extra(self, stream, steps=3):
        """plain kernel rate on the same operands, dominant-kernel time, status"""
        import torch

        from mpc_cuda_b200 import tune

        M = self.M
        c = self.cplx
        # the plain kernel's block shape, tuned for this C on a short k
        tune.autotune_gemm_warps(self.prec, self.m, self.n, min(self.k, 64), c)
        warps = M.get_gemm_warps(self.prec, c)
        M.gemm(self.prec, self.m, self.n, self.k, self.dA, self.k, self.dB, self.n, self.dC2, self.n, c, stream=stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            M.gemm(self.prec, self.m, self.n, self.k, self.dA, self.k, self.dB, self.n, self.dC2, self.n, c,
                   stream=stream)
        e1.record()
        torch.cuda.synchronize()
        plain_ms = e0.elapsed_time(e1) / steps
        st = self.status.cpu().tolist()
        return {"plain_ms_per_step": plain_ms, "plain_value": self.units() / (plain_ms / 1e3), "status": st,
                "plain_warps": warps, "accuracy": self.accuracy()}

    def accuracy(self, rows=(0, None, -1)):
        """Error of the timed exact GEMM's result on a row sample (first, middle
        and last rows of C, every column): ULPs of PB bits against the dot
        product rounded at 4 PB bits (MPFR mpfr_dot / MPC mpc_dot), and whether
        every entry equals the correctly rounded dot product at PB bits."""
        import oracle as O
        from mpc_cuda_b200 import layout

        A, B = self.host
        c, p = self.cplx, self.prec
        got = layout.vec_to_aos(p, self.dC.cpu().numpy(), self.m * self.n, c)
        es, e4s = layout.aos_bytes(p), layout.aos_bytes(4 * p)
        ulps, equal, picked = [], True, []
        for r in rows:
            r = self.m // 2 if r is None else (r % self.m)
            picked.append(r)
            sel = slice(r * self.n, (r + 1) * self.n)
            want = O.gemm_exact(p, self.m, self.n, self.k, A, self.k, B, self.n, cplx=c, impl="mp", rows=(r, r + 1))
            equal = equal and O.mismatches(p, got[sel], want[sel], c)[0] == 0
            w4 = O.gemm_exact(p, self.m, self.n, self.k, A, self.k, B, self.n, cplx=c, out_prec=4 * p,
                              rows=(r, r + 1))
            for part in ((0, 1) if c else (0,)):
                ulps.append(O.ulp_errors(p, got[sel][:, part * es:(part + 1) * es], 4 * p,
                                         w4[sel][:, part * e4s:(part + 1) * e4s]))
        u = np.concatenate(ulps)
        return {"rows": picked, "entries": int(u.size), "ulp_max": float(u.max()), "ulp_mean": float(u.mean()),
                "reference": f"{'mpc_dot' if c else 'mpfr_dot'} at {4 * p} bits"
                             + (", per component" if c else ""),
                "equal_to_correctly_rounded_dot": bool(equal)}

    def roofline_tensor(self, tensor_ms, int8_ops):
        ops = 2.0 * self.nprod * self.units() * self.pairs
        achieved = ops / (tensor_ms / 1e3)
        return {"bound": "tensor", "achieved": round(achieved / 1e12, 1), "unit": "TOP/s (int8)",
                "peak": round(int8_ops / 1e12, 1) if int8_ops else None,
                "frac": round(achieved / int8_ops, 4) if int8_ops else None,
                "ops_per_unit": 2 * self.nprod * self.pairs, "kernel": "k_diag_gemm (tcgen05.mma kind::i8)",
                "kernel_ms": round(tensor_ms, 4),
                "peak_source": "cuBLASLt int8 GEMM 8192^3 (torch._int_mm), measured in this run",
                "traffic": None}

    def cpu_run(self, impl, count):
        """The first rows of C on the CPU (sequential-k, per-operation
        rounding: the reference's matmul); returns the units computed."""
        import oracle as O

        A, B = self.host
        rows = max(1, min(self.m, count // (self.n * self.k)))
        O.gemm(self.prec, self.m, self.n, self.k, A, self.k, B, self.n, self.cplx, impl=impl, rows=(0, rows))
        return rows * self.n * self.k

    @property
    def cpu_probe_units(self):
        return self.n * self.k  # one row of C

    def config(self):
        return {"workload": self.desc, "prec": self.prec, "m": self.m, "n": self.n, "k": self.k,
                "sp_bits": self.sp_bits, "slices": self.S, "first_diagonal": getattr(self, "d0", None),
                "slice_pairs": getattr(self, "pairs", None),
                "units": ("complex mp-FMA (one complex product accumulated)" if self.cplx
                          else "mp-FMA (one exact product accumulated)"),
                "l2": "operands > L2 (143 MB real / 71 MB complex); digit and diagonal planes stream through HBM"}


class GemvBatchWorkload:
    """4096 independent GEMV problems y_out = A.x + y of uneven sizes and mixed
    precisions, planned once, autotuned, and run as one captured CUDA graph
    (one persistent kernel per precision, largest first) per step.  Operands
    live in one pool per precision and operand (7.9 GB of tiles > L2)."""

    def __init__(self, name, count, seed):
        self.name, self.count, self.seed = name, count, seed
        self.desc = (f"batched GEMV y=A.x+y, {count} independent problems, m,n log-uniform in [16,512], "
                     "PB uniform in {64,128,256,512,1024,2048}, exponents in [-24,24]; one CUDA graph "
                     "(persistent kernel per PB, autotuned launch shape) per step")

    default_steps = 20

    def make_host(self, rank):
        from mpc_cuda_b200 import layout, synth

        probs, pools = synth.gemv_batch(seed=shard_seed(self.seed, rank), count=self.count)
        aos = {p: tuple(layout.aos_from_parts(p, *P[k]) for k in ("A", "x", "y")) for p, P in pools.items()}
        return probs, aos

    def setup(self, rank, device):
        import torch

        import mpc_cuda_b200 as M
        from mpc_cuda_b200 import layout

        self.M = M
        self.probs, self.aos = self.make_host(rank)
        self.host = (self.probs, self.aos)
        self.dev, self.pin, self.stage = {}, {}, {}
        for p, (A, x, y) in self.aos.items():
            d = {k: dev_from(layout.aos_to_vec(p, a), device) for k, a in zip(("A", "x", "y"), (A, x, y))}
            d["yo"] = torch.zeros_like(d["y"])
            self.dev[p] = d
            if not getattr(self, "with_e2e", True):
                continue
            self.pin[p] = {"A": pinned_from(A), "x": pinned_from(x), "y": pinned_from(y),
                           "yo": [torch.empty(y.size, dtype=torch.uint8).pin_memory() for _ in range(2)]}
            self.stage[p] = {k: [torch.empty(a.size, dtype=torch.uint8, device=device) for _ in range(2)]
                             for k, a in (("A", A), ("x", x), ("y", y), ("yo", y))}
        tup = []
        for pr in self.probs:
            d, p = self.dev[pr["prec"]], pr["prec"]
            tup.append((p, pr["m"], pr["n"], pr["lda"], d["A"].data_ptr() + layout.vec_bytes(p, pr["a_off"]),
                        d["x"].data_ptr() + layout.vec_bytes(p, pr["x_off"]),
                        d["y"].data_ptr() + layout.vec_bytes(p, pr["y_off"]),
                        d["yo"].data_ptr() + layout.vec_bytes(p, pr["y_off"])))
        self.batch = M.BatchGemv(tup)
        self.batch.autotune()
        side = torch.cuda.Stream(device)
        self.batch.run(stream=side.cuda_stream)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=side):
            self.batch.run(stream=side.cuda_stream)
        torch.cuda.synchronize()

    def units(self):
        return sum(p["m"] * p["n"] for p in self.probs)

    def step(self, i, stream):
        self.graph.replay()

    @property
    def launches_per_step(self):
        return len(self.aos)  # one persistent kernel per precision present

    @property
    def e2e_launches_per_step(self):
        return 5 * len(self.aos)  # + pack A, x, y and unpack y_out per precision

    def e2e_h2d(self, s):
        for p in self.dev:
            for k in ("A", "x", "y"):
                self.stage[p][k][s].copy_(self.pin[p][k], non_blocking=True)

    def e2e_compute(self, s, stream):
        M = self.M
        for p, d in self.dev.items():
            for k in ("A", "x", "y"):
                M.pack_aos(p, self.aos[p][("A", "x", "y").index(k)].shape[0], self.stage[p][k][s], d[k], stream=stream)
        self.graph.replay()
        for p, d in self.dev.items():
            M.unpack_aos(p, self.aos[p][2].shape[0], d["yo"], self.stage[p]["yo"][s], stream=stream)

    def e2e_d2h(self, s):
        for p in self.dev:
            self.pin[p]["yo"][s].copy_(self.stage[p]["yo"][s], non_blocking=True)

    def e2e_bytes(self):
        h2d = sum(a.size for trip in self.aos.values() for a in trip)
        return h2d, sum(trip[2].size for trip in self.aos.values())

    def work(self):
        """per precision: (mp-FMAs, IMAD ops, algorithmic bytes)"""
        out = {}
        for pr in self.probs:
            p, m, n = pr["prec"], pr["m"], pr["n"]
            N, eb = p // 32, 4 * (p // 32 + 1)
            u, o, b = out.get(p, (0, 0, 0))
            out[p] = (u + m * n, o + rounded_product_imads(N) * m * n, b + (m * n + n + 2 * m) * eb)
        return out

    def roofline(self, kernel_s, peaks, imad_ops_s):
        w = self.work()
        ops = sum(v[1] for v in w.values())
        nbytes = sum(v[2] for v in w.values())
        hbm_peak, hbm_src = peaks
        imad = ops / kernel_s
        gbs = nbytes / kernel_s / 1e9
        tuned = self.batch.tuned_ms()
        return {"bound": "imad", "achieved": round(imad / 1e9, 1),
                "peak": round(imad_ops_s / 1e9, 1) if imad_ops_s else None, "unit": "Gop/s",
                "frac": round(imad / imad_ops_s, 4) if imad_ops_s else None, "ops_per_step": ops,
                "kernel": "k_batch_gemv<N>, one persistent kernel per PB back to back (one graph replay)",
                "peak_source": "libmpb_probe.so mad.lo/mad.hi throughput, measured in this run",
                "traffic": None,
                "hbm": {"achieved": round(gbs, 1), "peak": hbm_peak["hbm_gbs"], "unit": "GB/s",
                        "frac": round(gbs / hbm_peak["hbm_gbs"], 4), "bytes_per_step": nbytes,
                        "peak_source": hbm_src},
                "per_prec": {str(p): {"mp_fma": v[0], "imad_ops": v[1], "bytes": v[2],
                                      "solo_ms": round(tuned.get(p, -1.0), 4),
                                      "tuning": list(self.batch.tuning()[p]),
                                      "lanes_per_row": self.batch.splits()[p]} for p, v in sorted(w.items())}}

    def cpu_run(self, impl, count):
        """Problems in planned order until about count units; returns units done."""
        import oracle as O

        probs, aos = self.host
        done = 0
        for pr in probs:
            if done >= count:
                break
            A, x, y = aos[pr["prec"]]
            p, m, n = pr["prec"], pr["m"], pr["n"]
            O.gemv(p, m, n, A[pr["a_off"]:pr["a_off"] + m * pr["lda"]], pr["lda"],
                   x[pr["x_off"]:pr["x_off"] + n], y[pr["y_off"]:pr["y_off"] + m], impl=impl)
            done += m * n
        return done

    cpu_probe_units = 200000

    def config(self):
        w = self.work()
        return {"workload": self.desc, "problems": self.count, "mp_fma_per_step": self.units(),
                "mp_fma_by_prec": {str(p): v[0] for p, v in sorted(w.items())},
                "units": "mp-FMA (one multiply + one add, each rounded)",
                "l2": "operand pools 7.9 GB of tiles > L2"}


def _elem_params(NW):
    """the series parameters of mpb/elem.cuh at NW limbs (em1_halvings ..
    odd_terms there): expm1 halvings and terms, sin/cos halvings and terms,
    the atanh terms of log after its exponential reduction"""
    import math

    def ilog2(v):
        return v.bit_length() - 1 if v > 1 else 0

    need = 32 * NW + 8
    s_e = math.isqrt(38 * NW)
    T_e, bits = 1, 0
    while bits < need:
        T_e += 1
        bits += s_e + ilog2(T_e)
    s_c = max(4, (9 * math.isqrt(NW) - 5) // 2)
    T_c, bits = 0, 0
    while bits < need:
        T_c += 1
        bits += 2 * s_c + ilog2((2 * T_c) * (2 * T_c + 1))
    T_l = (need + 2 * 48 - 1) // (2 * 48)  # atanh terms after the exp reduction
    return s_e, T_e, s_c, T_c, T_l


class DivSqrtWorkload(AxpyWorkload):
    """z = x / y, sqrt(x) (correctly rounded: mpfr_div / mpfr_sqrt), exp(x),
    log(x) or sin(x) (faithful, the reference's contract) over n elements at
    precision prec; the CPU baseline is the reference's own cu_fdiv / cu_sqrt /
    cu_exp / cu_log / cu_sin built for the host."""

    NAMES = {"div": ("correctly rounded divisions", "mp-div/s", "division z=x/y, RNDN (one rounding)"),
             "sqrt": ("correctly rounded square roots", "mp-sqrt/s", "square root z=sqrt(x), RNDN (one rounding)"),
             "exp": ("faithful exponentials", "mp-exp/s", "exponential z=exp(x), faithful (x in (-8, 8))"),
             "log": ("faithful logarithms", "mp-log/s", "logarithm z=log(x), faithful (x > 0)"),
             "sin": ("faithful sines", "mp-sin/s", "sine z=sin(x), faithful (x in (-32, 32))")}

    def __init__(self, name, op, prec, n, seed):
        super().__init__(name, False, prec, n, seed)
        self.op = op
        what, self.unit, desc = self.NAMES[op]
        self.metric = f"{what}/s at PB={prec}"
        self.desc = (f"real {desc}, cu_freal<{prec}>, n=2^{n.bit_length() - 1}, full random significands")

    @property
    def default_steps(self):  # about 1 s of GPU time: long enough for clock sampling
        return {"div": 8000, "sqrt": 1300, "exp": 200, "log": 100, "sin": 100}[self.op]

    def make_host(self, rank):
        from mpc_cuda_b200 import layout, synth

        rng = np.random.default_rng(shard_seed(self.seed, rank))
        lo, hi = {"div": (-40, 40), "sqrt": (-40, 40), "exp": (-3, 3), "log": (-20, 20), "sin": (-5, 5)}[self.op]
        x = synth.random_elems(rng, self.prec, self.n, lo, hi)
        y = synth.random_elems(rng, self.prec, self.n, lo, hi)
        if self.op in ("sqrt", "log"):
            x = (x[0], x[1] & np.uint32(0xFFFFFFFE))  # positive
        a = synth.from_doubles(self.prec, np.array([1.0]))
        return layout.aos_from_parts(self.prec, *a), layout.aos_from_parts(self.prec, *x), \
            layout.aos_from_parts(self.prec, *y)

    def step(self, i, stream):
        x, y, z = self.sets[i % self.nsets]
        if self.op == "div":
            self.M.div(self.prec, self.n, x, y, z, stream=stream)
        elif self.op == "sin":
            self.M.fmath("sin", self.prec, self.n, x, z, stream=stream)
        else:
            getattr(self.M, self.op)(self.prec, self.n, x, z, stream=stream)

    def e2e_h2d(self, s):
        self.dx_aos[s].copy_(self.hx, non_blocking=True)
        if self.op == "div":
            self.dy_aos[s].copy_(self.hy, non_blocking=True)

    def e2e_bytes(self):
        return (2 if self.op == "div" else 1) * self.host[1].size, self.host[1].size

    @property
    def e2e_launches_per_step(self):
        return 4 if self.op == "div" else 3

    def e2e_compute(self, s, stream):
        M = self.M
        M.pack_aos(self.prec, self.n, self.dx_aos[s], self.ex, stream=stream)
        if self.op == "div":
            M.pack_aos(self.prec, self.n, self.dy_aos[s], self.ey, stream=stream)
            M.div(self.prec, self.n, self.ex, self.ey, self.ez, stream=stream)
        elif self.op == "sin":
            M.fmath("sin", self.prec, self.n, self.ex, self.ez, stream=stream)
        else:
            getattr(M, self.op)(self.prec, self.n, self.ex, self.ez, stream=stream)
        M.unpack_aos(self.prec, self.n, self.ez, self.dz_aos[s], stream=stream)

    def roofline(self, kernel_s, peaks, imad_ops_s):
        N = self.prec // 32
        NW = N + 4  # working precision of the elementary functions
        s_e, T_e, s_c, T_c, T_l = _elem_params(NW)
        mulw, divw = rounded_product_imads(NW), 2 * NW * (NW + 2)
        dui = 5 * (NW + 2)  # division by a small integer: per quotient limb ~5
        # multiply-adds (lo + hi) per element, from the implemented algorithms:
        # a long division is (N+2) quotient limbs x N; the square root about
        # log2(32(N+1)/50) + 2 divisions of (2N+3) by (N+1) limbs; at NW = N+4
        # limbs exp is k ln2, T_e - 1 Taylor steps (a product and a small
        # division), the last product and s_e doublings; log (away from 1) one
        # exp, the product m exp(-y0), a division, T_l atanh steps and e ln2;
        # sin two series of T_c steps and s_c doublings of two products --
        # estimates: counts vary with the argument
        per = {"div": 2 * N * (N + 2),
               "sqrt": int(2 * (N + 1) * (N + 2) * (np.log2(32 * (N + 1) / 50.0) + 2)),
               "exp": (T_e - 1) * (mulw + dui) + (2 + s_e) * mulw,
               "log": (T_e - 1) * (mulw + dui) + (1 + s_e) * mulw + divw + T_l * (mulw + dui) + 4 * mulw,
               "sin": 2 * T_c * (mulw + dui) + 3 * mulw + 2 * s_c * mulw}[self.op]
        imad = per * self.n / kernel_s
        return {"bound": "imad", "achieved": round(imad / 1e9, 1),
                "peak": round(imad_ops_s / 1e9, 1) if imad_ops_s else None, "unit": "Gop/s",
                "frac": round(imad / imad_ops_s, 4) if imad_ops_s else None, "ops_per_unit": per,
                "peak_source": "libmpb_probe.so mad.lo/mad.hi throughput, measured in this run", "traffic": None}

    def cpu_run(self, impl, count):
        import oracle as O

        _, X, Y = self.host
        kind = "ref" if impl == "ref" else "mp"
        if self.op == "div":
            O.div(self.prec, X[:count], Y[:count], impl=kind)
        elif self.op == "sin":
            O.fn("sin", self.prec, X[:count], impl=kind)
        else:
            getattr(O, self.op)(self.prec, X[:count], impl=kind)
        return count

    def config(self):
        return {"workload": self.desc, "prec": self.prec, "n": self.n,
                "units": "one " + {"div": "correctly rounded division", "sqrt": "correctly rounded square root",
                                   "exp": "faithful exponential", "log": "faithful logarithm",
                                   "sin": "faithful sine"}[self.op],
                "l2": f"{self.nsets} rotating input sets > L2"}


class CfnWorkload(AxpyWorkload):
    """z = c<op>(x) over n complex elements at precision prec (each component
    faithful, the contract of the reference's cu_cexp); the CPU baseline is
    the reference's own cu_fcmath function built for the host."""

    def __init__(self, name, op, prec, n, seed):
        super().__init__(name, True, prec, n, seed)
        self.op = op
        self.metric = f"faithful complex {op} (c{op}) per second at PB={prec}"
        self.unit = f"mp-c{op}/s"
        self.desc = (f"complex {op} z=c{op}(x), cu_fcomplex<{prec}>, each component faithful, "
                     f"n=2^{n.bit_length() - 1}, full random significands, component exponents in [-3, 3]")

    @property
    def default_steps(self):  # about 1 s of GPU time
        return 100

    def make_host(self, rank):
        from mpc_cuda_b200 import synth

        rng = np.random.default_rng(shard_seed(self.seed, rank))
        re = synth.random_elems(rng, self.prec, self.n, -3, 3)
        im = synth.random_elems(rng, self.prec, self.n, -3, 3)
        x = synth.interleave_complex(self.prec, re, im)
        return x[:1], x, x  # one input: the AXPY plumbing's a and y go unused

    def step(self, i, stream):
        x, _, z = self.sets[i % self.nsets]
        self.M.cfmath(self.op, self.prec, self.n, x, z, stream=stream)

    def e2e_h2d(self, s):
        self.dx_aos[s].copy_(self.hx, non_blocking=True)

    def e2e_bytes(self):
        return self.host[1].size, self.host[1].size

    e2e_launches_per_step = 3

    def e2e_compute(self, s, stream):
        M = self.M
        M.pack_aos(self.prec, self.n, self.dx_aos[s], self.ex, True, stream=stream)
        M.cfmath(self.op, self.prec, self.n, self.ex, self.ez, stream=stream)
        M.unpack_aos(self.prec, self.n, self.ez, self.dz_aos[s], True, stream=stream)

    def roofline(self, kernel_s, peaks, imad_ops_s):
        NW = self.prec // 32 + 4
        s_e, T_e, s_c, T_c, _ = _elem_params(NW)
        mulw, dui = rounded_product_imads(NW), 5 * (NW + 2)
        # cexp: the exponential of the real part, sine and cosine of the
        # imaginary part (the two series and the doublings), two products --
        # estimated from the implemented algorithms, as for the real functions
        per = ((T_e - 1) * (mulw + dui) + (2 + s_e) * mulw + 2 * T_c * (mulw + dui) + 3 * mulw
               + 2 * s_c * mulw + 2 * mulw)
        imad = per * self.n / kernel_s
        return {"bound": "imad", "achieved": round(imad / 1e9, 1),
                "peak": round(imad_ops_s / 1e9, 1) if imad_ops_s else None, "unit": "Gop/s",
                "frac": round(imad / imad_ops_s, 4) if imad_ops_s else None, "ops_per_unit": per,
                "peak_source": "libmpb_probe.so mad.lo/mad.hi throughput, measured in this run", "traffic": None}

    def cpu_run(self, impl, count):
        import oracle as O

        O.cfn(self.op, self.prec, self.host[1][:count], impl="ref" if impl == "ref" else "mp")
        return count

    def config(self):
        return {"workload": self.desc, "prec": self.prec, "n": self.n,
                "units": f"one faithful complex {self.op} (both components)",
                "l2": f"{self.nsets} rotating input sets > L2"}


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of
# the dominant kernel, from one ncu capture of that kernel on this workload
# (the summaries under profiles/ give the commands); None where no capture exists
NCU_TRAFFIC = {
    "axpy_r256": (82.6e6, "k_axpy_r<8>, profiles/k_axpy_r_pb256_n1048576.md"),
    "axpy_c1024": (180.0e6, "k_axpy_c<32>, profiles/k_axpy_c_pb1024_n262144.md"),
    "gemm_r512": (1.314e9, "k_diag_gemm main pass, profiles/k_diag_gemm_gemm_r512_1024cube.md"),
}

WORKLOADS = {
    "cexp_c512": lambda: CfnWorkload("cexp_c512", "exp", 512, 1 << 18, 0x5EEDB),
    "div_r512": lambda: DivSqrtWorkload("div_r512", "div", 512, 1 << 20, 0x5EED6),
    "sqrt_r512": lambda: DivSqrtWorkload("sqrt_r512", "sqrt", 512, 1 << 20, 0x5EED7),
    "exp_r512": lambda: DivSqrtWorkload("exp_r512", "exp", 512, 1 << 18, 0x5EED8),
    "log_r512": lambda: DivSqrtWorkload("log_r512", "log", 512, 1 << 18, 0x5EED9),
    "sin_r512": lambda: DivSqrtWorkload("sin_r512", "sin", 512, 1 << 18, 0x5EEDA),
    "gemv_batch": lambda: GemvBatchWorkload("gemv_batch", 4096, 0x5EED4),
    "axpy_c1024": lambda: AxpyWorkload("axpy_c1024", True, 1024, 1 << 18, 0x5EED2),
    "axpy_r256": lambda: AxpyWorkload("axpy_r256", False, 256, 1 << 20, 0x5EED1),
    "gemm_r512": lambda: GemmWorkload("gemm_r512", 512, 1024, 1024, 1024, 32,
                                      lambda seed: __import__("mpc_cuda_b200.synth", fromlist=["x"]).gemm_r512(seed)),
    "gemm_c256": lambda: GemmWorkload("gemm_c256", 256, 512, 512, 512, 16,
                                      lambda seed: __import__("mpc_cuda_b200.synth", fromlist=["x"]).gemm_c256(seed),
                                      cplx=True),
}
DEFAULT_WORKLOAD = "gemm_r512"


# ------------------------------------------------------------------ CPU side
def cpu_baseline(wl, seconds=10.0):
    """Time the reference's CPU implementation on a bounded sample (~10 s of
    CPU work: whole passes over the workload, or a prefix of it)."""
    import oracle as O

    impl, kind = ("ref", "reference") if O.ref_available() else ("orc", "port")
    n_total = wl.units()
    t0 = time.perf_counter()
    got = wl.cpu_run(impl, min(n_total, wl.cpu_probe_units))
    dt = max(time.perf_counter() - t0, 1e-6)
    target = min(n_total, max(got, int(got * seconds / 2 / dt)))
    passes, done, t0 = 0, 0, time.perf_counter()
    while True:
        done += wl.cpu_run(impl, target)
        passes += 1
        el = time.perf_counter() - t0
        if el >= seconds or passes >= 1000:
            break
    src = ("reference headers include/mpc_cuda/cu_freal.cuh, cu_fcomplex.cuh, cu_fmath.cuh built for the host "
           "(oracle/_ref), OpenMP" if kind == "reference" else "oracle C restatement, OpenMP")
    return {"value": done / el, "unit": getattr(wl, "unit", "mp-FMA/s"), "cores": O.num_threads(), "kind": kind,
            "sample": f"{passes} pass(es) over {target} of {n_total} units of the same workload, "
                      f"{el:.1f} s; {src}"}


def run_reference(args):
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    wl = WORKLOADS[args.workload]()
    wl.host = wl.make_host(0)
    import oracle as O

    impl, kind = ("ref", "reference") if O.ref_available() else ("orc", "port")
    t0 = time.perf_counter()
    got = wl.cpu_run(impl, min(wl.units(), wl.cpu_probe_units))
    dt = max(time.perf_counter() - t0, 1e-6)
    per_step = min(wl.units(), max(got, int(got * 30.0 / max(args.steps + args.warmup, 1) / dt)))
    for _ in range(args.warmup):
        wl.cpu_run(impl, per_step)
    done = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        done += wl.cpu_run(impl, per_step)
    dt = time.perf_counter() - t0
    per_step = done // args.steps
    value = done / dt
    line = {
        "impl": "reference", "metric": getattr(wl, "metric", METRIC), "value": value,
        "unit": getattr(wl, "unit", "mp-FMA/s"), "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic", "config": wl.config(),
        "cpu_baseline": {"value": value, "unit": getattr(wl, "unit", "mp-FMA/s"), "cores": O.num_threads(), "kind": kind,
                         "sample": f"{per_step} of {wl.units()} units per step"},
        "e2e": {"value": value, "unit": getattr(wl, "unit", "mp-FMA/s"), "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU side
class E2EPipeline:
    """The end-to-end leg, double-buffered over three streams: step i's H2D
    copies (copy-in stream) overlap step i-1's compute (the bench stream) and
    step i-2's D2H copy (copy-out stream).  Every step still copies its own
    inputs in and its result out inside the timed region; slot s = i % 2 of
    the AoS staging buffers is reused only after the step two back has
    finished with it."""

    def __init__(self, wl, main):
        import torch

        self.wl, self.main = wl, main
        self.cin, self.cout = torch.cuda.Stream(main.device), torch.cuda.Stream(main.device)
        mk = lambda: [torch.cuda.Event() for _ in range(2)]  # noqa: E731
        self.ev_in, self.ev_used, self.ev_out = mk(), mk(), mk()
        self.issued = [False, False]

    def start(self):
        self.cin.wait_stream(self.main)
        self.cout.wait_stream(self.main)

    def step(self, i):
        import torch

        s = i & 1
        with torch.cuda.stream(self.cin):
            if self.issued[s]:
                self.cin.wait_event(self.ev_used[s])
            self.wl.e2e_h2d(s)
            self.ev_in[s].record(self.cin)
        self.main.wait_event(self.ev_in[s])
        if self.issued[s]:
            self.main.wait_event(self.ev_out[s])
        self.wl.e2e_compute(s, self.main.cuda_stream)
        self.ev_used[s].record(self.main)
        with torch.cuda.stream(self.cout):
            self.cout.wait_event(self.ev_used[s])
            self.wl.e2e_d2h(s)
            self.ev_out[s].record(self.cout)
        self.issued[s] = True

    def finish(self):
        for s in range(2):
            if self.issued[s]:
                self.main.wait_event(self.ev_out[s])


def split_targets(wl):
    """(kind, prec) of the thread-vs-warp split a workload's kernels read."""
    import mpc_cuda_b200 as M

    if isinstance(wl, AxpyWorkload) and wl.cplx:
        return [(M.SPLIT_AXPY_C, wl.prec)]
    if isinstance(wl, GemvBatchWorkload):
        return [(M.SPLIT_GEMV_R, 1024), (M.SPLIT_GEMV_R, 2048)]
    raise SystemExit(f"--split: workload {wl.name} has no warp-cooperative form")


def shard_seed(base, rank):
    """Seed of a rank's shard: every rank generates its own operands of the
    full workload size (weak scaling; no data crosses ranks)."""
    return base + 1000 * rank


def max_over_ranks_of(v, world, device):
    """The max of v over the ranks of the default process group (the job's
    time is its slowest rank's); device: the tensor's device for the backend
    (cuda for NCCL, cpu for gloo)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_gpu(args):
    import torch
    import torch.distributed as dist

    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    local = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=device)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v):
        return max_over_ranks_of(v, world, device)

    wl = WORKLOADS[args.workload]()
    wl.with_e2e = not args.no_e2e
    if args.split:
        import mpc_cuda_b200 as M

        for kind, prec in split_targets(wl):
            M.set_split(kind, prec, args.split)
    wl.setup(rank, device)
    stream = torch.cuda.current_stream(device)
    sp = stream.cuda_stream

    for i in range(args.warmup):
        wl.step(i, sp)
    torch.cuda.synchronize()

    clocks = make_clocks(local) if rank == 0 else None
    barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
    M = wl.M
    profiled = hasattr(wl, "roofline_tensor")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(args.steps):
        wl.step(i, sp)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    tensor_ms = profiled_ms = None
    if profiled:
        # a second timed region of the same K steps with a CUDA event pair around
        # the tensor-core kernel only: the kernel's own time for the roofline.
        # Events between stages cost their launch overlap, so the step time
        # (`value`) comes from the region above, which records none.
        barrier()
        M.lib().mpb_profile_phases(1 << 2)
        M.lib().mpb_profile_enable(1)
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        for i in range(args.steps):
            wl.step(i, sp)
        e3.record(stream)
        torch.cuda.synchronize()
        profiled_ms = e2.elapsed_time(e3) / args.steps
        cnt = M.lib().mpb_profile_phase_count(2)
        tensor_ms = M.lib().mpb_profile_phase_ms(2) / max(cnt, 1)
        M.lib().mpb_profile_enable(0)
        M.lib().mpb_profile_phases(0xFFFFFFFF)
    barrier()
    clk = clocks.stop() if clocks else None
    ms_max = max_over_ranks(ms)
    kernel_s = ms / args.steps / 1e3

    # end to end through the C ABI from host AoS buffers
    ms_e2e = None
    if not args.no_e2e:
        pipe = E2EPipeline(wl, stream)
        pipe.start()
        for i in range(max(1, args.warmup)):
            pipe.step(i)
        pipe.finish()
        torch.cuda.synchronize()
        barrier()
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        pipe.start()
        for i in range(args.steps):
            pipe.step(i)
        pipe.finish()
        e3.record(stream)
        torch.cuda.synchronize()
        ms_e2e = max_over_ranks(e2.elapsed_time(e3))
        barrier()

    units = wl.units() * world * args.steps
    if rank == 0:
        peaks = measured_peaks()
        extra = wl.extra(sp) if hasattr(wl, "extra") else None
        if profiled:
            roof = wl.roofline_tensor(tensor_ms, int8_peak_ops(device))
            roof["kernel_timing"] = (f"CUDA events around the tensor-core kernel in a second timed region of the same "
                                     f"{args.steps} steps ({profiled_ms:.4f} ms per step there); the headline step "
                                     f"time comes from the first region, which records no events")
        else:
            roof = wl.roofline(kernel_s, peaks, imad_peak(sp))
        if roof.get("traffic") is None and wl.name in NCU_TRAFFIC:
            roof["traffic"], roof["traffic_source"] = NCU_TRAFFIC[wl.name]
        cpu = cpu_baseline(wl) if world == 1 and not args.no_cpu else None
        h2d, d2h = wl.e2e_bytes()
        line = {
            "metric": getattr(wl, "metric", METRIC), "value": units / (ms_max / 1e3),
            "unit": getattr(wl, "unit", "mp-FMA/s"), "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic", "config": {**wl.config(), "parallelism": f"{world} independent shard(s), "
                                                                          "no collective"},
            "roofline": roof, "cpu_baseline": cpu,
            "e2e": None if ms_e2e is None else {
                "value": units / (ms_e2e / 1e3), "unit": getattr(wl, "unit", "mp-FMA/s"), "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e / args.steps,
                "path": "pinned host AoS -> H2D -> mpb_pack_aos -> kernel -> mpb_unpack_aos -> D2H, "
                        "double-buffered: H2D, compute and D2H of consecutive steps overlap"},
            "gpu_launches": wl.launches_per_step * args.steps,
            "gpu_launches_e2e": wl.e2e_launches_per_step * args.steps,
            "clocks": clk,
        }
        if extra:
            line["plain"] = {"value": extra["plain_value"], "unit": "mp-FMA/s",
                             "ms_per_step": extra["plain_ms_per_step"],
                             "kernel": "k_gemm_r (sequential-k, per-operation rounding)",
                             "warps_per_block": extra.get("plain_warps")}
            line["exact_over_plain"] = line["value"] / extra["plain_value"]
            line["status"] = {"fallback_rows_cols": extra["status"][0], "kernel_error": extra["status"][1]}
            if extra.get("accuracy"):
                line["accuracy"] = extra["accuracy"]
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------ kernel tour (profiling)
def run_kernel_tour(args):
    """One launch of each kernel family that has no workload of its own, at
    moderate sizes, for ncu captures (`ncu -k regex:... python bench.py
    --workload kernel_tour`): GEMV at 512 bits (one thread per row) and at 2048
    bits (cooperative), the plain complex GEMM at 256 bits (256^3), the exact
    GEMM's preparation and tail stages (512^3 at 512 bits), division and square
    root (2^18 at 512 bits), sine and complex exponential (2^16 at 512 bits) and
    the cooperative complex AXPY (2^16 at 1024 bits).  Prints one JSON line
    with the wall time of the tour; not a throughput measurement."""
    import torch

    import mpc_cuda_b200 as M
    from mpc_cuda_b200 import layout, synth

    torch.cuda.set_device(0)
    rng = np.random.default_rng(3)

    def vec(prec, n, e=8, cplx=False):
        if cplx:
            re, im = synth.random_elems(rng, prec, n, -e, e), synth.random_elems(rng, prec, n, -e, e)
            return torch.from_numpy(layout.aos_to_vec(prec, synth.interleave_complex(prec, re, im), True).copy()).cuda()
        lm, hd = synth.random_elems(rng, prec, n, -e, e)
        return torch.from_numpy(layout.vec_from_parts(prec, lm, hd).copy()).cuda()

    def posvec(prec, n):
        lm, hd = synth.random_elems(rng, prec, n, -8, 8)
        return torch.from_numpy(layout.vec_from_parts(prec, lm, hd & ~np.uint32(1)).copy()).cuda()

    t0 = time.time()
    m, n = 4096, 256
    M.gemv(512, m, n, vec(512, m * n), n, vec(512, n), vec(512, m), M.empty(512, m))
    m, n = 512, 256
    M.gemv(2048, m, n, vec(2048, m * n), n, vec(2048, n), vec(2048, m), M.empty(2048, m))
    m = 256
    M.gemm(256, m, m, m, vec(256, m * m, cplx=True), m, vec(256, m * m, cplx=True), m, M.empty(256, m * m, True), m,
           cplx=True)
    m = 512
    M.gemm_exact(512, m, m, m, vec(512, m * m), m, vec(512, m * m), m, M.empty(512, m * m), m, sp_bits=32)
    n = 1 << 18
    M.div(512, n, vec(512, n), vec(512, n), M.empty(512, n))
    M.sqrt(512, n, posvec(512, n), M.empty(512, n))
    n = 1 << 16
    M.fmath("sin", 512, n, vec(512, n, e=2), M.empty(512, n))
    M.cfmath("exp", 512, n, vec(512, n, e=2, cplx=True), M.empty(512, n, True))
    old = M.get_split(M.SPLIT_AXPY_C, 1024)
    M.set_split(M.SPLIT_AXPY_C, 1024, 4)
    M.axpy(1024, n, vec(1024, 1, cplx=True), vec(1024, n, cplx=True), vec(1024, n, cplx=True),
           M.empty(1024, n, True), cplx=True)
    M.set_split(M.SPLIT_AXPY_C, 1024, old)
    torch.cuda.synchronize()
    print(json.dumps({"workload": "kernel_tour", "wall_s": round(time.time() - t0, 3), "note": "profiling aid"}))
    return 0


# ------------------------------------------------------------------ drop-in user kernels
DROPIN_PRECS = (64, 96, 128, 160, 256, 288, 512, 1024, 1056, 2048, 4096)  # 4096: the real kernels only


def _uk_lib(path, pre):
    import ctypes as C

    L = C.CDLL(path)
    I, Lg, V, D = C.c_int, C.c_long, C.c_void_p, C.c_double
    for f in ("axpy_r", "axpy_c"):
        getattr(L, pre + f).argtypes = [I, Lg, V, V, V, V, I, I, V]
    getattr(L, pre + "axpy_d").argtypes = [I, Lg, D, V, V, V, I, I, V]
    getattr(L, pre + "caxpy_d").argtypes = [I, Lg, D, D] + [V] * 6 + [I, I, V]
    return L


def run_dropin(args):
    """Kernels written against the cu_fp surface (tests/dropin/user_kernels.cu)
    compiled through this repository's drop-in headers and, beside them, the
    same source compiled against the reference's own headers
    (oracle/_ref/libref_user_kernels.so), timed on the same GPU and data:
    AXPY over device AoS arrays of full-precision cu_freal / cu_fcomplex
    (n = 2^20 real, 2^18 complex; rotating sets larger than L2) and the
    reference's benchmark kernel (demos/bench_3way.cu:44-59: FP64 in and out,
    N = 4096, <<<128, 32>>>, the configuration of its published table)."""
    import torch

    import oracle as O

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    uk = _uk_lib(os.path.join(ROOT, "tests", "dropin", "libuser_kernels.so"), "uk_")
    ref_path = os.path.join(ROOT, "oracle", "_ref", "libref_user_kernels.so")
    refuk = _uk_lib(ref_path, "refuk_") if os.path.exists(ref_path) else None

    def timed(fn, reps):
        for _ in range(args.warmup):
            fn(0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(reps):
            fn(i)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps

    clocks = make_clocks(0)
    clocks.start()
    rows = []
    for prec in DROPIN_PRECS:
        es = O.elem_bytes(prec)
        row = {"prec": prec}
        for kind, n in (("real", 1 << 20), ("complex", 1 << 18)):
            cplx = kind == "complex"
            if cplx and prec > 2048:
                continue
            if prec >= 1024:
                n >>= 2
            X, Y = O.gen_pairs(prec, n, 0xD00D + prec, cplx=cplx)
            a = O.gen_pairs(prec, 1, 0xD00E + prec, cplx=cplx)[0]
            eb = es * (2 if cplx else 1)
            nsets = max(2, -(-2 * L2_BYTES // (3 * n * eb)))
            ta = torch.from_numpy(a.reshape(-1).copy()).to(dev)
            sets = []
            for _ in range(nsets):
                sets.append((torch.from_numpy(X.reshape(-1).copy()).to(dev),
                             torch.from_numpy(Y.reshape(-1).copy()).to(dev),
                             torch.empty(n * eb, dtype=torch.uint8, device=dev)))
            fname = "axpy_c" if cplx else "axpy_r"
            entry = {}
            for tag, L, pre in (("dropin", uk, "uk_"), ("reference", refuk, "refuk_")):
                if L is None:
                    continue
                f = getattr(L, pre + fname)

                def go(i, f=f):
                    x, y, z = sets[i % nsets]
                    rc = f(prec, n, ta.data_ptr(), x.data_ptr(), y.data_ptr(), z.data_ptr(), 0, 128, sp)
                    assert rc == 0, rc

                reps = max(5, min(2000, int(2e9 / (n * (4 if cplx else 1) * (prec // 32) ** 2 * 30))))
                t = timed(go, reps)
                entry[tag] = {"mp_fma_per_s": round(n / t, 1), "ms": round(t * 1e3, 4)}
            if "reference" in entry:
                entry["dropin_over_reference"] = round(entry["reference"]["ms"] / entry["dropin"]["ms"], 3)
            entry["n"] = n
            row[kind] = entry
            del sets
        # the reference's benchmark kernel: FP64 in/out, N = 4096, <<<128, 32>>>
        rng = np.random.default_rng(prec)
        N = 4096
        x, y = (torch.from_numpy(rng.uniform(-1, 1, N)).to(dev) for _ in range(2))
        o = torch.empty(N, dtype=torch.float64, device=dev)
        b3 = {}
        for tag, L, pre in (("dropin", uk, "uk_"), ("reference", refuk, "refuk_")):
            if L is None:
                continue
            f = getattr(L, pre + "axpy_d")
            t = timed(lambda i, f=f: f(prec, N, 1.5, x.data_ptr(), y.data_ptr(), o.data_ptr(), 128, 32, sp), 8)
            b3[tag] = {"ms": round(t * 1e3, 4), "mp_fma_per_s": round(N / t, 1)}
        row["bench_3way_fp64_io_n4096"] = b3
        rows.append(row)
        print(json.dumps(row), file=sys.stderr)
    clk = clocks.stop()
    head = next(r for r in rows if r["prec"] == 256)["real"]
    line = {"metric": "drop-in user-kernel AXPY mp-FMA/s (cu_fp operators in a user kernel), "
                      "reference header on the same GPU beside it",
            "value": head["dropin"]["mp_fma_per_s"], "unit": "mp-FMA/s", "n_gpus": 1,
            "steps": None, "warmup": args.warmup, "higher_is_better": True, "scaling": None,
            "vs_baseline": None, "dtype": "u32 limbs (drop-in: 64-bit limbs in memory)", "data": "synthetic",
            "config": {"workload": "user kernels through include/mpc_cuda headers: real AXPY PB=256 n=2^20 "
                                   "(value), every PB and the complex / FP64-I/O forms in per_prec",
                       "l2": "rotating input sets larger than L2"},
            "clocks": clk, "per_prec": rows}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: the workload's, about 2 s of GPU time)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("mpb", "reference"), default="mpb")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["dropin_axpy", "kernel_tour"], default=DEFAULT_WORKLOAD)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiling runs)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--split", type=int, default=0,
                    help="lanes per element for the kernels with a warp-cooperative form (mpb_set_split); "
                         "0 keeps the library's default")
    ap.add_argument("--problems", type=int, default=None,
                    help="gemv_batch only: number of problems (profiling runs on a small case)")
    args = ap.parse_args()
    if args.problems is not None:
        if args.workload != "gemv_batch" or args.problems < 1:
            ap.error("--problems applies to --workload gemv_batch, with a positive count")
        WORKLOADS["gemv_batch"] = lambda: GemvBatchWorkload("gemv_batch", args.problems, 0x5EED4)
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "dropin_axpy":
        return run_dropin(args)
    if args.workload == "kernel_tour":
        return run_kernel_tour(args)
    if args.steps is None:
        args.steps = WORKLOADS[args.workload]().default_steps
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
