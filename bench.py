"""Benchmark of the SHGEMM hot path on B200.

Default (``--workload headline``): the served sketch stream -- Poisson arrivals at 2000
requests/s of sketch requests Y = A [Omega_1 .. Omega_4], m log-U[1024, 65536], k
log-U[1024, 16384], n in {64, 128, 256}, A low rank (rank n, sigma_j = j^-2) plus noise,
Gaussian Omega generated on the device, TF32 compute, 40 GB HBM admission budget -- for
``--duration`` seconds (10 by default; the stream the workload names runs 60). ``value`` is
the served TFLOP/s (2 m n k per draw, completed requests over the stream's span) with
p50/p99 latency, next to the same requests as plain per-call shgemm launches and the
server's saturation throughput on them. The same JSON line nests the grouped batch of 512
uneven sketches (one CUDA-graph-captured launch against its per-call loop) and the large
square SHGEMM at 16384^3 (binary16 timed, binary16 and TF32 errors against FP64).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload headline|served|grouped|square16k|...]
    python bench.py --impl reference ...   # the reference algorithm on the host cores

Prints one JSON line (rank 0). Under torchrun (N > 1) every rank runs an independent
replica (the path has no cross-GPU exchange); times are the max over ranks and values
aggregates.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "served TFLOP/s & p99 latency vs per-call SHGEMM; rel. error vs FP64"

SERVED = dict(m=0, n=0, k=0, op_a=0, op_b=0, tc=1, alpha=1.0, beta=0.0, dist="served", bound="tensor",
              rate=2000.0, duration=10.0, budget=40 << 30, draws=4, m_min=1024, m_max=65536, k_min=1024,
              k_max=16384, ns=(64, 128, 256),
              desc="served sketch stream: Poisson arrivals at 2000 req/s, m log-U[1024,65536], "
                   "k log-U[1024,16384], n in {64,128,256}, 4 Gaussian Omega draws per resident A "
                   "(rank n, sigma_j = j^-2, + N(0,1e-6)), tf32 compute, 40 GB admission budget")

WORKLOADS = {
    # the headline: the served stream, with the grouped batch and the large square SHGEMM nested
    "headline": dict(SERVED, dist="headline"),
    # the served stream alone
    "served": SERVED,
    # the large square SHGEMM
    "square16k": dict(m=16384, n=16384, k=16384, op_a=0, op_b=0, tc=0, alpha=1.0, beta=0.5, dist="wide",
                      desc="large square SHGEMM 16384^3 NN, fp16 compute, A N(0,1)*2^U(-15,15), B N(0,1), beta=0.5"),
    # the same product with A transposed: the FP32 operand K-major (rows of k contiguous floats)
    "square16k_tn": dict(m=16384, n=16384, k=16384, op_a=1, op_b=0, tc=0, alpha=1.0, beta=0.5, dist="wide",
                         desc="large square SHGEMM 16384^3 TN, fp16 compute, A N(0,1)*2^U(-15,15), B N(0,1), "
                              "beta=0.5"),
    # the large square SHGEMM with lda = m + 1 (4-byte aligned columns): TMA cannot address A, so
    # it is staged into the workspace (sized here to hold all of A: one k-slab)
    "square16k_oddld": dict(m=16384, n=16384, k=16384, op_a=0, op_b=0, tc=0, alpha=1.0, beta=0.5, dist="wide",
                            lda_pad=1, desc="large square SHGEMM 16384^3 NN with lda = 16385, fp16 compute, "
                                            "A N(0,1)*2^U(-15,15), B N(0,1), beta=0.5"),
    # a smaller square case of the same kernel, for profiler captures (inputs still exceed L2)
    "square8k": dict(m=8192, n=8192, k=8192, op_a=0, op_b=0, tc=0, alpha=1.0, beta=0.5, dist="wide",
                     desc="square SHGEMM 8192^3 NN, fp16 compute, A N(0,1)*2^U(-15,15), B N(0,1), beta=0.5"),
    # square8k with A transposed (K-major FP32 operand), for profiler captures of that load path
    "square8k_tn": dict(m=8192, n=8192, k=8192, op_a=1, op_b=0, tc=0, alpha=1.0, beta=0.5, dist="wide",
                        desc="square SHGEMM 8192^3 TN, fp16 compute, A N(0,1)*2^U(-15,15), B N(0,1), beta=0.5"),
    # a still smaller square case: with square8k it shows how DRAM traffic scales with the problem
    "square4k": dict(m=4096, n=4096, k=4096, op_a=0, op_b=0, tc=0, alpha=1.0, beta=0.5, dist="wide",
                     desc="square SHGEMM 4096^3 NN, fp16 compute, A N(0,1)*2^U(-15,15), B N(0,1), beta=0.5"),
    # the small square SHGEMM (1024^3)
    "square1k": dict(m=1024, n=1024, k=1024, op_a=0, op_b=0, tc=0, alpha=1.0, beta=0.0, dist="uniform",
                     desc="plain SHGEMM 1024^3 NN, fp16 compute, A U[-1,1], B U[-1,1]"),
    "square1k_tf32": dict(m=1024, n=1024, k=1024, op_a=0, op_b=0, tc=1, alpha=1.0, beta=0.0, dist="uniform",
                          desc="plain SHGEMM 1024^3 NN, tf32 compute, A U[-1,1], B U[-1,1]"),
    # Y = Omega^T A as hsgemm(op_t, op_n) -> internal shgemm(op_t, op_n, 4096, 256, 2^20, op_c = t)
    "sketch": dict(m=4096, n=256, k=1 << 20, op_a=1, op_b=0, tc=0, alpha=1.0, beta=0.0, dist="sketch",
                   desc="left sketch Y = Omega^T A, A 2^20 x 4096 FP32 (low rank + noise), Omega 2^20 x 256 "
                        "binary16 N(0,1/256), split-K, fp16 compute", op_c=1, bound="hbm"),
    "sketch_tf32": dict(m=4096, n=256, k=1 << 20, op_a=1, op_b=0, tc=1, alpha=1.0, beta=0.0, dist="sketch",
                        desc="left sketch Y = Omega^T A as the binary16 sketch, tf32 compute", op_c=1, bound="hbm"),
    "sketch128k_tf32": dict(m=4096, n=256, k=1 << 17, op_a=1, op_b=0, tc=1, alpha=1.0, beta=0.0, dist="sketch",
                            op_c=1, desc="left sketch Y = Omega^T A at 2^17, tf32 compute", bound="hbm"),
    # the sketch at 1/8 of its length (A 2 GiB, still 16x L2), for profiler captures
    "sketch128k": dict(m=4096, n=256, k=1 << 17, op_a=1, op_b=0, tc=0, alpha=1.0, beta=0.0, dist="sketch",
                       op_c=1, desc="left sketch Y = Omega^T A, A 2^17 x 4096 FP32 (low rank + noise), "
                                    "Omega 2^17 x 256 binary16", bound="hbm"),
    # 512 uneven right sketches in one graph-captured grouped launch
    "grouped": dict(m=0, n=0, k=0, op_a=0, op_b=0, tc=0, alpha=1.0, beta=0.0, dist="grouped", count=512, bound="hbm",
                    desc="grouped batch of 512 uneven right sketches Y_i = A_i Omega_i, m_i log-U[64,8192], "
                         "k_i log-U[256,16384], n_i in {32,64,128,256}, A_i rank n_i/2 (sigma_j = j^-1.5) + N(0,1e-4), "
                         "Omega_i Rademacher/sqrt(n_i) (block-sign +-1 operand, the scale as alpha), fp16 compute, "
                         "one CUDA-graph-captured launch"),
    # the reference's power test: square 2^10 .. 2^14 NN, TF32 and fp16, ~10 s loops under NVML
    "energy": dict(m=0, n=0, k=0, op_a=0, op_b=0, tc=0, alpha=1.0, beta=0.0, dist="energy",
                   desc="energy per call: square SHGEMM m = n = k = 2^10 .. 2^14 NN, inputs uniform (0, 1], "
                        "tf32 and fp16 compute, a ~10 s loop per shape with NVML power sampled every 50 ms"),
    # the same batch with Omega_i generated inside the grouped kernel (no Omega in memory)
    "grouped_fused": dict(m=0, n=0, k=0, op_a=0, op_b=0, tc=0, alpha=1.0, beta=0.0, dist="grouped", count=512,
                          bound="hbm", fused=True,
                          desc="grouped batch of 512 uneven right sketches (shapes as the fp16 batch), Omega_i "
                               "block-sign Rademacher generated inside the grouped kernel (no Omega reads), "
                               "scale 1/sqrt(n_i) as alpha, fp16 compute, one CUDA-graph-captured launch"),
    # the same batch in TF32 compute, Omega_i handed over widened to FP32 (as the sketch server keeps it)
    "grouped_tf32": dict(m=0, n=0, k=0, op_a=0, op_b=0, tc=1, alpha=1.0, beta=0.0, dist="grouped", count=512,
                         bound="hbm", b_fp32=True,
                         desc="grouped batch of 512 uneven right sketches (shapes as the fp16 batch), tf32 compute, "
                              "Omega_i widened to FP32 once, one CUDA-graph-captured launch"),
}


# ---------------------------------------------------------------- common
class Ctx:
    """Rank, device and process group of this replica."""

    def __init__(self, timeout_s=600):
        import torch

        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            torch.cuda.set_device(self.local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist
        self.dev = torch.device(f"cuda:{self.local}")
        torch.cuda.set_device(self.dev)

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def reduce(self, x: float, op: str = "max") -> float:
        """x reduced over ranks (max or sum); every rank gets the result."""
        if self.dist is None:
            return x
        import torch

        t = torch.tensor([x], device=self.dev, dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX if op == "max" else self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def tensor_peak(sustained: bool, tc: int):
    """Dense tensor peak for the roofline: measured bf16 (binary16 runs at the same rate),
    burst or sustained, halved for TF32."""
    peaks, kind = load_peaks()
    p = peaks.get("bf16_tflops_sustained", 1400.0) if sustained else peaks.get("bf16_tflops", 1590.0)
    label = f"{kind} bf16 dense {'sustained' if sustained else 'burst'}"
    if tc:
        p /= 2
        label += " / 2 (TF32 rate)"
    return p, label


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons, pw = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
                pw.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_median": statistics.median(pw) if pw else None}


def energy(clk, ms_per_call, flops_per_call):
    """Board energy per call from the power samples of the timed region (the reference's
    J-per-GEMM figure, test/power_consumption_test.cu:94-123, from nvidia-smi instead of NVML)."""
    p = clk.get("power_w_median")
    if not p:
        return None
    j = p * ms_per_call * 1e-3
    return {"avg_board_power_w": p, "joules_per_call": j, "effective_gflop_per_joule": flops_per_call / j / 1e9,
            "source": "nvidia-smi power.draw median over the timed region (whole board)"}


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def nvml_monitor(device_index):
    """An NVML power monitor of the device (energy counter + 50 ms samples), or None."""
    try:
        from shgemm_b200 import energy as en

        return en.PowerMonitor(device_index, 50.0)
    except Exception:
        return None


def nvml_energy(mon, calls, flops_per_call):
    """Energy per call of a timed region from the NVML monitor that ran over it (the
    reference's J-per-GEMM figure, test/power_consumption_test.cu:94-123)."""
    if mon is None:
        return None
    try:
        r = mon.result()
    except Exception:
        return None
    j = r["joules"] / calls
    if not j > 0:  # the counter did not advance over a region this short
        return None
    return {"avg_board_power_w": r["avg_w"], "joules_per_call": j, "effective_gflop_per_joule": flops_per_call / j / 1e9,
            "source": r["source"] + " over the timed region (whole board)", "samples": r["samples"]}


def traffic_for(key):
    """DRAM bytes per launch from a committed ncu summary (profiles/traffic.json), if captured."""
    f = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(f):
        with open(f) as fh:
            return json.load(fh).get(key)
    return None


# ---------------------------------------------------------------- square / sketch workloads
def make_inputs(wl, dev, seed=0):
    import torch

    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    m, n, k = wl["m"], wl["n"], wl["k"]
    a_rows = (m if wl["op_a"] == 0 else k) + wl.get("lda_pad", 0)  # a padded lda: not TMA-addressable
    b_rows = k if wl["op_b"] == 0 else n
    na = a_rows * (k if wl["op_a"] == 0 else m)
    nb = k * n
    if wl["dist"] == "wide":
        A = torch.randn(na, generator=g, device=dev)
        A.mul_(torch.exp2(torch.empty(na, device=dev).uniform_(-15, 15, generator=g)))
        B = torch.randn(nb, generator=g, device=dev).to(torch.float16)
    elif wl["dist"] == "sketch":
        # A (k x m, K-contiguous for op_t) = U diag(sigma) V^T, rank 512, sigma_i = i^-2, + N(0, 1e-6) noise
        r = 512
        U = torch.linalg.qr(torch.randn(k, r, generator=g, device=dev))[0]
        V = torch.linalg.qr(torch.randn(m, r, generator=g, device=dev))[0]
        sig = torch.arange(1, r + 1, device=dev, dtype=torch.float32).pow(-2.0)
        Amat = (U * sig) @ V.T  # k x m; column-major storage of an (a_rows=k) x m matrix = row-major m x k
        Amat.add_(torch.randn(k, m, generator=g, device=dev), alpha=1e-6)
        A = Amat.T.contiguous().reshape(-1)  # element (kk, i) at kk + i * k
        del U, V, Amat
        B = (torch.randn(nb, generator=g, device=dev) / 16.0).to(torch.float16)  # N(0, 1/256)
    else:
        A = torch.empty(na, device=dev).uniform_(-1, 1, generator=g)
        B = torch.empty(nb, device=dev).uniform_(-1, 1, generator=g).to(torch.float16)
    op_c = wl.get("op_c", 0)
    C = torch.empty(m * n, device=dev).uniform_(-1, 1, generator=g)
    return A, a_rows, B, b_rows, C, (m if op_c == 0 else n)


def gpu_error(h, wl, A, lda, B, ldb, C_out, ldc, C0, c64=None):
    """Relative Frobenius error vs the FP64 product (GPU), plus FP32 SGEMM's (torch, no TF32).
    Returns (error dict, c64) so a second compute type can reuse the FP64 product."""
    import torch

    from shgemm_b200 import evaluation as ev

    m, n, k = wl["m"], wl["n"], wl["k"]
    op_c = wl.get("op_c", 0)
    if c64 is None:
        c64 = ev.fp64_product(h, wl["op_a"], wl["op_b"], m, n, k, A, lda, B, ldb)
    e = ev.error(h, m, n, C_out, ldc, c64, wl["alpha"], wl["beta"], C0 if wl["beta"] != 0 else None, op_c)
    # plain FP32 SGEMM of the same inputs for comparison
    torch.backends.cuda.matmul.allow_tf32 = False
    Am = A.view(-1, lda).T if wl["op_a"] == 0 else A.view(-1, lda)  # logical m x k
    Bm = B.float().view(-1, ldb).T if wl["op_b"] == 0 else B.float().view(-1, ldb)
    S = Am[:m, :k] @ Bm[:k, :n]  # m x n
    S = S.mul_(wl["alpha"])
    if wl["beta"] != 0:
        C0m = C0.view(-1, ldc).T[:m, :n] if op_c == 0 else C0.view(-1, ldc)[:m, :n]
        S.add_(C0m, alpha=wl["beta"])
    Sbuf = S.T.contiguous().reshape(-1) if op_c == 0 else S.contiguous().reshape(-1)
    torch.cuda.synchronize()  # Sbuf comes from torch's stream, the error kernel runs on the handle's
    es = ev.error(h, m, n, Sbuf, m if op_c == 0 else n, c64, wl["alpha"], wl["beta"],
                  C0 if wl["beta"] != 0 else None, op_c)
    # binary16 compute: an FP32 entry of magnitude >= 65520 rounds to inf in the hi part (as in
    # the reference), so every output of its row of op(A) is non-finite while FP64 stays finite
    expected = 0
    if wl["tc"] == 0:
        rows = (Am[:m, :k].abs() >= 65520.0).any(dim=1)
        expected = int(rows.sum().item()) * n
    del S, Sbuf
    finite = 1.0 - (e["nonfinite_mismatch"] / float(m * n))
    out = {"rel_err_fp64": e["rel_fro"], "max_rel_err_fp64": e["max_rel"],
           "finite_fraction": finite,
           "nonfinite_mismatch": e["nonfinite_mismatch"],
           "sgemm_rel_err_fp64": es["rel_fro"]}
    if wl["tc"] == 0:
        out["nonfinite_expected_fp16_overflow"] = expected
        out["note"] = ("rel_err over entries finite in both; non-finite outputs come from binary16 overflow of "
                       "the FP32 operand (rows with |a| >= 65520), the reference's behaviour")
    return out, c64


def square_case(args, wl, ctx, traffic_key, tf32_error=False, e2e=True):
    """One plain SHGEMM workload: autotuned, W warm-up and K timed calls (CUDA events on the
    launching stream), error against FP64, host-buffer end to end. Returns a result dict."""
    import torch

    import shgemm_b200 as sg

    dev = ctx.dev
    h = sg.Handle(ctx.local)
    stream = torch.cuda.current_stream(dev)
    h.set_stream(stream)
    m, n, k = wl["m"], wl["n"], wl["k"]
    op_c = wl.get("op_c", 0)
    A, lda, B, ldb, C, ldc = make_inputs(wl, dev, seed=ctx.rank)
    C0 = C.clone() if wl["beta"] != 0 else None

    h.set_config(sg.CFG_K_CHUNK, args.k_chunk)
    if args.group_m:
        h.set_config(sg.CFG_GROUP_M, args.group_m)
    h.set_config(sg.CFG_TM_STAGES, args.stages)
    h.set_config(sg.CFG_PAIR_TILES, args.pair)
    if (wl["tc"] == 1 or tf32_error) and wl["op_b"] == 0:
        # room for the widened FP32 copy of B (the TF32 kernels that load B unconverted) and for
        # split-K partials beside it
        h.set_workspace_size(n * ((k + 3) // 4 * 4) * 4 + (64 << 20))
    if wl.get("lda_pad"):
        # room for the staged copy of A (aligned leading dimension) in one k-slab
        cols = k if wl["op_a"] == 0 else m
        h.set_workspace_size((64 << 20) + ((lda - wl["lda_pad"] + 3) // 4 * 4) * cols * 4)
    if wl["tc"] == 0 and wl["op_b"] == 0 and ldb * 2 >= (1 << 20):
        # room for B re-laid out as contiguous k-blocks (columns >= 1 MiB apart) plus the split-K partials
        h.set_workspace_size((64 << 20) + n * ((k + 63) // 64 * 64) * 2)
    tuned = None
    if not args.no_autotune and op_c == 0 and not wl.get("lda_pad"):  # tuning takes TMA-addressable operands
        tuned = h.autotune(wl["op_a"], wl["op_b"], m, n, k, A, lda, B, ldb, C, ldc, wl["tc"])
        if C0 is not None:
            C.copy_(C0)
        torch.cuda.synchronize(dev)

    def step(tc=wl["tc"]):
        return sg.shgemm(h, wl["op_a"], wl["op_b"], m, n, k, wl["alpha"], A, lda, B, ldb, wl["beta"], C, ldc, tc, op_c)

    level = None
    for _ in range(args.warmup):
        level = step()
    torch.cuda.synchronize(dev)
    if h.check_error() != 0:
        raise RuntimeError("device-side timeout during warm-up")

    ctx.barrier()
    torch.cuda.synchronize(dev)
    launches0 = h.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    mon = nvml_monitor(ctx.local)
    with ClockSampler(ctx.local) as clk, (mon or _Null()):
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    launches = h.launch_count() - launches0
    ctx.barrier()
    ms_total = ctx.reduce(ev0.elapsed_time(ev1))
    ms_step = ms_total / args.steps
    flops_eff = 2.0 * m * n * k
    flops_issued = 4.0 * m * n * k
    value = ctx.world * flops_eff * args.steps / (ms_total * 1e-3) / 1e12
    if h.check_error() != 0:
        raise RuntimeError("device-side timeout in the timed region")

    # ---- error vs FP64 (outside the timed region; fresh C from the same C0)
    err, c64 = {}, None
    if not args.no_error:
        if C0 is not None:
            C.copy_(C0)
        step()
        torch.cuda.synchronize(dev)
        err, c64 = gpu_error(h, wl, A, lda, B, ldb, C, ldc, C0)
    tf32 = None
    if tf32_error and not args.no_error:
        # the same inputs in TF32 compute (no binary16 overflow: the check covers all of C)
        wl32 = dict(wl, tc=1)
        for _ in range(2):
            if C0 is not None:
                C.copy_(C0)
            step(tc=1)
        torch.cuda.synchronize(dev)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if C0 is not None:
            C.copy_(C0)
        t0.record(stream)
        step(tc=1)
        t1.record(stream)
        torch.cuda.synchronize(dev)
        ms32 = t0.elapsed_time(t1)
        e32, _ = gpu_error(h, wl32, A, lda, B, ldb, C, ldc, C0, c64=c64)
        tf32 = {"error": e32, "ms_per_call": ms32, "tflops": flops_eff / (ms32 * 1e-3) / 1e12,
                "note": "one TF32 call of the same inputs (widened-B route), timed alone after two warm-up calls"}
    del c64

    # ---- end to end through the public API with host buffers (pinned), copies timed
    e2e_d = None
    if e2e and not args.no_e2e:
        hA = torch.empty(A.numel(), dtype=A.dtype, pin_memory=True)
        hB = torch.empty(B.numel(), dtype=B.dtype, pin_memory=True)
        hC = torch.empty(C.numel(), dtype=C.dtype, pin_memory=True)
        hA.copy_(A)
        hB.copy_(B)
        hC.copy_(C0 if C0 is not None else C)
        h2d = hA.numel() * 4 + hB.numel() * 2 + (hC.numel() * 4 if wl["beta"] != 0 else 0)
        d2h = hC.numel() * 4
        e2e_steps = max(1, min(args.steps, 5))

        def e2e_step():
            # the library's host-buffer entry point: A up once, then C in column blocks whose
            # B/C uploads, computation and C downloads overlap on separate streams
            return sg.shgemm_host(h, wl["op_a"], wl["op_b"], m, n, k, wl["alpha"], hA, lda, hB, ldb, wl["beta"], hC,
                                  ldc, wl["tc"], op_c)

        e2e_step()
        torch.cuda.synchronize(dev)
        ctx.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            e2e_step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        te = ctx.reduce(e0.elapsed_time(e1))
        e2e_d = {"value": ctx.world * flops_eff * e2e_steps / (te * 1e-3) / 1e12, "unit": "TFLOP/s",
                 "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
                 "path": "shgemm_b200_shgemm_host on page-locked host buffers (copies overlapped with compute)"}
        sg.release_host_staging(h)
        del hA, hB, hC

    # ---- roofline of the tile kernel (its launches are the timed steps)
    bytes_min = 4.0 * m * k + 2.0 * k * n + 4.0 * m * n * (2 if wl["beta"] != 0 else 1)
    if wl.get("bound", "tensor") == "hbm":
        peaks, peak_kind = load_peaks()
        peak = peaks.get("hbm_gbs", 6650.0)
        achieved = bytes_min / (ms_step * 1e-3) / 1e9
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": None, "peak_kind": f"{peak_kind} HBM copy bandwidth",
                    "work_per_launch": f"A + B + C = {bytes_min:.4e} bytes (each operand read once)"}
        # the issued tensor work against its own peak beside the bandwidth fraction: a sketch in
        # TF32 (half the binary16 rate) can be tensor-bound
        t_peak, t_label = tensor_peak(ms_total >= 100.0, wl["tc"])
        t_ach = flops_issued / (ms_step * 1e-3) / 1e12
        roofline["tensor"] = {"achieved": t_ach, "peak": t_peak, "unit": "TFLOP/s", "frac": t_ach / t_peak,
                              "peak_kind": t_label}
    else:
        # burst peak for a short timed region, the power-capped sustained one for a long one
        peak, label = tensor_peak(ms_total >= 100.0, wl["tc"])
        achieved = flops_issued / (ms_step * 1e-3) / 1e12
        roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": None, "peak_kind": label,
                    "work_per_launch": f"4mnk = {flops_issued:.4e} issued tensor flops (two MMAs per k: hi and lo)"}
    roofline["traffic"] = traffic_for(traffic_key + ("_tf32" if wl["tc"] else ""))
    if roofline["traffic"] is not None:
        roofline["traffic_source"] = traffic_for(traffic_key + ("_tf32" if wl["tc"] else "") + "_source")
    clocks = clk.summary()
    h.close()
    del A, B, C, C0
    torch.cuda.empty_cache()
    return {"value": value, "ms_per_step": ms_step, "steps": args.steps, "level": level, "tuned": tuned,
            "issued_tflops": ctx.world * flops_issued * args.steps / (ms_total * 1e-3) / 1e12,
            "gpu_launches": launches, "roofline": roofline, "clocks": clocks,
            "energy": nvml_energy(mon, args.steps, flops_eff) or energy(clocks, ms_step, flops_eff),
            "error": err, "tf32": tf32, "e2e": e2e_d}


# ---------------------------------------------------------------- grouped batch
def make_grouped_batch(count, dev, seed=0):
    """The uneven sketch batch on the device; returns problem tuples, sizes, the tensors to
    keep, and each problem's Omega seed. Omega_i is the block-sign Rademacher operand of its
    seed (entries +1 / -1, generated on the device) and the 1/sqrt(n_i) scale is alpha, so the
    same batch can also run with Omega_i generated inside the grouped kernel."""
    import numpy as np
    import torch

    from shgemm_b200 import server as srv

    rng = np.random.default_rng(seed)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    ms = np.exp(rng.uniform(np.log(64), np.log(8192), count)).astype(int)
    ks = np.exp(rng.uniform(np.log(256), np.log(16384), count)).astype(int)
    ns = rng.choice([32, 64, 128, 256], count)
    probs, shapes, keep, seeds = [], [], [], []
    for i, (m, k, n) in enumerate(zip(ms, ks, ns)):
        m, k, n = int(m), int(k), int(n)
        lda = (m + 3) // 4 * 4
        ldb = (k + 7) // 8 * 8
        r = max(1, n // 2)
        # A = U diag(sigma) V^T + N(0, 1e-4): rank n/2, sigma_j = j^-1.5
        U = torch.randn(m, r, device=dev, generator=g) / np.sqrt(m)
        V = torch.randn(k, r, device=dev, generator=g) / np.sqrt(k)
        sig = torch.arange(1, r + 1, device=dev, dtype=torch.float32).pow(-1.5)
        Afull = torch.empty(k, lda, device=dev)  # column-major m x k with leading dimension lda
        Afull[:, :m] = ((U * sig) @ V.T).T
        Afull[:, :m].add_(torch.randn(k, m, device=dev, generator=g), alpha=1e-2)
        Om = torch.zeros(n, ldb, device=dev, dtype=torch.float16)  # column-major k x n, ld = ldb
        sd = seed * 1000003 + i
        srv.generate_omega(Om, ldb, k, n, srv.RADEMACHER_BLOCKS, sd, 1.0)
        Y = torch.zeros(n, m, device=dev)
        A = Afull.reshape(-1)
        B = Om.reshape(-1)
        C = Y.reshape(-1)
        keep.append((A, B, C))
        probs.append((m, n, k, A, lda, B, ldb, C, m, float(n) ** -0.5, 0.0))
        shapes.append((m, n, k))
        seeds.append(sd)
    return probs, shapes, keep, seeds


def grouped_case(args, wl, ctx, steps=None):
    """The grouped batch: one graph-captured launch replayed K times, its per-call loop,
    and errors of a sample of problems against FP64."""
    import torch

    import shgemm_b200 as sg
    from shgemm_b200 import evaluation as ev
    from shgemm_b200 import server as srv

    steps = steps or args.steps
    dev = ctx.dev
    h = sg.Handle(ctx.local)
    stream = torch.cuda.Stream(dev)
    h.set_stream(stream)
    probs, shapes, keep, seeds = make_grouped_batch(args.count or wl["count"], dev, seed=ctx.rank)
    torch.cuda.synchronize(dev)
    flops = sum(2.0 * m * n * k for (m, n, k) in shapes)
    b_bytes = 0.0 if wl.get("fused") else (4.0 if wl.get("b_fp32") else 2.0)
    bytes_min = sum(4.0 * m * k + b_bytes * k * n + 4.0 * m * n for (m, n, k) in shapes)
    gprobs, keep_w = probs, []
    if wl.get("fused"):
        # Omega_i generated inside the grouped kernel from its seed: not read at all
        gprobs = [(m, n, k, A, lda, None, 0, C, ldc, al, be, srv.RADEMACHER_BLOCKS, sd)
                  for (m, n, k, A, lda, B, ldb, C, ldc, al, be), sd in zip(probs, seeds)]
    elif wl.get("b_fp32"):
        # Omega_i widened to FP32 once (exact: binary16 values), K-major with a 16-byte ld
        gprobs = []
        for (m, n, k, A, lda, B, ldb, C, ldc, al, be) in probs:
            ldb4 = (k + 3) // 4 * 4
            Bw = torch.zeros(n, ldb4, device=dev)
            Bw[:, :k] = B.view(n, ldb)[:, :k].float()
            keep_w.append(Bw)
            gprobs.append((m, n, k, A, lda, Bw.reshape(-1), ldb4, C, ldc, al, be))
        h.set_config(sg.CFG_GROUPED_B_FP32, 1)

    # tile N per n bucket tuned on this batch (not timed), then the launch captured once and
    # replayed per step
    tiles = None
    if not args.no_autotune:
        h.autotune_grouped(gprobs, wl["tc"])
        tiles = {f"n in [{1 << L}, {2 << L})": h.autotune_grouped_lookup(1 << L, wl["tc"], 0, bool(wl.get("b_fp32")))
                 for L in sorted({int(n).bit_length() - 1 for (_, n, _) in shapes})}
    with torch.cuda.stream(stream):
        sg.shgemm_grouped(h, gprobs, wl["tc"])
    stream.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        sg.shgemm_grouped(h, gprobs, wl["tc"])
    with torch.cuda.stream(stream):  # replays run on the current stream
        for _ in range(args.warmup):
            graph.replay()
    torch.cuda.synchronize(dev)
    ctx.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(ctx.local) as clk, torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(steps):
            graph.replay()
        e1.record(stream)
        torch.cuda.synchronize(dev)
    ms_step = ctx.reduce(e0.elapsed_time(e1)) / steps
    value = ctx.world * flops / (ms_step * 1e-3) / 1e12
    assert h.check_error() == 0

    # the per-call baseline: one shgemm launch per problem, same stream
    def per_call():
        for (m, n, k, A, lda, B, ldb, C, ldc, al, be) in probs:
            sg.shgemm(h, 0, 0, m, n, k, al, A, lda, B, ldb, be, C, ldc, wl["tc"])

    with torch.cuda.stream(stream):
        per_call()
        stream.synchronize()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        steps_pc = max(1, min(steps, 5))
        p0.record(stream)
        for _ in range(steps_pc):
            per_call()
        p1.record(stream)
    torch.cuda.synchronize(dev)
    ms_pc = ctx.reduce(p0.elapsed_time(p1)) / steps_pc
    per_call_tflops = flops / (ms_pc * 1e-3) / 1e12

    # error on a sample of problems vs the FP64 product (outputs of a graph replay)
    for (_, _, C) in keep:
        C.zero_()
    with torch.cuda.stream(stream):
        graph.replay()
    torch.cuda.synchronize(dev)
    errs = []
    torch.backends.cuda.matmul.allow_tf32 = False
    if not args.no_error:
        with torch.cuda.stream(stream):  # the library's error kernels run on the handle's stream
            for i in range(0, len(probs), max(1, len(probs) // 16)):
                m, n, k, A, lda, B, ldb, C, ldc, al, be = probs[i]
                c64 = ev.fp64_product(h, 0, 0, m, n, k, A, lda, B, ldb)
                e_sh = ev.error(h, m, n, C, ldc, c64, al)["rel_fro"]
                Bf = B.view(n, ldb)[:, :k].float()
                Af = A.view(k, lda)[:, :m].T
                S = (Af @ Bf.T).mul_(al).T.contiguous().reshape(-1)  # n x m row-major == m x n column-major
                errs.append((e_sh, ev.error(h, m, n, S, m, c64, al)["rel_fro"]))
        torch.cuda.synchronize(dev)
    del graph
    h.close()
    del probs, gprobs, keep, keep_w
    torch.cuda.empty_cache()

    peaks, peak_kind = load_peaks()
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = bytes_min / (ms_step * 1e-3) / 1e9
    # the Omega-generating launch reads no Omega: its ratio is not the measured one
    ratio = None if wl.get("fused") else traffic_for("grouped" + ("_tf32" if wl["tc"] else "") + "_dram_ratio")
    return {
        "value": value, "unit": "TFLOP/s", "ms_per_step": ms_step, "steps": steps,
        "workload": wl["desc"].replace("batch of 512", f"batch of {len(shapes)}"),
        "problems": len(shapes), "total_flops_2mnk": flops, "algorithmic_bytes": bytes_min,
        "autotuned_tile_n": tiles,
        "per_call_baseline": {"value": per_call_tflops, "unit": "TFLOP/s", "ms_per_step": ms_pc,
                              "launches_per_step": len(shapes),
                              "what": "the same problems as one shgemm call (one launch) each, back to back"},
        "speedup_vs_per_call": value / ctx.world / per_call_tflops,
        "issued_tflops": 2 * value,
        "gpu_launches": steps,  # one grouped kernel per graph replay
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": (bytes_min * ratio) if ratio else None,
                     "traffic_source": "measured DRAM/algorithmic ratio of the kernel (profiles/traffic.json) x "
                                       "this batch's algorithmic bytes" if ratio else None,
                     "peak_kind": f"{peak_kind} HBM copy bandwidth",
                     "work_per_launch": f"sum over problems of A + Omega + Y = {bytes_min:.4e} bytes"},
        "clocks": clk.summary(),
        "error": ({"sample_rel_err_fp64": [e[0] for e in errs], "sample_sgemm_rel_err_fp64": [e[1] for e in errs],
                   "max_rel_err_fp64": max(e[0] for e in errs),
                   "max_ratio_to_sgemm": max(e[0] / e[1] for e in errs)} if errs else {}),
    }


# ---------------------------------------------------------------- served stream
def make_sketch_pools(wl, dev, seed):
    """One device-resident A per n: m_max x k_max column-major (lda = m_max), rank n with
    sigma_j = j^-2, plus N(0, 1e-6) noise. A request's A is an m x k window of the pool of
    its n (a window of a rank-n matrix has rank <= n), so the stream needs no per-request
    generation; each request is still charged its own A bytes by the server's admission."""
    import numpy as np
    import torch

    M, Kx = wl["m_max"], wl["k_max"]
    pools = {}
    torch.backends.cuda.matmul.allow_tf32 = False
    for n in wl["ns"]:
        g = torch.Generator(device=dev)
        g.manual_seed(seed * 1000 + n)
        U = torch.randn(M, n, device=dev, generator=g) / np.sqrt(M)
        V = torch.randn(Kx, n, device=dev, generator=g) / np.sqrt(Kx)
        sig = torch.arange(1, n + 1, device=dev, dtype=torch.float32).pow(-2.0)
        T = torch.empty(Kx, M, device=dev)  # row j of T = column j of A
        torch.matmul(V * sig, U.T, out=T)
        for c in range(0, Kx, 1024):
            T[c:c + 1024].add_(torch.randn(min(1024, Kx - c), M, device=dev, generator=g), alpha=1e-3)
        del U, V
        pools[n] = T
    torch.cuda.synchronize(dev)
    return pools


def request_shapes(wl, seed, count):
    """Seeded request shapes and A window origins: (m, n, k, r0, c0, omega seed)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    M, Kx = wl["m_max"], wl["k_max"]
    out = []
    for i in range(count):
        m = int(np.exp(rng.uniform(np.log(wl["m_min"]), np.log(M))))
        k = int(np.exp(rng.uniform(np.log(wl["k_min"]), np.log(Kx))))
        n = int(rng.choice(wl["ns"]))
        r0 = int(rng.integers(0, M - m + 1)) // 4 * 4  # 16-byte aligned window
        c0 = int(rng.integers(0, Kx - k + 1))
        out.append((m, n, k, r0, c0, seed * 1000003 + i))
    return out


def sketch_requests(wl, pools, seed, count):
    """Requests on the device pools: (m, n, k, A address, lda, omega seed)."""
    M = wl["m_max"]
    return [(m, n, k, pools[n].data_ptr() + 4 * (r0 + c0 * M), M, sd)
            for (m, n, k, r0, c0, sd) in request_shapes(wl, seed, count)]


def served_e2e(wl, ctx, pools, sample, draws, tc):
    """Served sketches end to end from host memory: per request, A (m x k, compact, page-locked)
    is copied up, the request is served, and Y (m x draws n) is copied back to page-locked host
    memory. Two device slots for A let request j + 1's upload run while request j is served.
    Wall-clock timed from the first upload to the last download."""
    import torch
    from cuda.bindings import runtime as rt

    from shgemm_b200 import server as srv

    dev = ctx.dev
    M, Kx = wl["m_max"], wl["k_max"]
    hpool = torch.empty(M * Kx, dtype=torch.float32, pin_memory=True)  # host copy of a rank-256 pool
    hpool.copy_(pools[wl["ns"][-1]].reshape(-1))
    amax = max(((m + 3) // 4 * 4) * k for (m, _, k, _, _, _) in sample)
    ymax = max(m * n * draws for (m, n, _, _, _, _) in sample)
    dA = [torch.empty(amax, device=dev) for _ in range(2)]
    hY = torch.empty(ymax, dtype=torch.float32, pin_memory=True)
    cs = torch.cuda.Stream(dev)
    srv_e = srv.SketchServer(ctx.local, hbm_budget_bytes=wl["budget"], compute_type=tc, streams=2, auto_release=False)
    d2h_kind = rt.cudaMemcpyKind.cudaMemcpyDeviceToHost
    pending = {}
    h2d = d2h = 0
    flops = 0.0

    def finish(j):
        t, nbytes = pending.pop(j)
        srv_e.wait(t)
        _, y, _, _ = srv_e.poll(t)
        (err,) = rt.cudaMemcpyAsync(hY.data_ptr(), y, nbytes, d2h_kind, cs.cuda_stream)
        if int(err) != 0:
            raise RuntimeError(f"device-to-host copy of Y failed: {err}")
        cs.synchronize()
        srv_e.release(t)
        return nbytes

    # one untimed request through the same path
    m, n, k, _, _, sd = sample[0]
    lda_d = (m + 3) // 4 * 4
    dA[0][:lda_d * k].copy_(hpool[:lda_d * k])
    pending[-1] = (srv_e.submit(m, n, k, dA[0], lda_d, draws=draws, seed=sd), 4 * m * n * draws)
    finish(-1)
    torch.cuda.synchronize(dev)
    ctx.barrier()
    w0 = time.perf_counter()
    for j, (m, n, k, _, _, sd) in enumerate(sample):
        if j >= 2:
            d2h += finish(j - 2)  # frees slot j % 2
        lda_d = (m + 3) // 4 * 4
        with torch.cuda.stream(cs):
            dA[j % 2][:lda_d * k].copy_(hpool[:lda_d * k], non_blocking=True)
        cs.synchronize()
        h2d += 4 * lda_d * k
        pending[j] = (srv_e.submit(m, n, k, dA[j % 2], lda_d, draws=draws, seed=sd), 4 * m * n * draws)
        flops += 2.0 * m * n * draws * k
    for j in sorted(pending):
        d2h += finish(j)
    wall = ctx.reduce(time.perf_counter() - w0)
    srv_e.close()
    del hpool, dA, hY
    return {"value": ctx.reduce(flops, "sum") / wall / 1e12, "unit": "TFLOP/s",
            "h2d_bytes_per_step": int(h2d / len(sample)), "d2h_bytes_per_step": int(d2h / len(sample)),
            "steps": len(sample), "seconds": wall,
            "path": "per request: A page-locked host -> device (cudaMemcpyAsync), shgemm_b200_server_submit/wait, "
                    "Y device -> page-locked host; one step = one request, wall clock"}


def served_case(args, wl, ctx):
    """Poisson stream into the sketch server; the same requests as plain per-call shgemm
    launches and as a saturating burst; a host-resident end-to-end leg; errors."""
    import numpy as np
    import torch

    import shgemm_b200 as sg
    from shgemm_b200 import evaluation as ev
    from shgemm_b200 import server as srv

    dev = ctx.dev
    rate = args.rate or wl["rate"]
    duration = args.duration or wl["duration"]
    draws, tc = wl["draws"], wl["tc"]
    pools = make_sketch_pools(wl, dev, seed=ctx.rank)
    reqs = sketch_requests(wl, pools, seed=ctx.rank, count=int(rate * duration * 1.5) + 64)

    server = srv.SketchServer(ctx.local, hbm_budget_bytes=wl["budget"], compute_type=tc, streams=args.server_streams,
                              auto_release=True)
    # warm-up: a few short bursts through the same server (kernels, arena, streams)
    warm = sketch_requests(wl, pools, seed=10_000 + ctx.rank, count=8 * args.warmup)
    for (m, n, k, a, lda, sd) in warm:
        server.submit(m, n, k, a, lda, draws=draws, seed=sd)
    server.drain()
    server.reset_stats()
    ctx.barrier()

    arrival = np.random.default_rng(20_000 + ctx.rank)
    with ClockSampler(ctx.local) as clk:
        t0 = time.perf_counter()
        due, i = 0.0, 0
        while i < len(reqs):
            due += arrival.exponential(1.0 / rate)
            if due > duration:
                break
            while time.perf_counter() - t0 < due:
                pass
            m, n, k, a, lda, sd = reqs[i]
            server.submit(m, n, k, a, lda, draws=draws, seed=sd)
            i += 1
        submitted_s = time.perf_counter() - t0
        server.drain(timeout_ms=1e6)
    st = server.stats()
    done = reqs[:i]  # every request submitted in the stream (all completed unless st["failed"])
    offered = sum(2.0 * m * n * draws * k for (m, n, k, _, _, _) in done) / duration / 1e12
    span = ctx.reduce(st["span_s"])
    flops = ctx.reduce(st["flops_completed"], "sum")
    value = flops / span / 1e12

    # saturation: the same requests submitted at once, admitted as the budget frees up
    server.reset_stats()
    for (m, n, k, a, lda, sd) in done:
        server.submit(m, n, k, a, lda, draws=draws, seed=sd)
    server.drain(timeout_ms=1e6)
    sat = server.stats()
    server.close()
    capacity = ctx.reduce(sat["flops_completed"], "sum") / ctx.reduce(sat["span_s"]) / 1e12

    # per-call baselines on the same requests: each request's Omega draws generated, then
    # (a) one plain shgemm call per draw, (b) one call over the draws side by side
    h = sg.Handle(ctx.local)
    stream = torch.cuda.Stream(dev)
    h.set_stream(stream)
    h.set_workspace_size(256 << 20)  # room for the widened B of the TF32 route at n = 4 x 256
    ldb_max = max((k + 7) // 8 * 8 for (_, _, k, _, _, _) in done)
    n_max = max(n for (_, n, _, _, _, _) in done)
    om = torch.empty(n_max * draws * ldb_max, device=dev, dtype=torch.float16)
    Y = torch.empty(max(m * n for (m, n, _, _, _, _) in done) * draws, device=dev)
    om_addr, y_addr = om.data_ptr(), Y.data_ptr()

    def gen(k, n, sd, ldb):
        for j in range(draws):
            srv.generate_omega(om_addr + 2 * j * n * ldb, ldb, k, n, srv.GAUSSIAN, srv.draw_seed(sd, j), n ** -0.5,
                               stream=stream)

    def per_draw(rs):
        for (m, n, k, a, lda, sd) in rs:
            ldb = (k + 7) // 8 * 8
            gen(k, n, sd, ldb)
            for j in range(draws):
                sg.shgemm(h, 0, 0, m, n, k, 1.0, a, lda, om_addr + 2 * j * n * ldb, ldb, 0.0,
                          y_addr + 4 * j * m * n, m, tc)

    def per_request(rs):
        for (m, n, k, a, lda, sd) in rs:
            ldb = (k + 7) // 8 * 8
            gen(k, n, sd, ldb)
            sg.shgemm(h, 0, 0, m, n * draws, k, 1.0, a, lda, om_addr, ldb, 0.0, y_addr, m, tc)

    pc = {}
    for name, fn in (("per_draw", per_draw), ("per_request", per_request)):
        with torch.cuda.stream(stream):
            fn(done[:8])
            stream.synchronize()
            p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            p0.record(stream)
            fn(done)
            p1.record(stream)
        torch.cuda.synchronize(dev)
        pc_ms = ctx.reduce(p0.elapsed_time(p1))
        pc_flops = ctx.reduce(sum(2.0 * m * n * draws * k for (m, n, k, _, _, _) in done), "sum")
        pc[name] = {"value": pc_flops / (pc_ms * 1e-3) / 1e12, "unit": "TFLOP/s", "seconds": pc_ms * 1e-3,
                    "requests": len(done)}
    pc["per_draw"]["what"] = ("the stream's requests as plain shgemm calls back to back on one stream: each "
                              "request's Omega draws generated on the device, then one call per draw")
    pc["per_request"]["what"] = ("the same requests, one plain shgemm call per request over its draws side by "
                                 "side (n = 4 x n_i columns)")
    assert h.check_error() == 0

    # error of a few served results against the FP64 product (results kept: no auto-release)
    errs = []
    if not args.no_error:
        chk = srv.SketchServer(ctx.local, hbm_budget_bytes=8 << 30, compute_type=tc, auto_release=False)
        small = [r for r in done if r[0] * r[2] <= (1 << 26)][:4]
        for (m, n, k, a, lda, sd) in small:
            ldb = (k + 7) // 8 * 8
            with torch.cuda.stream(stream):
                gen(k, n, sd, ldb)
            t = chk.submit(m, n, k, a, lda, draws=draws, seed=sd)
            chk.wait(t)
            _, y, ldy, _ = chk.poll(t)
            torch.cuda.synchronize(dev)
            for j in range(draws):
                c64 = ev.fp64_product(h, 0, 0, m, n, k, a, lda, om_addr + 2 * j * n * ldb, ldb)
                e_s = ev.error(h, m, n, y + 4 * j * m * n, m, c64)["rel_fro"]
                # plain FP32 SGEMM of the same operands (torch, no TF32)
                Af = torch.as_strided(pools[n], (m, k), (1, lda), (a - pools[n].data_ptr()) // 4)
                Bf = torch.as_strided(om, (k, n), (1, ldb), j * n * ldb).float()
                S = (Af @ Bf).T.contiguous().reshape(-1)
                torch.cuda.synchronize(dev)  # S comes from torch's stream, the error kernel runs on the handle's
                errs.append((e_s, ev.error(h, m, n, S, m, c64)["rel_fro"]))
            chk.release(t)
        chk.close()
    h.close()
    del om, Y

    # end to end with host-resident A: each request's A (compact, page-locked) goes up, the
    # server sketches it, and Y comes back; the next request's upload overlaps the current
    # request's GPU work (two device slots for A)
    e2e = None
    if not args.no_e2e:
        e2e = served_e2e(wl, ctx, pools, done[:64], draws, tc)
    del pools
    torch.cuda.empty_cache()

    peak, label = tensor_peak(True, tc)
    busy = ctx.reduce(st["kernel_busy_s"])
    issued = 2.0 * flops  # two MMAs per (i, j, k): hi and lo
    kernel_tflops = issued / busy / 1e12 if busy > 0 else None
    return {
        "value": value, "span_s": span, "completed": st["completed"], "failed": st["failed"],
        "requests": i, "rate": rate, "duration": duration, "submit_s": submitted_s, "offered_tflops": offered,
        "stats": st, "saturation": {"value": capacity, "unit": "TFLOP/s", "span_s": sat["span_s"],
                                    "p50_ms": sat["p50_ms"], "p99_ms": sat["p99_ms"], "batches": sat["batches"],
                                    "what": "the stream's requests submitted at once, admitted as the budget frees"},
        "per_call": pc,
        "roofline": {"bound": "tensor", "achieved": kernel_tflops, "peak": peak, "unit": "TFLOP/s",
                     "frac": (kernel_tflops / peak) if kernel_tflops else None,
                     "traffic": traffic_for("served_grouped_tf32"), "peak_kind": label,
                     "kernel": "shgemm_grouped_kernel<TF32, 256, op_n, K-major B, widened B>",
                     "work_per_launch": "issued 4 m (draws n) k of each batch's requests (hi and lo MMAs), "
                                        "over the device time during which a grouped launch ran (CUDA events on "
                                        "the server's streams, union of the launches' intervals)",
                     "kernel_busy_s": busy, "omega_s": st["omega_s"]},
        "clocks": clk.summary(), "gpu_launches": int(st["launches"]),
        "error": ({"sample_rel_err_fp64": [e[0] for e in errs], "sample_sgemm_rel_err_fp64": [e[1] for e in errs],
                   "max_rel_err_fp64": max(e[0] for e in errs),
                   "max_ratio_to_sgemm": max(e[0] / e[1] for e in errs)} if errs else {}),
        "e2e": e2e,
    }


# ---------------------------------------------------------------- CPU baseline and reference arm
def max_over_ranks(ms: float, dist, device) -> float:
    """Length of a timed region as the maximum over ranks (each rank timed its own device)."""
    if dist is None:
        return ms
    import torch

    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_tflops(world: int, flops_per_rank: float, ms: float) -> float:
    """Whole-job TFLOP/s: every replica's work over the slowest rank's time."""
    return world * flops_per_rank / (ms * 1e-3) / 1e12


CPU_REQUEST_FLOPS_CAP = 6e10  # a request of the CPU sample: at most this many 2mnk flops (all draws)


def cpu_sample(wl, count):
    """Requests of the served stream (seed 0, in arrival order) small enough for the host
    cores: the first `count` whose four draws total at most CPU_REQUEST_FLOPS_CAP flops.
    Returns (m, n, k, seed) tuples."""
    out = []
    for (m, n, k, _, _, sd) in request_shapes(wl, 0, 100000):
        if 2.0 * m * n * wl["draws"] * k <= CPU_REQUEST_FLOPS_CAP:
            out.append((m, n, k, sd))
            if len(out) == count:
                break
    return out


def cpu_request_inputs(wl, m, n, k, sd):
    """Host inputs of one sampled request: A (m x k, column-major) of rank n with sigma_j = j^-2
    plus noise, and its draws of Gaussian Omega (k x draws n, binary16, N(0, 1/n))."""
    import numpy as np

    rng = np.random.default_rng(sd)
    U = rng.standard_normal((m, n)).astype(np.float32) / np.sqrt(m)
    V = rng.standard_normal((k, n)).astype(np.float32) / np.sqrt(k)
    sig = np.arange(1, n + 1, dtype=np.float32) ** -2.0
    A = ((U * sig) @ V.T).astype(np.float32)  # m x k
    A += 1e-3 * rng.standard_normal((m, k)).astype(np.float32)
    A_cm = np.asfortranarray(A).ravel(order="F")
    B = (rng.standard_normal((wl["draws"] * n, k)) / np.sqrt(n)).astype(np.float16)  # rows = columns of Omega
    return A_cm, B.ravel()  # B: k x (draws n) column-major, ld = k


def cpu_baseline(wl, count=3):
    """The restated reference SHGEMM (oracle port, OpenMP) on a bounded sample of the served
    workload -- whole requests of the stream, their draws side by side -- plus a plain
    OpenMP FP64 and FP32 GEMM of the same shapes, on the host cores."""
    import numpy as np

    import oracle

    sample = cpu_sample(wl, count)
    t_port = t64 = t32 = 0.0
    flops = 0.0
    for (m, n, k, sd) in sample:
        A, B = cpu_request_inputs(wl, m, n, k, sd)
        cols = n * wl["draws"]
        C = np.zeros(m * cols, np.float32)
        t0 = time.perf_counter()
        oracle.shgemm(wl["tc"], 0, 0, m, cols, k, 1.0, A, m, B, k, 0.0, C, m, 0, 0)
        t_port += time.perf_counter() - t0
        Bf = B.astype(np.float64)
        t0 = time.perf_counter()
        oracle.cpu_gemm(A.astype(np.float64), Bf, m, cols, k, np.float64)
        t64 += time.perf_counter() - t0
        t0 = time.perf_counter()
        oracle.cpu_gemm(A, Bf.astype(np.float32), m, cols, k, np.float32)
        t32 += time.perf_counter() - t0
        flops += 2.0 * m * cols * k
    desc = (f"{len(sample)} requests of the served stream (seed 0, the first with <= {CPU_REQUEST_FLOPS_CAP:.0e} "
            f"flops: (m, n, k) = {[(m, n, k) for (m, n, k, _) in sample]}), 4 draws side by side, "
            f"{flops:.3e} flops (2mnk)")
    return {"value": flops / t_port / 1e12, "unit": "TFLOP/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": "restated reference SHGEMM (oracle port, TF32 split, OpenMP) on " + desc,
            "seconds": t_port,
            "openmp_fp64_gemm": {"value": flops / t64 / 1e12, "unit": "TFLOP/s", "seconds": t64},
            "openmp_fp32_gemm": {"value": flops / t32 / 1e12, "unit": "TFLOP/s", "seconds": t32}}


def cpu_baseline_plain(wl, seconds_target=12.0):
    """The oracle's restated SHGEMM (C, OpenMP) on a bounded square sample of a plain workload."""
    import numpy as np

    import oracle

    rng = np.random.default_rng(0)
    k = min(wl["k"] or 4096, 16384)
    ms = ns = 256
    while True:  # grow the sample until it takes a few seconds
        A = rng.standard_normal(ms * k).astype(np.float32)
        B = rng.standard_normal(k * ns).astype(np.float16)
        C = np.zeros(ms * ns, np.float32)
        t0 = time.perf_counter()
        oracle.shgemm(wl["tc"], 0, 0, ms, ns, k, 1.0, A, ms, B, k, 0.0, C, ms, 0, 0)
        dt = time.perf_counter() - t0
        if dt > seconds_target / 4 or ms >= 4096:
            break
        ms *= 2
        ns *= 2
    return {"value": 2.0 * ms * ns * k / dt / 1e12, "unit": "TFLOP/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": f"restated reference SHGEMM (oracle, fp64 fragment sums) {ms}x{ns}x{k}, {dt:.2f} s, "
                      "2mnk effective flops"}


def run_reference_arm(args, wl):
    """--impl reference: the reference's algorithm on the host cores, through the oracle port
    (the reference itself cannot be built: its arithmetic submodule is not vendored). Served
    workloads: each step is one request of the CPU sample (cpu_baseline's requests, cycled);
    plain workloads: a 512 x 512 x k sample per step. Rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import numpy as np

    import oracle

    served = wl["dist"] in ("served", "headline")
    if served:
        sample = cpu_sample(wl, 3)
        inputs = [cpu_request_inputs(wl, m, n, k, sd) for (m, n, k, sd) in sample]
        shapes = [(m, n * wl["draws"], k) for (m, n, k, _) in sample]
        desc = (f"one request of the served stream per step, cycling over the CPU sample's {len(sample)} "
                f"(m, 4n, k) = {shapes} (restated reference SHGEMM, TF32 split, OpenMP)")
    else:
        rng = np.random.default_rng(0)
        k = min(wl["k"] or 4096, 16384)
        inputs = [(rng.standard_normal(512 * k).astype(np.float32), rng.standard_normal(k * 512).astype(np.float16))]
        shapes = [(512, 512, k)]
        desc = f"512x512x{k} per step (restated reference SHGEMM, OpenMP, the workload's k)"

    def step(i):
        (A, B), (m, n, k) = inputs[i % len(inputs)], shapes[i % len(shapes)]
        C = np.zeros(m * n, np.float32)
        oracle.shgemm(wl["tc"], 0, 0, m, n, k, 1.0, A, m, B, k, 0.0, C, m, 0, 0)
        return 2.0 * m * n * k

    for i in range(args.warmup):
        step(i)
    flops, t = 0.0, 0.0
    for i in range(args.steps):
        t0 = time.perf_counter()
        flops += step(i)
        t += time.perf_counter() - t0
    value = flops / t / 1e12
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 split to fp16/tf32", "data": "synthetic",
            "config": {"workload": wl["desc"], "sample": desc},
            "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": oracle.num_threads(), "kind": "port",
                             "sample": desc},
            "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "same_sample_as_cpu_baseline": served,
            "note": "reference not buildable (wmma_extension/cutf submodules absent); its algorithm is timed "
                    "through the oracle port"}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- JSON lines
def dtype_of(tc):
    return "f32 split to tf32 (tensor) / f32 accumulate" if tc else "f32 split to fp16 (tensor) / f32 accumulate"


def served_line(args, wl, ctx, s, cpu):
    """The JSON line of the served stream (the headline's top level)."""
    pc = s["per_call"]
    st = s["stats"]
    return {
        "metric": METRIC, "value": s["value"], "unit": "TFLOP/s", "n_gpus": ctx.world, "steps": int(s["completed"]),
        "warmup": args.warmup, "ms_per_step": 1e3 * s["span_s"] / max(1, s["completed"]), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": dtype_of(wl["tc"]),
        "data": "synthetic (seeded; A windows of device-resident low-rank pools, Omega generated on the device "
                "per request)",
        "config": {"workload": wl["desc"], "rate_req_s": s["rate"], "duration_s": s["duration"],
                   "requests": s["requests"], "draws": wl["draws"], "budget_bytes": wl["budget"], "streams": 2,
                   "step": "one served request (ms_per_step = stream span / requests completed)",
                   "timing": "host clock: first submit to the last completion seen by the server; kernel time by "
                             "CUDA events on the server's streams",
                   "l2": "operands exceed L2 (a request's A averages ~0.3 GB; no flush needed)",
                   "parallelism": f"replicas x{ctx.world}"},
        "served": {"p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"], "max_ms": st["max_ms"],
                   "completed": st["completed"], "failed": st["failed"], "batches": st["batches"],
                   "span_s": s["span_s"], "submit_s": s["submit_s"], "offered_tflops": s["offered_tflops"],
                   "peak_resident_bytes": st["peak_resident_bytes"], "saturation": s["saturation"]},
        "per_call_baseline": pc["per_draw"],
        "per_call_baseline_per_request": pc["per_request"],
        "speedup_vs_per_call": s["value"] / pc["per_draw"]["value"],
        "speedup_vs_per_call_per_request": s["value"] / pc["per_request"]["value"],
        "saturation_speedup_vs_per_call": s["saturation"]["value"] / pc["per_draw"]["value"],
        "saturation_speedup_vs_per_call_per_request": s["saturation"]["value"] / pc["per_request"]["value"],
        "speedup_note": ("the stream is arrival-bound (served = offered load while the server keeps up), and the "
                         "per-call loops run the same requests back to back: the stream ratios set an arrival "
                         "rate against a capacity; the saturation ratios compare capacities"),
        "issued_tflops": 2 * s["value"],
        "gpu_launches": s["gpu_launches"],
        "roofline": s["roofline"],
        "clocks": s["clocks"],
        "error": s["error"],
        "e2e": s["e2e"],
        "cpu_baseline": cpu,
    }


def plain_line(args, wl, ctx, r, cpu):
    m, n, k = wl["m"], wl["n"], wl["k"]
    op_c = wl.get("op_c", 0)
    return {
        "metric": METRIC, "value": r["value"], "unit": "TFLOP/s", "n_gpus": ctx.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": dtype_of(wl["tc"]),
        "data": "synthetic (seeded, workload's shapes and distributions)",
        "config": {"workload": wl["desc"], "m": m, "n": n, "k": k, "op_a": "NT"[wl["op_a"]],
                   "op_b": "NT"[wl["op_b"]], "op_c": "NT"[op_c], "compute_type": ["fp16", "tf32"][wl["tc"]],
                   "kernel_level": r["level"], "autotuned": r["tuned"], "k_chunk": args.k_chunk,
                   "l2": "inputs exceed L2 (no flush needed)", "parallelism": f"replicas x{ctx.world}"},
        "issued_tflops": r["issued_tflops"], "gpu_launches": r["gpu_launches"], "roofline": r["roofline"],
        "clocks": r["clocks"], "energy": r["energy"], "error": r["error"], "tf32": r["tf32"], "e2e": r["e2e"],
        "cpu_baseline": cpu,
    }


def nested_square(wl, r):
    """The large square SHGEMM as nested in the headline line."""
    return {"workload": wl["desc"], "value": r["value"], "unit": "TFLOP/s", "ms_per_call": r["ms_per_step"],
            "calls": r["steps"], "issued_tflops": r["issued_tflops"], "kernel_level": r["level"],
            "autotuned": r["tuned"], "gpu_launches": r["gpu_launches"], "roofline": r["roofline"],
            "clocks": r["clocks"], "energy": r["energy"], "error_fp16": r["error"], "tf32": r["tf32"],
            "e2e": r["e2e"]}


# ---------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="headline", choices=sorted(WORKLOADS))
    ap.add_argument("--tc", default=None, choices=["fp16", "tf32"])
    ap.add_argument("--no-error", action="store_true", help="skip the FP64 error measurement")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end measurement")
    ap.add_argument("--no-autotune", action="store_true", help="plain workloads: use the heuristic plan")
    ap.add_argument("--count", type=int, default=0,
                    help="grouped workloads: a batch of COUNT problems from the same distributions (a smaller profiling case)")
    ap.add_argument("--no-nested", action="store_true", help="headline: skip the grouped and square results")
    ap.add_argument("--k-chunk", type=int, default=64, choices=[64, 128],
                    help="k between FP32 drains in the tensor-memory kernel (SHGEMM_CFG_K_CHUNK)")
    ap.add_argument("--group-m", type=int, default=0,
                    help="plain workloads: tile rasterisation group along m (with --no-autotune)")
    ap.add_argument("--stages", type=int, default=0, choices=[0, 1],
                    help="tensor-memory kernel operand ring (SHGEMM_CFG_TM_STAGES, with --no-autotune)")
    ap.add_argument("--pair", type=int, default=0, choices=[0, 1],
                    help="tensor-memory kernel in CTA pairs (SHGEMM_CFG_PAIR_TILES, with --no-autotune)")
    ap.add_argument("--rate", type=float, default=None, help="served: arrivals per second")
    ap.add_argument("--duration", type=float, default=None, help="served: seconds of arrivals")
    ap.add_argument("--server-streams", type=int, default=3, help="served: the sketch server's streams (slots)")
    args = ap.parse_args()
    wl = dict(WORKLOADS[args.workload])
    if args.tc:
        wl["tc"] = 0 if args.tc == "fp16" else 1
        wl["desc"] = wl["desc"].replace("fp16 compute", f"{args.tc} compute").replace("tf32 compute",
                                                                                       f"{args.tc} compute")
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return run_reference_arm(args, wl)

    ctx = Ctx()
    if wl["dist"] in ("served", "headline"):
        s = served_case(args, wl, ctx)
        nested = {}
        if wl["dist"] == "headline" and not args.no_nested:
            gw = WORKLOADS["grouped"]
            g = grouped_case(args, gw, ctx)
            nested["grouped"] = g
            gf = grouped_case(args, WORKLOADS["grouped_fused"], ctx)
            nested["grouped_fused_omega"] = {key: gf[key] for key in (
                "value", "unit", "ms_per_step", "workload", "algorithmic_bytes", "per_call_baseline",
                "speedup_vs_per_call", "roofline", "error", "autotuned_tile_n")}
            sw = WORKLOADS["square16k"]
            sq = square_case(args, sw, ctx, "square16k", tf32_error=True)
            nested["square16k"] = nested_square(sw, sq)
        cpu = cpu_baseline(wl) if ctx.rank == 0 and ctx.world == 1 and not args.no_cpu else None
        line = served_line(args, wl, ctx, s, cpu)
        line.update(nested)
    elif wl["dist"] == "energy":
        import shgemm_b200 as sg
        from shgemm_b200 import energy

        h = sg.Handle(ctx.local)
        rows = energy.power_sweep(h, seconds=args.duration or 10.0, device_index=ctx.local)
        h.close()
        top = [r for r in rows if r["m"] == 16384 and r["compute_type"] == "fp16"]
        line = {"metric": METRIC, "value": top[0]["tflops"] if top else None, "unit": "TFLOP/s",
                "n_gpus": ctx.world, "steps": sum(r["calls"] for r in rows), "warmup": 16, "ms_per_step": None,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype_of(0),
                "data": "synthetic (uniform (0, 1], seed 0)", "config": {"workload": wl["desc"]},
                "energy_table": rows}
    elif wl["dist"] == "grouped":
        g = grouped_case(args, wl, ctx)
        cpu = None
        if ctx.rank == 0 and ctx.world == 1 and not args.no_cpu:
            cpu = cpu_baseline_plain(dict(wl, k=4096))
        line = {"metric": METRIC, "value": g["value"], "unit": "TFLOP/s", "n_gpus": ctx.world, "steps": g["steps"],
                "warmup": args.warmup, "ms_per_step": g["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": dtype_of(wl["tc"]),
                "data": "synthetic (seeded, the batch's shapes and distributions)",
                "config": {"workload": wl["desc"], "problems": g["problems"], "total_flops_2mnk": g["total_flops_2mnk"],
                           "algorithmic_bytes": g["algorithmic_bytes"], "l2": "inputs exceed L2 (no flush needed)",
                           "parallelism": f"replicas x{ctx.world}"},
                "per_call_baseline": g["per_call_baseline"], "speedup_vs_per_call": g["speedup_vs_per_call"],
                "issued_tflops": g["issued_tflops"], "gpu_launches": g["gpu_launches"], "roofline": g["roofline"],
                "clocks": g["clocks"], "error": g["error"], "e2e": None, "cpu_baseline": cpu}
    else:
        r = square_case(args, wl, ctx, args.workload, tf32_error=args.workload == "square16k" and wl["tc"] == 0)
        cpu = cpu_baseline_plain(wl) if ctx.rank == 0 and ctx.world == 1 and not args.no_cpu else None
        line = plain_line(args, wl, ctx, r, cpu)
    if ctx.rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
