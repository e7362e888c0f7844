"""Benchmark of the SHGEMM hot path on B200.

Default workload: large square SHGEMM m = n = k = 16384, op_n/op_n, FP32 operand
N(0,1) * 2^U(-15,15), binary16 operand N(0,1), alpha = 1, beta = 0.5 with C
uniform[-1, 1], fp16 compute (seeded synthetic data of that shape and
distribution). One step = one SHGEMM call over the whole problem; inputs (1.5 GiB)
exceed the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload square16k|square1k|sketch]
    python bench.py --impl reference ...   # the reference algorithm on the host cores

Prints one JSON line (rank 0). Under torchrun (N > 1) every rank runs an
independent replica (the path has no cross-GPU exchange); time is the max over
ranks and `value` the aggregate.
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

WORKLOADS = {
    # the large square SHGEMM
    "square16k": dict(m=16384, n=16384, k=16384, op_a=0, op_b=0, tc=0, alpha=1.0, beta=0.5, dist="wide",
                      desc="large square SHGEMM 16384^3 NN, fp16 compute, A N(0,1)*2^U(-15,15), B N(0,1), beta=0.5"),
    # the same product with A transposed: the FP32 operand K-major (rows of k contiguous floats)
    "square16k_tn": dict(m=16384, n=16384, k=16384, op_a=1, op_b=0, tc=0, alpha=1.0, beta=0.5, dist="wide",
                         desc="large square SHGEMM 16384^3 TN, fp16 compute, A N(0,1)*2^U(-15,15), B N(0,1), "
                              "beta=0.5"),
    # a smaller square case of the same kernel, for profiler captures (inputs still exceed L2)
    "square8k": dict(m=8192, n=8192, k=8192, op_a=0, op_b=0, tc=0, alpha=1.0, beta=0.5, dist="wide",
                     desc="square SHGEMM 8192^3 NN, fp16 compute, A N(0,1)*2^U(-15,15), B N(0,1), beta=0.5"),
    # square8k with A transposed (K-major FP32 operand), for profiler captures of that load path
    "square8k_tn": dict(m=8192, n=8192, k=8192, op_a=1, op_b=0, tc=0, alpha=1.0, beta=0.5, dist="wide",
                        desc="square SHGEMM 8192^3 TN, fp16 compute, A N(0,1)*2^U(-15,15), B N(0,1), beta=0.5"),
    # a still smaller square case: with square8k it shows how DRAM traffic scales with the problem
    "square4k": dict(m=4096, n=4096, k=4096, op_a=0, op_b=0, tc=0, alpha=1.0, beta=0.5, dist="wide",
                     desc="square SHGEMM 4096^3 NN, fp16 compute, A N(0,1)*2^U(-15,15), B N(0,1), beta=0.5"),
    # small square SHGEMM
    "square1k": dict(m=1024, n=1024, k=1024, op_a=0, op_b=0, tc=0, alpha=1.0, beta=0.0, dist="uniform",
                     desc="plain SHGEMM 1024^3 NN, fp16 compute, A U[-1,1], B U[-1,1]"),
    # Y = Omega^T A as hsgemm(op_t, op_n) -> internal shgemm(op_t, op_n, 4096, 256, 2^20, op_c = t)
    "sketch": dict(m=4096, n=256, k=1 << 20, op_a=1, op_b=0, tc=0, alpha=1.0, beta=0.0, dist="sketch",
                   desc="left sketch Y = Omega^T A, A 2^20 x 4096 FP32 (low rank + noise), Omega 2^20 x 256 "
                        "binary16 N(0,1/256), split-K, fp16 compute", op_c=1, bound="hbm"),
    # the sketch at 1/8 of its length (A 2 GiB, still 16x L2), for profiler captures
    "sketch128k": dict(m=4096, n=256, k=1 << 17, op_a=1, op_b=0, tc=0, alpha=1.0, beta=0.0, dist="sketch",
                       op_c=1, desc="left sketch Y = Omega^T A, A 2^17 x 4096 FP32 (low rank + noise), "
                                    "Omega 2^17 x 256 binary16", bound="hbm"),
    # 512 uneven right sketches in one graph-captured grouped launch
    "grouped": dict(m=0, n=0, k=0, op_a=0, op_b=0, tc=0, alpha=1.0, beta=0.0, dist="grouped", count=512, bound="hbm",
                    desc="grouped batch of 512 uneven right sketches Y_i = A_i Omega_i, m_i log-U[64,8192], "
                         "k_i log-U[256,16384], n_i in {32,64,128,256}, A_i rank n_i/2 (sigma_j = j^-1.5) + N(0,1e-4), "
                         "Omega_i Rademacher/sqrt(n_i), fp16 compute, one CUDA-graph-captured launch"),
    # a Poisson stream of sketch requests into the sketch server
    "served": dict(m=0, n=0, k=0, op_a=0, op_b=0, tc=1, alpha=1.0, beta=0.0, dist="served", bound="tensor",
                   rate=2000.0, duration=60.0, budget=40 << 30, draws=4, m_min=1024, m_max=65536, k_min=1024,
                   k_max=16384, ns=(64, 128, 256),
                   desc="served sketch stream: Poisson arrivals at 2000 req/s, m log-U[1024,65536], "
                        "k log-U[1024,16384], n in {64,128,256}, 4 Gaussian Omega draws per resident A "
                        "(rank n, sigma_j = j^-2, + N(0,1e-6)), tf32 compute, 40 GB admission budget"),
    # the same batch in TF32 compute, Omega_i handed over widened to FP32 (as the sketch server keeps it)
    "grouped_tf32": dict(m=0, n=0, k=0, op_a=0, op_b=0, tc=1, alpha=1.0, beta=0.0, dist="grouped", count=512,
                         bound="hbm", b_fp32=True,
                         desc="grouped batch of 512 uneven right sketches (shapes as the fp16 batch), tf32 compute, "
                              "Omega_i widened to FP32 once, one CUDA-graph-captured launch"),
}


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


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


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


def make_inputs(wl, dev, seed=0):
    import torch

    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    m, n, k = wl["m"], wl["n"], wl["k"]
    a_rows = m if wl["op_a"] == 0 else k
    b_rows = k if wl["op_b"] == 0 else n
    na = m * k
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
    c_rows = m if op_c == 0 else n
    C = torch.empty(m * n, device=dev).uniform_(-1, 1, generator=g)
    return A, a_rows, B, b_rows, C, c_rows


def gpu_error(h, wl, A, lda, B, ldb, C_out, ldc, C0):
    """Relative Frobenius error vs the FP64 product (GPU), plus FP32 SGEMM's (torch, no TF32)."""
    import torch

    from shgemm_b200 import evaluation as ev

    m, n, k = wl["m"], wl["n"], wl["k"]
    op_c = wl.get("op_c", 0)
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
    es = ev.error(h, m, n, Sbuf, m if op_c == 0 else n, c64, wl["alpha"], wl["beta"],
                  C0 if wl["beta"] != 0 else None, op_c)
    # binary16 compute: an FP32 entry of magnitude >= 65520 rounds to inf in the hi part (as in
    # the reference), so every output of its row of op(A) is non-finite while FP64 stays finite
    expected = 0
    if wl["tc"] == 0:
        rows = (Am[:m, :k].abs() >= 65520.0).any(dim=1)
        expected = int(rows.sum().item()) * n
    del c64, S, Sbuf
    return {"rel_err_fp64": e["rel_fro"], "max_rel_err_fp64": e["max_rel"],
            "nonfinite_mismatch": e["nonfinite_mismatch"],
            "nonfinite_expected_fp16_overflow": expected,
            "note": "rel_err over entries finite in both; non-finite outputs come from binary16 "
                    "overflow of the FP32 operand (rows with |a| >= 65520), the reference's behaviour",
            "sgemm_rel_err_fp64": es["rel_fro"]}


def cpu_baseline(wl, seconds_target=12.0):
    """The oracle's restated SHGEMM (C, OpenMP) on a bounded sample of the workload."""
    import numpy as np

    import oracle

    rng = np.random.default_rng(0)
    k = min(wl["k"] or 4096, 16384)
    ms = ns = 256
    # grow the sample until it takes a few seconds
    while True:
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
    flops = 2.0 * ms * ns * k
    return {"value": flops / dt / 1e12, "unit": "TFLOP/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": f"restated reference SHGEMM (oracle, fp64 fragment sums) {ms}x{ns}x{k}, "
                      f"{dt:.2f} s, 2mnk effective flops"}


def run_reference_arm(args, wl):
    """--impl reference: the reference algorithm on the host cores (the reference itself
    cannot be built: its arithmetic submodule is not vendored), bounded sample per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import numpy as np

    import oracle

    rng = np.random.default_rng(0)
    k = min(wl["k"] or 4096, 16384)  # batch / stream workloads: a representative k
    ms = ns = 512
    A = rng.standard_normal(ms * k).astype(np.float32)
    B = rng.standard_normal(k * ns).astype(np.float16)
    C = np.zeros(ms * ns, np.float32)
    for _ in range(args.warmup):
        oracle.shgemm(wl["tc"], 0, 0, ms, ns, k, 1.0, A, ms, B, k, 0.0, C, ms, 0, 0)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.shgemm(wl["tc"], 0, 0, ms, ns, k, 1.0, A, ms, B, k, 0.0, C, ms, 0, 0)
        times.append(time.perf_counter() - t0)
    dt = sum(times)
    flops = 2.0 * ms * ns * k * args.steps
    value = flops / dt / 1e12
    sample = f"{ms}x{ns}x{k} per step (restated reference SHGEMM, OpenMP, the workload's k)"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 split to fp16/tf32", "data": "synthetic",
            "config": {"workload": wl["desc"], "sample": sample},
            "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": oracle.num_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference not buildable (wmma_extension/cutf submodules absent); its algorithm is timed "
                    "through the oracle port"}
    print(json.dumps(line), flush=True)
    return 0


def make_grouped_batch(count, dev, seed=0):
    """Config 4's uneven sketch batch on the device; returns problem tuples and sizes."""
    import numpy as np
    import torch

    rng = np.random.default_rng(seed)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    ms = np.exp(rng.uniform(np.log(64), np.log(8192), count)).astype(int)
    ks = np.exp(rng.uniform(np.log(256), np.log(16384), count)).astype(int)
    ns = rng.choice([32, 64, 128, 256], count)
    probs, shapes, keep = [], [], []
    for m, k, n in zip(ms, ks, ns):
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
        Om = torch.empty(n, ldb, device=dev, dtype=torch.float16)  # column-major k x n, ld = ldb
        Om[:, :k] = ((torch.randint(0, 2, (n, k), device=dev, generator=g) * 2 - 1).float() / np.sqrt(n)).half()
        Y = torch.zeros(n, m, device=dev)
        A = Afull.reshape(-1)
        B = Om.reshape(-1)
        C = Y.reshape(-1)
        keep.append((A, B, C))
        probs.append((m, n, k, A, lda, B, ldb, C, m, 1.0, 0.0))
        shapes.append((m, n, k))
    return probs, shapes, keep


def run_grouped(args, wl):
    import numpy as np
    import torch

    import shgemm_b200 as sg
    from shgemm_b200 import evaluation as ev

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    h = sg.Handle(local)
    stream = torch.cuda.Stream(dev)
    h.set_stream(stream)
    probs, shapes, keep = make_grouped_batch(wl["count"], dev, seed=rank)
    torch.cuda.synchronize(dev)
    flops = sum(2.0 * m * n * k for (m, n, k) in shapes)
    b_bytes = 4.0 if wl.get("b_fp32") else 2.0
    bytes_min = sum(4.0 * m * k + b_bytes * k * n + 4.0 * m * n for (m, n, k) in shapes)
    gprobs, keep_w = probs, []
    if wl.get("b_fp32"):
        # Omega_i widened to FP32 once (exact: binary16 values), K-major with a 16-byte ld
        gprobs = []
        for (m, n, k, A, lda, B, ldb, C, ldc, al, be) in probs:
            ldb4 = (k + 3) // 4 * 4
            Bw = torch.zeros(n, ldb4, device=dev)
            Bw[:, :k] = B.view(n, ldb)[:, :k].float()
            keep_w.append(Bw)
            gprobs.append((m, n, k, A, lda, Bw.reshape(-1), ldb4, C, ldc, al, be))
        h.set_config(sg.CFG_GROUPED_B_FP32, 1)

    # capture the grouped launch once, replay it per step
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
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk, torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            graph.replay()
        e1.record(stream)
        torch.cuda.synchronize(dev)
    # graph replays do not pass through the library's counter: one grouped kernel per replay
    launches = args.steps
    t = torch.tensor([e0.elapsed_time(e1)], device=dev, dtype=torch.float64)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_step = float(t.item()) / args.steps
    value = world * flops / (ms_step * 1e-3) / 1e12
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
        steps_pc = max(1, min(args.steps, 5))
        p0.record(stream)
        for _ in range(steps_pc):
            per_call()
        p1.record(stream)
    torch.cuda.synchronize(dev)
    ms_pc = p0.elapsed_time(p1) / steps_pc
    per_call_tflops = flops / (ms_pc * 1e-3) / 1e12

    # error on a sample of problems vs the FP64 product (outputs of a graph replay)
    for (_, _, C) in keep:
        C.zero_()
    with torch.cuda.stream(stream):
        graph.replay()
    torch.cuda.synchronize(dev)
    errs = []
    torch.backends.cuda.matmul.allow_tf32 = False
    with torch.cuda.stream(stream):  # the library's error kernels run on the handle's stream
        for i in range(0, len(probs), max(1, len(probs) // 16)):
            m, n, k, A, lda, B, ldb, C, ldc, al, be = probs[i]
            c64 = ev.fp64_product(h, 0, 0, m, n, k, A, lda, B, ldb)
            e_sh = ev.error(h, m, n, C, ldc, c64)["rel_fro"]
            Bf = B.view(n, ldb)[:, :k].float()
            Af = A.view(k, lda)[:, :m].T
            S = (Af @ Bf.T).T.contiguous().reshape(-1)  # n x m row-major == m x n column-major
            errs.append((e_sh, ev.error(h, m, n, S, m, c64)["rel_fro"]))
    torch.cuda.synchronize(dev)
    del graph

    peaks, peak_kind = load_peaks()
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = bytes_min / (ms_step * 1e-3) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(dict(wl, k=4096, tc=wl["tc"]))
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 split to fp16 (tensor) / f32 accumulate" if wl["tc"] == 0
            else "f32 split to tf32 (tensor) / f32 accumulate",
            "data": "synthetic (seeded, config 4 shapes and distributions)",
            "config": {"workload": wl["desc"], "problems": len(probs), "total_flops_2mnk": flops,
                       "algorithmic_bytes": bytes_min, "l2": "inputs exceed L2 (no flush needed)",
                       "parallelism": f"replicas x{world}"},
            "per_call_baseline": {"value": per_call_tflops, "unit": "TFLOP/s", "ms_per_step": ms_pc,
                                  "launches_per_step": len(probs),
                                  "what": "the same problems as one shgemm call (one launch) each"},
            "speedup_vs_per_call": value / world / per_call_tflops,
            "issued_tflops": 2 * value,
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_kind": f"{peak_kind} HBM copy bandwidth",
                         "work_per_launch": f"sum over problems of A + Omega + Y = {bytes_min:.4e} bytes"},
            "clocks": clk.summary(),
            "error": {"sample_rel_err_fp64": [e[0] for e in errs], "sample_sgemm_rel_err_fp64": [e[1] for e in errs],
                      "max_rel_err_fp64": max(e[0] for e in errs)},
            "e2e": None,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    h.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


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


def sketch_requests(wl, pools, seed, count):
    """Seeded request shapes and A windows: (m, n, k, A address, lda, omega seed)."""
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
        out.append((m, n, k, pools[n].data_ptr() + 4 * (r0 + c0 * M), M, seed * 1000003 + i))
    return out


def run_served(args, wl):
    import numpy as np
    import torch

    import shgemm_b200 as sg
    from shgemm_b200 import evaluation as ev
    from shgemm_b200 import server as srv

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    rate = args.rate or wl["rate"]
    duration = args.duration or wl["duration"]
    draws, tc = wl["draws"], wl["tc"]
    pools = make_sketch_pools(wl, dev, seed=rank)
    reqs = sketch_requests(wl, pools, seed=rank, count=int(rate * duration * 1.5) + 64)
    mean_flops = float(np.mean([2.0 * m * n * draws * k for (m, n, k, _, _, _) in reqs]))

    server = srv.SketchServer(local, hbm_budget_bytes=wl["budget"], compute_type=tc, streams=2, auto_release=True)
    # warm-up: a few short bursts through the same server (kernels, arena, streams)
    warm = sketch_requests(wl, pools, seed=10_000 + rank, count=8 * args.warmup)
    for (m, n, k, a, lda, sd) in warm:
        server.submit(m, n, k, a, lda, draws=draws, seed=sd)
    server.drain()
    server.reset_stats()
    if dist:
        dist.barrier()

    arrival = np.random.default_rng(20_000 + rank)
    with ClockSampler(local) as clk:
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
    server.close()
    offered = i * mean_flops / duration / 1e12
    span = st["span_s"]
    flops = st["flops_completed"]
    tt = torch.tensor([span, flops, st["p50_ms"], st["p99_ms"]], device=dev, dtype=torch.float64)
    if dist:
        spans = tt.clone()
        dist.all_reduce(spans, op=dist.ReduceOp.MAX)
        fl = tt.clone()
        dist.all_reduce(fl, op=dist.ReduceOp.SUM)
        span, flops = float(spans[0]), float(fl[1])
    value = flops / span / 1e12

    # per-call baseline: the same kind of requests as plain shgemm calls, one per Omega draw
    h = sg.Handle(local)
    stream = torch.cuda.Stream(dev)
    h.set_stream(stream)
    sample = reqs[:min(len(reqs), 64)]
    oms = []
    for (m, n, k, a, lda, sd) in sample:
        ldb = (k + 7) // 8 * 8
        om = torch.empty(n * draws * ldb, device=dev, dtype=torch.float16)
        for j in range(draws):
            srv.generate_omega(om[j * n * ldb:], ldb, k, n, srv.GAUSSIAN, srv.draw_seed(sd, j), n ** -0.5,
                               stream=stream)
        oms.append((om, ldb))
    ymax = max(m * n for (m, n, _, _, _, _) in sample)
    Y = torch.empty(ymax, device=dev)

    def per_call():
        for (m, n, k, a, lda, sd), (om, ldb) in zip(sample, oms):
            for j in range(draws):
                sg.shgemm(h, 0, 0, m, n, k, 1.0, a, lda, om[j * n * ldb:], ldb, 0.0, Y, m, tc)

    with torch.cuda.stream(stream):
        per_call()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        per_call()
        p1.record(stream)
    torch.cuda.synchronize(dev)
    pc_flops = sum(2.0 * m * n * draws * k for (m, n, k, _, _, _) in sample)
    per_call_tflops = pc_flops / (p0.elapsed_time(p1) * 1e-3) / 1e12

    # error of a few served results against the FP64 product (results kept: no auto-release)
    errs = []
    if not args.no_error:
        chk = srv.SketchServer(local, hbm_budget_bytes=8 << 30, compute_type=tc, auto_release=False)
        for (m, n, k, a, lda, sd), (om, ldb) in list(zip(sample, oms))[:4]:
            t = chk.submit(m, n, k, a, lda, draws=draws, seed=sd)
            chk.wait(t)
            _, y, ldy, _ = chk.poll(t)
            for j in range(draws):
                c64 = ev.fp64_product(h, 0, 0, m, n, k, a, lda, om[j * n * ldb:], ldb)
                errs.append(ev.error(h, m, n, y + 4 * j * m * n, m, c64)["rel_fro"])
            chk.release(t)
        chk.close()
    h.close()

    peaks, peak_kind = load_peaks()
    tf32_peak = peaks.get("bf16_tflops_sustained", 1376.1) / 2  # TF32 runs at half the 16-bit rate
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": int(st["completed"]),
            "warmup": args.warmup, "ms_per_step": 1e3 * span / max(1, st["completed"]), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 split to tf32 (tensor) / f32 accumulate" if tc else "f32 split to fp16 (tensor) / f32 accumulate",
            "data": "synthetic (seeded, config 5 shapes and distributions; A windows of device-resident "
                    "low-rank pools, Omega generated on the device per request)",
            "config": {"workload": wl["desc"], "rate_req_s": rate, "duration_s": duration, "requests": i,
                       "draws": draws, "budget_bytes": wl["budget"], "streams": 2,
                       "step": "one served request (ms_per_step = stream span / requests completed)",
                       "timing": "host clock: first submit to the last completion seen by the server",
                       "parallelism": f"replicas x{world}"},
            "served": {"p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"],
                       "max_ms": st["max_ms"], "completed": st["completed"], "failed": st["failed"],
                       "batches": st["batches"], "span_s": span, "submit_s": submitted_s,
                       "offered_tflops": offered, "peak_resident_bytes": st["peak_resident_bytes"]},
            "per_call_baseline": {"value": per_call_tflops, "unit": "TFLOP/s",
                                  "what": f"first {len(sample)} requests as plain shgemm calls, one per Omega draw, "
                                          "back to back on one stream"},
            "speedup_vs_per_call": value / world / per_call_tflops,
            "issued_tflops": 2 * value,
            # per batch: one grouped launch plus one Omega generation per draw of each request
            "gpu_launches": int(st["batches"]) + int(st["completed"]) * draws,
            "roofline": {"bound": "tensor", "achieved": 2 * value / world, "peak": tf32_peak if tc else
                         peaks.get("bf16_tflops_sustained", 1376.1), "unit": "TFLOP/s",
                         "frac": 2 * value / world / (tf32_peak if tc else peaks.get("bf16_tflops_sustained", 1376.1)),
                         "traffic": None,
                         "peak_kind": f"{peak_kind} sustained dense bf16 (halved for tf32)",
                         "work_per_launch": "issued 4mnk of the batch's requests"},
            "clocks": clk.summary(),
            "error": {"sample_rel_err_fp64": errs, "max_rel_err_fp64": max(errs) if errs else None},
            "e2e": None,
            "e2e_note": "requests reference device-resident A by design (the server keeps A, Omega and Y on "
                        "the device); no host copies are part of a request",
            "cpu_baseline": None,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="square16k", choices=sorted(WORKLOADS))
    ap.add_argument("--tc", default=None, choices=["fp16", "tf32"])
    ap.add_argument("--no-error", action="store_true", help="skip the FP64 error measurement")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end measurement")
    ap.add_argument("--no-autotune", action="store_true", help="plain workloads: use the heuristic plan")
    ap.add_argument("--k-chunk", type=int, default=64, choices=[64, 128],
                    help="k between FP32 drains in the tensor-memory kernel (SHGEMM_CFG_K_CHUNK)")
    ap.add_argument("--rate", type=float, default=None, help="served: arrivals per second")
    ap.add_argument("--duration", type=float, default=None, help="served: seconds of arrivals")
    args = ap.parse_args()
    wl = dict(WORKLOADS[args.workload])
    if args.tc:
        wl["tc"] = 0 if args.tc == "fp16" else 1
        wl["desc"] = wl["desc"].replace("fp16 compute", f"{args.tc} compute").replace("tf32 compute",
                                                                                       f"{args.tc} compute")
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return run_reference_arm(args, wl)
    if wl["dist"] == "grouped":
        return run_grouped(args, wl)
    if wl["dist"] == "served":
        return run_served(args, wl)

    import torch

    import shgemm_b200 as sg

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)

    h = sg.Handle(local)
    stream = torch.cuda.current_stream(dev)
    h.set_stream(stream)
    m, n, k = wl["m"], wl["n"], wl["k"]
    op_c = wl.get("op_c", 0)
    A, lda, B, ldb, C, ldc = make_inputs(wl, dev, seed=rank)
    C0 = C.clone() if wl["beta"] != 0 else None

    h.set_config(sg.CFG_K_CHUNK, args.k_chunk)
    if wl["tc"] == 1 and wl["op_b"] == 0:
        # room for the widened FP32 copy of B (the TF32 route that loads B unconverted)
        h.set_workspace_size(max(64 << 20, n * ((k + 3) // 4 * 4) * 4 + (1 << 20)))
    if wl["tc"] == 0 and wl["op_b"] == 0 and ldb * 2 >= (1 << 20):
        # room for B re-laid out as contiguous k-blocks (columns >= 1 MiB apart) plus the split-K partials
        h.set_workspace_size((64 << 20) + n * ((k + 63) // 64 * 64) * 2)
    # one-off autotune of the shape's bucket (not timed); C is overwritten by it, then restored
    tuned = None
    if not args.no_autotune and op_c == 0:
        tuned = h.autotune(wl["op_a"], wl["op_b"], m, n, k, A, lda, B, ldb, C, ldc, wl["tc"])
        if C0 is not None:
            C.copy_(C0)
        torch.cuda.synchronize(dev)

    def step():
        return sg.shgemm(h, wl["op_a"], wl["op_b"], m, n, k, wl["alpha"], A, lda, B, ldb, wl["beta"], C, ldc, wl["tc"],
                         op_c)

    for _ in range(args.warmup):
        level = step()
    torch.cuda.synchronize(dev)
    if h.check_error() != 0:
        raise RuntimeError("device-side timeout during warm-up")

    # ---- timed region: device events on the launching stream, barrier + sync on both sides
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    launches0 = h.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    launches = h.launch_count() - launches0
    if dist:
        dist.barrier()
    ms_total = max_over_ranks(ev0.elapsed_time(ev1), dist, dev)
    ms_step = ms_total / args.steps
    flops_eff = 2.0 * m * n * k
    flops_issued = 4.0 * m * n * k
    value = aggregate_tflops(world, flops_eff * args.steps, ms_total)
    if h.check_error() != 0:
        raise RuntimeError("device-side timeout in the timed region")

    # ---- error vs FP64 (outside the timed region; fresh C from the same C0)
    err = {}
    if not args.no_error:
        if C0 is not None:
            C.copy_(C0)
        step()
        torch.cuda.synchronize(dev)
        err = gpu_error(h, wl, A, lda, B, ldb, C, ldc, C0)

    # ---- end to end through the public API with host buffers (pinned), copies timed
    e2e = None
    if not args.no_e2e:
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
        if dist:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            e2e_step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        te = max_over_ranks(e0.elapsed_time(e1), dist, dev)
        e2e = {"value": aggregate_tflops(world, flops_eff * e2e_steps, te), "unit": "TFLOP/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
               "path": "shgemm_b200_shgemm_host on page-locked host buffers (copies overlapped with compute)"}
        sg.release_host_staging(h)
        del hA, hB, hC

    # ---- roofline of the tile kernel (its launches are the timed steps)
    peaks, peak_kind = load_peaks()
    bytes_min = 4.0 * m * k + 2.0 * k * n + 4.0 * m * n * (2 if wl["beta"] != 0 else 1)
    if wl.get("bound", "tensor") == "hbm":
        peak = peaks.get("hbm_gbs", 6650.0)
        achieved = bytes_min / (ms_step * 1e-3) / 1e9
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": None, "peak_kind": f"{peak_kind} HBM copy bandwidth",
                    "work_per_launch": f"A + B + C = {bytes_min:.4e} bytes (each operand read once)"}
    else:
        # burst peak for a short timed region, the power-capped sustained one for a long one;
        # TF32 MMAs run at half the 16-bit rate
        sustained = ms_total >= 100.0
        peak = peaks.get("bf16_tflops_sustained", 1400.0) if sustained else peaks.get("bf16_tflops", 1590.0)
        if wl["tc"]:
            peak /= 2
        achieved = flops_issued / (ms_step * 1e-3) / 1e12
        roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": None,
                    "peak_kind": f"{peak_kind} bf16 dense {'sustained' if sustained else 'burst'}"
                                 + (" / 2 (TF32 rate)" if wl["tc"] else ""),
                    "work_per_launch": f"4mnk = {flops_issued:.4e} issued tensor flops (two MMAs per k: hi and lo)"}
    traffic_file = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(traffic_file):
        with open(traffic_file) as f:
            tr = json.load(f).get(args.workload + ("_tf32" if wl["tc"] else ""))
        if tr:
            roofline["traffic"] = tr

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(wl)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 split to fp16 (tensor) / f32 accumulate" if wl["tc"] == 0
            else "f32 split to tf32 (tensor) / f32 accumulate",
            "data": "synthetic (seeded, workload's shapes and distributions)",
            "config": {"workload": wl["desc"], "m": m, "n": n, "k": k, "op_a": "NT"[wl["op_a"]],
                       "op_b": "NT"[wl["op_b"]], "op_c": "NT"[op_c], "compute_type": ["fp16", "tf32"][wl["tc"]],
                       "kernel_level": level, "autotuned": tuned, "k_chunk": args.k_chunk,
                       "l2": "inputs exceed L2 (no flush needed)",
                       "parallelism": f"replicas x{world}"},
            "issued_tflops": world * flops_issued * args.steps / (ms_total * 1e-3) / 1e12,
            "gpu_launches": launches,
            "roofline": roofline,
            "clocks": clk.summary(),
            "energy": energy(clk.summary(), ms_step, flops_eff),
            "error": err,
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    h.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
