"""Energy per SHGEMM call, measured the way the reference's power test does.

The reference samples the board power through NVML every 50 ms while a loop of about
10 s of identical shgemm calls runs, and reports throughput, average power and the
integrated energy per call, for square m = n = k = 2^10 .. 2^14, op_n/op_n, TF32 and
binary16 compute, inputs uniform (0, 1] (test/power_consumption_test.cu:55-123,
251-286; its sampler is the un-vendored gpu_monitor submodule). Here NVML is read
through pynvml: the board's energy counter (millijoules since the driver loaded) gives
the energy of the loop exactly, and the 50 ms power samples give the average power and
its spread. NVML is only read; no GPU setting is changed.
"""
from __future__ import annotations

import threading
import time


class PowerMonitor:
    """Samples one GPU's board power every `interval_ms` and reads its energy counter
    around a timed region. `nvml` is the pynvml module (injectable for tests)."""

    def __init__(self, device_index: int = 0, interval_ms: float = 50.0, nvml=None):
        if nvml is None:
            import pynvml as nvml
        self.nvml = nvml
        self.interval = interval_ms * 1e-3
        nvml.nvmlInit()
        self.handle = self._handle(device_index)
        self.samples = []  # (seconds since start, watts)
        self._stop = threading.Event()
        self._thread = None

    def _handle(self, device_index):
        """The NVML handle of the CUDA device (matched by UUID, then PCI bus id, when torch knows them)."""
        nv = self.nvml
        try:
            import torch

            props = torch.cuda.get_device_properties(device_index)
            uuid = getattr(props, "uuid", None)
            if uuid is not None:
                u = str(uuid)
                return nv.nvmlDeviceGetHandleByUUID(u if u.startswith("GPU-") else "GPU-" + u)
        except Exception:
            pass
        try:
            import torch

            props = torch.cuda.get_device_properties(device_index)
            bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(device_index)

    def _energy_mj(self):
        try:
            return float(self.nvml.nvmlDeviceGetTotalEnergyConsumption(self.handle))
        except Exception:
            return None

    def _run(self):
        t0 = self._t0
        while not self._stop.is_set():
            try:
                w = self.nvml.nvmlDeviceGetPowerUsage(self.handle) * 1e-3
                self.samples.append((time.perf_counter() - t0, w))
            except Exception:
                pass
            self._stop.wait(self.interval)

    def __enter__(self):
        self.samples = []
        self._stop.clear()
        self._t0 = time.perf_counter()
        self._e0 = self._energy_mj()
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        self._e1 = self._energy_mj()
        self.elapsed = time.perf_counter() - self._t0
        self._stop.set()
        self._thread.join(timeout=5)

    def result(self) -> dict:
        """Elapsed seconds, energy in joules (counter if available, else the integral of the
        samples by the trapezoid rule) and the average / peak sampled power."""
        s = self.samples
        integ = 0.0
        for (t0, w0), (t1, w1) in zip(s, s[1:]):
            integ += 0.5 * (w0 + w1) * (t1 - t0)
        if s:  # the samples cover [first, last]; extend the ends at their edge values
            integ += s[0][1] * s[0][0] + s[-1][1] * max(0.0, self.elapsed - s[-1][0])
        counter = None
        if self._e0 is not None and self._e1 is not None and self._e1 >= self._e0:
            counter = (self._e1 - self._e0) * 1e-3
        joules = counter if counter is not None else integ
        watts = [w for _, w in s]
        return {"seconds": self.elapsed, "joules": joules, "joules_sampled": integ,
                "source": "NVML energy counter" if counter is not None else "NVML power samples (trapezoid)",
                "avg_w": joules / self.elapsed if self.elapsed > 0 else None,
                "sampled_avg_w": sum(watts) / len(watts) if watts else None,
                "peak_w": max(watts) if watts else None, "samples": len(watts)}


def measure(call, count: int, device_index: int = 0, interval_ms: float = 50.0, sync=None, nvml=None) -> dict:
    """Runs `call()` `count` times under a PowerMonitor (synchronising with `sync()` on both
    sides) and returns the monitor's result plus joules per call."""
    mon = PowerMonitor(device_index, interval_ms, nvml=nvml)
    if sync:
        sync()
    with mon:
        for _ in range(count):
            call()
        if sync:
            sync()
    r = mon.result()
    r["calls"] = count
    r["joules_per_call"] = r["joules"] / count
    return r


def power_sweep(handle, log_sizes=range(10, 15), compute_types=(1, 0), seconds: float = 10.0, device_index: int = 0,
                seed: int = 0):
    """The reference's power test (test/power_consumption_test.cu:251-286) on this library:
    square SHGEMM op_n/op_n for m = n = k = 2^s, inputs uniform (0, 1] (B binary16),
    alpha = 1, beta = 0; a warm-up of 16 calls sizes a loop of about `seconds`, which runs
    under NVML. Returns one row per (size, compute type)."""
    import torch

    import shgemm_b200 as sg

    dev = torch.device(f"cuda:{device_index}")
    nmax = 1 << max(log_sizes)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    A = torch.rand(nmax * nmax, device=dev, generator=g)
    B = torch.rand(nmax * nmax, device=dev, generator=g).to(torch.float16)
    C = torch.empty(nmax * nmax, device=dev)
    rows = []
    for s in log_sizes:
        n = 1 << s
        for tc in compute_types:
            def call():
                return sg.shgemm(handle, 0, 0, n, n, n, 1.0, A, n, B, n, 0.0, C, n, tc)

            t0 = time.perf_counter()
            for _ in range(16):
                level = call()
            torch.cuda.synchronize(dev)
            per_call = (time.perf_counter() - t0) / 16
            count = max(1, int(seconds / per_call))
            r = measure(call, count, device_index, 50.0, sync=lambda: torch.cuda.synchronize(dev))
            flops = 2.0 * n * n * n
            rows.append({"compute_type": "tf32" if tc else "fp16", "m": n, "n": n, "k": n, "op_a": "N", "op_b": "N",
                         "tflops": flops * count / r["seconds"] / 1e12, "avg_power_w": r["avg_w"],
                         "joules_per_call": r["joules_per_call"],
                         "gflop_per_joule": flops / r["joules_per_call"] / 1e9, "calls": count,
                         "seconds": r["seconds"], "kernel_level": level, "energy_source": r["source"],
                         "sampled_avg_w": r["sampled_avg_w"], "peak_w": r["peak_w"], "samples": r["samples"]})
    return rows
