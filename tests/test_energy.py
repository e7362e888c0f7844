"""The energy harness (shgemm_b200/energy.py) on the CPU against a fake NVML: the energy of a
timed region comes from the board's energy counter when it has one, else from the power
samples integrated by the trapezoid rule; nothing here touches a GPU or changes a setting."""
import time

from shgemm_b200 import energy


class FakeNVML:
    """Constant board power; an energy counter that advances with wall time (or none)."""

    def __init__(self, watts=500.0, counter=True):
        self.watts = watts
        self.counter = counter
        self.t0 = time.perf_counter()
        self.inits = 0

    def nvmlInit(self):
        self.inits += 1

    def nvmlDeviceGetHandleByIndex(self, i):
        return ("gpu", i)

    def nvmlDeviceGetHandleByUUID(self, u):
        raise RuntimeError("no uuid")

    def nvmlDeviceGetHandleByPciBusId(self, b):
        raise RuntimeError("no bus id")

    def nvmlDeviceGetPowerUsage(self, h):
        return int(self.watts * 1000)  # milliwatts

    def nvmlDeviceGetTotalEnergyConsumption(self, h):
        if not self.counter:
            raise RuntimeError("not supported")
        return int((time.perf_counter() - self.t0) * self.watts * 1000)  # millijoules


def _busy(seconds):
    t = time.perf_counter()
    while time.perf_counter() - t < seconds:
        pass


def test_counter_energy_per_call():
    nv = FakeNVML(400.0)
    r = energy.measure(lambda: _busy(0.05), 6, nvml=nv, interval_ms=10)
    assert r["source"] == "NVML energy counter"
    assert abs(r["avg_w"] - 400.0) < 40.0
    assert abs(r["joules_per_call"] - 400.0 * r["seconds"] / 6) < 1e-6 + 0.02 * r["joules_per_call"] * 6
    assert r["samples"] >= 5 and abs(r["sampled_avg_w"] - 400.0) < 1e-9


def test_sampled_energy_without_counter():
    nv = FakeNVML(250.0, counter=False)
    r = energy.measure(lambda: _busy(0.05), 4, nvml=nv, interval_ms=10)
    assert r["source"].startswith("NVML power samples")
    # constant power: the trapezoid integral over the region equals P * t
    assert abs(r["joules"] - 250.0 * r["seconds"]) < 0.05 * 250.0 * r["seconds"]
    assert r["peak_w"] == 250.0
