"""bench.py on the CPU: its workloads are well formed, the CLI parses, and the reference arm
(the restated reference algorithm timed on the host cores) prints the contract's JSON line."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

REQUIRED = {"m", "n", "k", "op_a", "op_b", "tc", "alpha", "beta", "dist", "desc"}


def test_workloads_well_formed():
    for name, wl in bench.WORKLOADS.items():
        assert REQUIRED <= set(wl), name
        assert wl["tc"] in (0, 1) and wl["op_a"] in (0, 1) and wl["op_b"] in (0, 1), name
        assert wl.get("bound", "tensor") in ("tensor", "hbm"), name
    for nested in ("grouped", "grouped_fused", "square16k", "served"):
        assert nested in bench.WORKLOADS


def test_cli_help():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0 and "--workload" in r.stdout


@pytest.mark.timeout(300)
def test_reference_arm_prints_the_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                        "square1k", "--steps", "1", "--warmup", "1"], capture_output=True, text=True, timeout=280,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference" and line["unit"] == "TFLOP/s" and line["value"] > 0
    assert line["steps"] == 1 and line["warmup"] >= 3
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["metric"] == bench.METRIC


def test_cmake_project_configures(tmp_path):
    """The CMake project (target `shgemm`, as the reference's) configures; building it is the
    same nvcc compile as build.py."""
    import shutil

    cmake = shutil.which("cmake")
    if cmake is None:
        pytest.skip("cmake not installed")
    r = subprocess.run([cmake, "-S", ROOT, "-B", str(tmp_path)], capture_output=True, text=True, timeout=240)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    r = subprocess.run([cmake, "--build", str(tmp_path), "--target", "help"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0 and "shgemm" in r.stdout
