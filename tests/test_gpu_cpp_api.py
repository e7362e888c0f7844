"""The mtk::shgemm C++ API as a drop-in: the reference README's calls, compiled
against include/shgemm/shgemm.hpp and linked to libshgemm_b200.so."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.gpu


def test_cpp_api_sample(cuda_device, tmp_path):
    import shgemm_b200

    libdir = os.path.dirname(shgemm_b200.library_path())
    exe = tmp_path / "api_sample"
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    env = dict(os.environ)
    env.pop("CC", None)
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-I",
                    os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "api_sample.cu"), "-L", libdir,
                    "-lshgemm_b200", "-Xlinker", f"-rpath={libdir}", "-o", str(exe)], check=True, env=env)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().endswith("OK")
