"""The C-ABI library builds, loads without a GPU and exports every entry point
that include/shgemm_b200.h declares (no compute calls here)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for hdr in ("shgemm_b200.h",):
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(shgemm_b200_\w+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "shgemm_b200_shgemm" in names and "shgemm_b200_hsgemm" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    import shgemm_b200

    path = shgemm_b200.library_path()
    assert os.path.exists(path), "run __graft_entry__.build() first"
    lib = ctypes.CDLL(path)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    for n in declared_symbols():
        assert re.search(rf"\bT {n}$", out, flags=re.M), n


def test_cpp_api_symbols_exported():
    import shgemm_b200

    out = subprocess.run(["nm", "-DC", "--defined-only", shgemm_b200.library_path()], capture_output=True,
                         text=True).stdout
    for fn in ("mtk::shgemm::create", "mtk::shgemm::destroy", "mtk::shgemm::set_cuda_stream",
               "mtk::shgemm::enable_kernel_level_fixing", "mtk::shgemm::disable_kernel_level_fixing",
               "mtk::shgemm::set_debug_mode", "mtk::shgemm::shgemm("):
        assert fn in out, fn


def test_status_strings_without_gpu():
    import shgemm_b200

    L = shgemm_b200.lib()
    assert L.shgemm_b200_status_string(0) == b"SHGEMM_STATUS_OK"
    assert L.shgemm_b200_status_string(5) == b"SHGEMM_STATUS_TIMEOUT"


def test_create_without_gpu_fails_cleanly():
    import torch

    import shgemm_b200

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(shgemm_b200.ShgemmError):
        shgemm_b200.Handle(0)


def test_library_is_built_for_sm100a_only():
    """Both build recipes compile device code for sm_100a alone (machine code, no PTX for
    other architectures to JIT from)."""
    from shgemm_b200 import build

    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    cmake = open(os.path.join(ROOT, "CMakeLists.txt")).read()
    assert re.search(r"CMAKE_CUDA_ARCHITECTURES\s+100a-real\)", cmake)


def test_c_header_is_plain_c_and_links(tmp_path):
    """include/shgemm_b200.h is strict C99 (what cgo, JNI and ctypes bindings include) and a
    C program links against the library with it."""
    import shgemm_b200

    src = tmp_path / "c_user.c"
    src.write_text('#include "shgemm_b200.h"\n'
                   "int main(void) { return shgemm_b200_noalloc_scratch_bytes() > 0 ? 0 : 1; }\n")
    libdir = os.path.dirname(shgemm_b200.library_path())
    env = dict(os.environ)
    env.pop("CC", None)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I",
                    os.path.join(ROOT, "include"), str(src), "-L", libdir, "-lshgemm_b200", "-o",
                    str(tmp_path / "c_user")], check=True, env=env)


def test_cpp_header_compiles_as_host_cpp(tmp_path):
    """include/shgemm/shgemm.hpp builds with the host C++ compiler alone (callers need not
    compile with nvcc to use the C++ API)."""
    src = tmp_path / "cpp_user.cpp"
    src.write_text("#include <shgemm/shgemm.hpp>\nint main() { return 0; }\n")
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    env = dict(os.environ)
    env.pop("CXX", None)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), "-I",
                    cuda_inc, "-c", str(src), "-o", str(tmp_path / "cpp_user.o")], check=True, env=env)


def test_host_entry_points_validate_without_gpu():
    """The host-buffer entry points reject a missing handle before any CUDA call."""
    import shgemm_b200

    L = shgemm_b200.lib()
    one = ctypes.c_float(1.0)
    lvl = ctypes.c_int(-7)
    for fn in (L.shgemm_b200_shgemm_host, L.shgemm_b200_hsgemm_host):
        st = fn(None, 0, 0, 4, 4, 4, ctypes.byref(one), None, 4, None, 4, ctypes.byref(one), None, 4, 0, 0,
                ctypes.byref(lvl))
        assert st == 1  # SHGEMM_STATUS_INVALID_VALUE
    assert L.shgemm_b200_release_host_staging(None) == 1


def test_cpp_api_sample_builds_without_gpu(tmp_path):
    """The reference README's usage (tests/cpp/api_sample.cu) compiles with nvcc for sm_100a
    and links against the library here; the GPU test suite runs it."""
    import shgemm_b200
    from shgemm_b200 import build

    libdir = os.path.dirname(shgemm_b200.library_path())
    env = dict(os.environ)
    env.pop("CC", None)
    subprocess.run([build.nvcc(), "-std=c++17", "-O2", *build.ARCH, "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "api_sample.cu"), "-L", libdir, "-lshgemm_b200",
                    "-o", str(tmp_path / "api_sample")], check=True, env=env)
    assert (tmp_path / "api_sample").exists()
