"""shgemm_b200 -- B200 (sm_100a) SHGEMM/HSGEMM with the reference's error-corrected method.

Host-side Python mirror of the reference's ``mtk::shgemm`` interface
(include/shgemm/shgemm.hpp:94-157) over the C ABI of ``libshgemm_b200.so``
(include/shgemm_b200.h). Operands are CUDA device buffers: torch tensors (their
data pointers are used) or raw integer device addresses. Column-major BLAS
semantics, host-side alpha/beta, asynchronous execution on the handle's stream.

There is no CPU fallback: every call goes to the CUDA library, and importing
this package fails loudly when the shared library is missing.
"""
from __future__ import annotations

import ctypes
import os

__all__ = [
    "op_n", "op_t", "fp16", "tf32", "P0", "P1", "ShgemmError", "Handle", "create", "destroy",
    "set_cuda_stream", "enable_kernel_level_fixing", "disable_kernel_level_fixing", "set_debug_mode",
    "shgemm", "hsgemm", "shgemm_device_scalars", "hsgemm_device_scalars", "shgemm_host", "hsgemm_host",
    "release_host_staging", "library_path",
]

op_n, op_t = 0, 1          # operation_t (include/shgemm/shgemm.hpp:36-39)
fp16, tf32 = 0, 1          # tc_t (include/shgemm/shgemm.hpp:41-44)
P0, P1 = 0, 1              # detail::kernel_level (include/shgemm/shgemm.hpp:30-34)

CFG_SPLIT_K, CFG_WAIT_LIMIT_MS, CFG_GROUP_M, CFG_GROUPED_B_FP32, CFG_AUTOTUNE, CFG_TILE_KERNEL, CFG_K_CHUNK = (
    2, 3, 4, 5, 6, 7, 8)
CFG_HOST_BLOCK_COLS, CFG_TM_STAGES, CFG_PAIR_TILES = 9, 10, 11

STATUS = {0: "OK", 1: "INVALID_VALUE", 2: "NOT_SUPPORTED", 3: "ALLOC_FAILED", 4: "LAUNCH_FAILED",
          5: "TIMEOUT", 6: "CUDA_ERROR", 7: "SCRATCH_TOO_SMALL"}

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libshgemm_b200.so")
_lib = None


class Problem(ctypes.Structure):
    """shgemm_b200_problem: one problem of a grouped launch (include/shgemm_b200.h)."""

    _fields_ = [("m", ctypes.c_size_t), ("n", ctypes.c_size_t), ("k", ctypes.c_size_t), ("a", ctypes.c_void_p),
                ("lda", ctypes.c_size_t), ("b", ctypes.c_void_p), ("ldb", ctypes.c_size_t), ("c", ctypes.c_void_p),
                ("ldc", ctypes.c_size_t), ("alpha", ctypes.c_float), ("beta", ctypes.c_float),
                ("b_generated", ctypes.c_int), ("omega_seed", ctypes.c_ulonglong)]


class TunedConfig(ctypes.Structure):
    """shgemm_b200_tuned_config: the autotuner's choice for a shape bucket (include/shgemm_b200.h)."""

    _fields_ = [("tile_n", ctypes.c_int), ("slices", ctypes.c_int), ("group_m", ctypes.c_int),
                ("time_us", ctypes.c_float), ("stages", ctypes.c_int), ("k_chunk", ctypes.c_int),
                ("cta_group", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {"tile_n": self.tile_n, "slices": self.slices, "group_m": self.group_m, "time_us": self.time_us,
                "stages": self.stages, "k_chunk": self.k_chunk, "cta_group": self.cta_group}


class ShgemmError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: SHGEMM_STATUS_{STATUS.get(status, status)}")


def library_path() -> str:
    return _LIB_PATH


def lib() -> ctypes.CDLL:
    """Loads the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise ImportError(f"{_LIB_PATH} is missing: build it with `python -m shgemm_b200.build`")
    L = ctypes.CDLL(_LIB_PATH)
    vp, sz, i, f, d = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_float, ctypes.c_double
    pi, pf, pd = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)
    sig = {
        "shgemm_b200_create": [ctypes.POINTER(vp), i],
        "shgemm_b200_destroy": [vp],
        "shgemm_b200_set_stream": [vp, vp],
        "shgemm_b200_set_kernel_level": [vp, i],
        "shgemm_b200_set_debug_mode": [vp, ctypes.c_uint],
        "shgemm_b200_shgemm": [vp, i, i, sz, sz, sz, pf, vp, sz, vp, sz, pf, vp, sz, i, i, pi],
        "shgemm_b200_hsgemm": [vp, i, i, sz, sz, sz, pf, vp, sz, vp, sz, pf, vp, sz, i, i, pi],
        "shgemm_b200_shgemm_device_scalars": [vp, i, i, sz, sz, sz, vp, vp, sz, vp, sz, vp, vp, sz, i, i, pi],
        "shgemm_b200_hsgemm_device_scalars": [vp, i, i, sz, sz, sz, vp, vp, sz, vp, sz, vp, vp, sz, i, i, pi],
        "shgemm_b200_shgemm_host": [vp, i, i, sz, sz, sz, pf, vp, sz, vp, sz, pf, vp, sz, i, i, pi],
        "shgemm_b200_release_host_staging": [vp],
        "shgemm_b200_hsgemm_host": [vp, i, i, sz, sz, sz, pf, vp, sz, vp, sz, pf, vp, sz, i, i, pi],
        "shgemm_b200_set_config": [vp, i, ctypes.c_longlong],
        "shgemm_b200_get_config": [vp, i, ctypes.POINTER(ctypes.c_longlong)],
        "shgemm_b200_set_workspace_size": [vp, sz],
        "shgemm_b200_get_workspace": [vp, ctypes.POINTER(vp), ctypes.POINTER(sz)],
        "shgemm_b200_plan_preview": [i, sz, sz, sz, i, sz, pi, pi, pi],
        "shgemm_b200_check_error": [vp, pi],
        "shgemm_b200_get_launch_count": [vp, ctypes.POINTER(ctypes.c_longlong)],
        "shgemm_b200_selftest_wait_timeout": [vp, ctypes.c_uint, pi],
        "shgemm_b200_eval_dgemm": [vp, i, i, sz, sz, sz, vp, sz, vp, sz, vp],
        "shgemm_b200_eval_dgemm_hs": [vp, i, i, sz, sz, sz, vp, sz, vp, sz, vp],
        "shgemm_b200_eval_error": [vp, sz, sz, vp, sz, i, vp, d, d, vp, pd],
        "shgemm_b200_shgemm_noalloc": [vp, i, i, sz, sz, sz, pf, vp, sz, vp, sz, pf, vp, sz, i, i, pi],
        "shgemm_b200_shgemm_grouped": [vp, i, i, i, i, ctypes.POINTER(Problem), i],
        "shgemm_b200_grouped_update": [vp, i, i, i, i, ctypes.POINTER(Problem), i],
        "shgemm_b200_noalloc_check_error": [vp, pi],
        "shgemm_b200_autotune": [vp, i, i, sz, sz, sz, vp, sz, vp, sz, vp, sz, i, ctypes.POINTER(TunedConfig)],
        "shgemm_b200_autotune_lookup": [vp, i, i, sz, sz, sz, i, ctypes.POINTER(TunedConfig)],
        "shgemm_b200_autotune_save": [vp, ctypes.c_char_p],
        "shgemm_b200_autotune_load": [vp, ctypes.c_char_p],
        "shgemm_b200_autotune_clear": [vp],
        "shgemm_b200_autotune_grouped": [vp, i, i, i, i, ctypes.POINTER(Problem), i, pi],
        "shgemm_b200_autotune_grouped_lookup": [vp, i, i, i, sz, pi],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = i
    L.shgemm_b200_noalloc_scratch_bytes.argtypes = []
    L.shgemm_b200_noalloc_scratch_bytes.restype = sz
    L.shgemm_b200_status_string.argtypes = [i]
    L.shgemm_b200_status_string.restype = ctypes.c_char_p
    _lib = L
    return L


def _check(status: int, what: str) -> None:
    if status != 0:
        raise ShgemmError(status, what)


def _addr(x) -> int:
    """Device address of a torch tensor or an integer pointer."""
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    ptr = getattr(x, "data_ptr", None)
    if ptr is None:
        raise TypeError(f"expected a CUDA tensor or a device address, got {type(x)!r}")
    if not getattr(x, "is_cuda", True):
        raise ValueError("operands must live in CUDA device memory")
    return ptr()


def _stream_addr(stream) -> int:
    if stream is None:
        return 0
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)


class Handle:
    """The reference's shgemmHandle_t (include/shgemm/shgemm.hpp:46-92)."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        self.device = device
        _check(lib().shgemm_b200_create(ctypes.byref(self._h), device), "shgemm_b200_create")
        self.cuda_stream = 0

    @property
    def ptr(self) -> ctypes.c_void_p:
        if not self._h:
            raise ShgemmError(1, "handle destroyed")
        return self._h

    def close(self) -> None:
        if self._h:
            _check(lib().shgemm_b200_destroy(self._h), "shgemm_b200_destroy")
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream) -> None:
        self.cuda_stream = _stream_addr(stream)
        _check(lib().shgemm_b200_set_stream(self.ptr, ctypes.c_void_p(self.cuda_stream)), "set_stream")

    def set_config(self, key: int, value: int) -> None:
        _check(lib().shgemm_b200_set_config(self.ptr, key, value), "set_config")

    def get_config(self, key: int) -> int:
        v = ctypes.c_longlong()
        _check(lib().shgemm_b200_get_config(self.ptr, key, ctypes.byref(v)), "get_config")
        return v.value

    def set_workspace_size(self, nbytes: int) -> None:
        _check(lib().shgemm_b200_set_workspace_size(self.ptr, nbytes), "set_workspace_size")

    def workspace(self) -> tuple[int, int]:
        """(device address, bytes) of the handle's workspace (the reference's w_ptr)."""
        p, n = ctypes.c_void_p(), ctypes.c_size_t()
        _check(lib().shgemm_b200_get_workspace(self.ptr, ctypes.byref(p), ctypes.byref(n)), "get_workspace")
        return int(p.value or 0), int(n.value)

    def check_error(self) -> int:
        """Synchronises and returns the device error code (0 = none)."""
        code = ctypes.c_int()
        st = lib().shgemm_b200_check_error(self.ptr, ctypes.byref(code))
        if st not in (0, 5):
            raise ShgemmError(st, "check_error")
        return code.value

    def autotune(self, op_a: int, op_b: int, m: int, n: int, k: int, A, lda: int, B, ldb: int, C, ldc: int,
                 compute_type: int) -> dict:
        """Times the candidate plans on these operands (C is overwritten), keeps the fastest
        for the shape's bucket and returns it."""
        best = TunedConfig()
        _check(lib().shgemm_b200_autotune(self.ptr, op_a, op_b, m, n, k, _addr(A), lda, _addr(B), ldb, _addr(C), ldc,
                                          compute_type, ctypes.byref(best)), "autotune")
        return best.as_dict()

    def autotune_lookup(self, op_a: int, op_b: int, m: int, n: int, k: int, compute_type: int):
        """The tuned entry of the shape's bucket, or None."""
        cfg = TunedConfig()
        st = lib().shgemm_b200_autotune_lookup(self.ptr, op_a, op_b, m, n, k, compute_type, ctypes.byref(cfg))
        return cfg.as_dict() if st == 0 else None

    def autotune_grouped(self, problems, compute_type: int, op_a: int = 0, op_b: int = 0, op_c: int = 0) -> int:
        """Tunes the tile N of grouped launches per n bucket on this batch (its C is overwritten);
        returns the number of buckets tuned."""
        arr = _problem_array(problems)
        n = ctypes.c_int()
        _check(lib().shgemm_b200_autotune_grouped(self.ptr, op_a, op_b, compute_type, op_c, arr, len(problems),
                                                  ctypes.byref(n)), "autotune_grouped")
        return n.value

    def autotune_grouped_lookup(self, n: int, compute_type: int, op_a: int = 0, b_fp32: bool = False):
        """The tuned tile N of grouped problems with this n's bucket, or None."""
        bn = ctypes.c_int()
        st = lib().shgemm_b200_autotune_grouped_lookup(self.ptr, op_a, compute_type, int(b_fp32), n, ctypes.byref(bn))
        return bn.value if st == 0 else None

    def autotune_save(self, path: str) -> None:
        _check(lib().shgemm_b200_autotune_save(self.ptr, os.fsencode(path)), "autotune_save")

    def autotune_load(self, path: str) -> None:
        _check(lib().shgemm_b200_autotune_load(self.ptr, os.fsencode(path)), "autotune_load")

    def autotune_clear(self) -> None:
        _check(lib().shgemm_b200_autotune_clear(self.ptr), "autotune_clear")

    def launch_count(self) -> int:
        v = ctypes.c_longlong()
        _check(lib().shgemm_b200_get_launch_count(self.ptr, ctypes.byref(v)), "get_launch_count")
        return v.value

    def selftest_wait_timeout(self, limit_us: int = 20000) -> tuple[int, int]:
        code = ctypes.c_int()
        st = lib().shgemm_b200_selftest_wait_timeout(self.ptr, limit_us, ctypes.byref(code))
        return st, code.value


# ---------------------------------------------------------------- reference-shaped API
def plan_preview(num_sms: int, m: int, n: int, k: int, compute_type: int, workspace_bytes: int) -> dict:
    """The heuristic plan of a call (kernel level, tile N, split-K slices), computed on the host
    without a device: the planner behind shgemm before autotuned entries or level fixing."""
    level, tile_n, slices = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _check(lib().shgemm_b200_plan_preview(num_sms, m, n, k, compute_type, workspace_bytes, ctypes.byref(level),
                                          ctypes.byref(tile_n), ctypes.byref(slices)), "plan_preview")
    return {"level": level.value, "tile_n": tile_n.value, "slices": slices.value}


def create(device: int = 0) -> Handle:
    """mtk::shgemm::create (include/shgemm/shgemm.hpp:94)."""
    return Handle(device)


def destroy(handle: Handle) -> None:
    """mtk::shgemm::destroy (include/shgemm/shgemm.hpp:95)."""
    handle.close()


def set_cuda_stream(handle: Handle, stream) -> None:
    """mtk::shgemm::set_cuda_stream (include/shgemm/shgemm.hpp:102)."""
    handle.set_stream(stream)


def enable_kernel_level_fixing(handle: Handle, level: int) -> None:
    """include/shgemm/shgemm.hpp:97."""
    _check(lib().shgemm_b200_set_kernel_level(handle.ptr, level), "enable_kernel_level_fixing")


def disable_kernel_level_fixing(handle: Handle) -> None:
    """include/shgemm/shgemm.hpp:98."""
    _check(lib().shgemm_b200_set_kernel_level(handle.ptr, -1), "disable_kernel_level_fixing")


def set_debug_mode(handle: Handle, on: int) -> None:
    """include/shgemm/shgemm.hpp:100."""
    _check(lib().shgemm_b200_set_debug_mode(handle.ptr, on), "set_debug_mode")


def shgemm(handle: Handle, op_a: int, op_b: int, m: int, n: int, k: int, alpha: float, a, lda: int, b, ldb: int,
           beta: float, c, ldc: int, compute_type: int, op_c: int = op_n) -> int:
    """mtk::shgemm::shgemm (include/shgemm/shgemm.hpp:105-119): A FP32, B binary16.

    Returns the kernel level, like the reference. Raises ShgemmError on failure.
    """
    al, be, lv = ctypes.c_float(alpha), ctypes.c_float(beta), ctypes.c_int(0)
    st = lib().shgemm_b200_shgemm(handle.ptr, op_a, op_b, m, n, k, ctypes.byref(al), _addr(a), lda, _addr(b), ldb,
                                  ctypes.byref(be), _addr(c), ldc, compute_type, op_c, ctypes.byref(lv))
    _check(st, "shgemm")
    return lv.value


def hsgemm(handle: Handle, op_a: int, op_b: int, m: int, n: int, k: int, alpha: float, a, lda: int, b, ldb: int,
           beta: float, c, ldc: int, compute_type: int, op_c: int = op_n) -> int:
    """mtk::shgemm::hsgemm (include/shgemm/shgemm.hpp:121-157): A binary16, B FP32."""
    al, be, lv = ctypes.c_float(alpha), ctypes.c_float(beta), ctypes.c_int(0)
    st = lib().shgemm_b200_hsgemm(handle.ptr, op_a, op_b, m, n, k, ctypes.byref(al), _addr(a), lda, _addr(b), ldb,
                                  ctypes.byref(be), _addr(c), ldc, compute_type, op_c, ctypes.byref(lv))
    _check(st, "hsgemm")
    return lv.value


def shgemm_device_scalars(handle: Handle, op_a: int, op_b: int, m: int, n: int, k: int, alpha_dev, a, lda: int, b,
                          ldb: int, beta_dev, c, ldc: int, compute_type: int, op_c: int = op_n) -> int:
    """shgemm with alpha and beta read from device memory by the kernels (one float each,
    e.g. 1-element CUDA tensors): a captured CUDA graph replays with whatever they hold."""
    lv = ctypes.c_int(0)
    st = lib().shgemm_b200_shgemm_device_scalars(handle.ptr, op_a, op_b, m, n, k, _addr(alpha_dev), _addr(a), lda,
                                                 _addr(b), ldb, _addr(beta_dev), _addr(c), ldc, compute_type, op_c,
                                                 ctypes.byref(lv))
    _check(st, "shgemm_device_scalars")
    return lv.value


def hsgemm_device_scalars(handle: Handle, op_a: int, op_b: int, m: int, n: int, k: int, alpha_dev, a, lda: int, b,
                          ldb: int, beta_dev, c, ldc: int, compute_type: int, op_c: int = op_n) -> int:
    """hsgemm (A binary16, B FP32) with device-resident alpha and beta."""
    lv = ctypes.c_int(0)
    st = lib().shgemm_b200_hsgemm_device_scalars(handle.ptr, op_a, op_b, m, n, k, _addr(alpha_dev), _addr(a), lda,
                                                 _addr(b), ldb, _addr(beta_dev), _addr(c), ldc, compute_type, op_c,
                                                 ctypes.byref(lv))
    _check(st, "hsgemm_device_scalars")
    return lv.value


# ---------------------------------------------------------------- host buffers
def _host_addr(x) -> int:
    """Host address of a CPU torch tensor, a C-contiguous numpy array or an integer pointer."""
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if getattr(x, "is_cuda", False):
            raise ValueError("shgemm_host takes host buffers; use shgemm for device memory")
        return x.data_ptr()
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    raise TypeError(f"expected a host tensor, a numpy array or an address, got {type(x)!r}")


def shgemm_host(handle: Handle, op_a: int, op_b: int, m: int, n: int, k: int, alpha: float, a, lda: int, b, ldb: int,
                beta: float, c, ldc: int, compute_type: int, op_c: int = op_n) -> int:
    """shgemm with A, B and C in host memory; copies overlap the computation.

    A goes to the device once, then C is computed in column blocks whose B/C uploads,
    computation and C download overlap on separate streams. Pass page-locked buffers
    (torch `pin_memory=True`) for the overlap. Asynchronous on the handle's stream:
    synchronise it before reading C. Returns the kernel level of the first block.
    """
    al, be, lv = ctypes.c_float(alpha), ctypes.c_float(beta), ctypes.c_int(0)
    st = lib().shgemm_b200_shgemm_host(handle.ptr, op_a, op_b, m, n, k, ctypes.byref(al), _host_addr(a), lda,
                                       _host_addr(b), ldb, ctypes.byref(be), _host_addr(c), ldc, compute_type, op_c,
                                       ctypes.byref(lv))
    _check(st, "shgemm_host")
    return lv.value


def hsgemm_host(handle: Handle, op_a: int, op_b: int, m: int, n: int, k: int, alpha: float, a, lda: int, b, ldb: int,
                beta: float, c, ldc: int, compute_type: int, op_c: int = op_n) -> int:
    """hsgemm (A binary16, B FP32) with A, B and C in host memory; see shgemm_host."""
    al, be, lv = ctypes.c_float(alpha), ctypes.c_float(beta), ctypes.c_int(0)
    st = lib().shgemm_b200_hsgemm_host(handle.ptr, op_a, op_b, m, n, k, ctypes.byref(al), _host_addr(a), lda,
                                       _host_addr(b), ldb, ctypes.byref(be), _host_addr(c), ldc, compute_type, op_c,
                                       ctypes.byref(lv))
    _check(st, "hsgemm_host")
    return lv.value


def release_host_staging(handle: Handle) -> None:
    """Frees the device staging that shgemm_host keeps in the handle."""
    _check(lib().shgemm_b200_release_host_staging(handle.ptr), "release_host_staging")


# ---------------------------------------------------------------- allocation-free path
def shgemm_noalloc(stream, op_a: int, op_b: int, m: int, n: int, k: int, alpha: float, a, lda: int, b, ldb: int,
                   beta: float, c, ldc: int, compute_type: int, op_c: int = op_n) -> int:
    """SHGEMM that allocates nothing: no handle, scratch in a fixed device array.

    For callers that cannot call cudaMalloc (an allocator callback, a memory
    manager that owns all device memory). Runs on the current device and
    `stream`; m * n is limited by noalloc_scratch_bytes() / 8. Concurrent calls
    share the scratch and must not overlap on the GPU. The first call on a device
    does its one-time set-up and should come before any stream capture.
    """
    al, be, lv = ctypes.c_float(alpha), ctypes.c_float(beta), ctypes.c_int(0)
    st = lib().shgemm_b200_shgemm_noalloc(ctypes.c_void_p(_stream_addr(stream)), op_a, op_b, m, n, k,
                                          ctypes.byref(al), _addr(a), lda, _addr(b), ldb, ctypes.byref(be), _addr(c),
                                          ldc, compute_type, op_c, ctypes.byref(lv))
    _check(st, "shgemm_noalloc")
    return lv.value


def noalloc_scratch_bytes() -> int:
    return lib().shgemm_b200_noalloc_scratch_bytes()


def noalloc_check_error(stream) -> int:
    """Synchronises `stream`; returns the allocation-free path's device error code."""
    code = ctypes.c_int()
    st = lib().shgemm_b200_noalloc_check_error(ctypes.c_void_p(_stream_addr(stream)), ctypes.byref(code))
    if st not in (0, 5):
        raise ShgemmError(st, "noalloc_check_error")
    return code.value


# ---------------------------------------------------------------- grouped launches
def _problem_array(problems):
    arr = (Problem * max(1, len(problems)))()
    for i, q in enumerate(problems):
        if isinstance(q, Problem):
            arr[i] = q
            continue
        m, n, k, a, lda, b, ldb, c, ldc = q[:9]
        alpha = q[9] if len(q) > 9 else 1.0
        beta = q[10] if len(q) > 10 else 0.0
        gen = q[11] if len(q) > 11 else 0  # RADEMACHER_BLOCKS: B generated in the kernel from q[12]
        seed = q[12] if len(q) > 12 else 0
        arr[i] = Problem(m, n, k, _addr(a), lda, _addr(b), ldb, _addr(c), ldc, alpha, beta, gen,
                         seed & 0xFFFFFFFFFFFFFFFF)
    return arr


def shgemm_grouped(handle: Handle, problems, compute_type: int, op_a: int = op_n, op_b: int = op_n,
                   op_c: int = op_n) -> None:
    """Many SHGEMMs in one persistent launch.

    ``problems``: sequence of ``(m, n, k, A, lda, B, ldb, C, ldc[, alpha[, beta]])`` (tensors or
    device addresses) or :class:`Problem`. Enqueued on the handle's stream; can be captured in a
    CUDA graph and replayed after :func:`grouped_update`.
    """
    arr = _problem_array(problems)
    _check(lib().shgemm_b200_shgemm_grouped(handle.ptr, op_a, op_b, compute_type, op_c, arr, len(problems)),
           "shgemm_grouped")


def grouped_update(handle: Handle, problems, compute_type: int, op_a: int = op_n, op_b: int = op_n,
                   op_c: int = op_n) -> None:
    """Rewrites the staged tables (no launch): the next replay of a captured grouped launch runs this batch."""
    arr = _problem_array(problems)
    _check(lib().shgemm_b200_grouped_update(handle.ptr, op_a, op_b, compute_type, op_c, arr, len(problems)),
           "grouped_update")
