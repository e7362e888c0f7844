"""Sketch server: Python view of the library's continuous-batching sketch service
(``shgemm_b200_server_*`` in include/shgemm_b200.h). No reference counterpart -- the
reference's callers loop over ``mtk::shgemm::shgemm`` (src/shgemm.cu:517-686) one
problem at a time.

The server thread, its admission queue, memory arena and grouped launches all live
in the C++ library; this module only declares the structs and wraps the calls.
"""
from __future__ import annotations

import ctypes

from . import ShgemmError, _addr, _check, _stream_addr, lib

GAUSSIAN, RADEMACHER, RADEMACHER_BLOCKS = 0, 1, 2             # SHGEMM_OMEGA_*
QUEUED, ADMITTED, RUNNING, DONE, FAILED, UNKNOWN = range(6)   # SHGEMM_REQ_*
_SEED_STEP = 1099511628211                                    # draw j uses seed * _SEED_STEP + j


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("compute_type", ctypes.c_int), ("max_batch", ctypes.c_int),
                ("streams", ctypes.c_int), ("auto_release", ctypes.c_int)]


class SketchRequest(ctypes.Structure):
    _fields_ = [("m", ctypes.c_size_t), ("n", ctypes.c_size_t), ("k", ctypes.c_size_t), ("a", ctypes.c_void_p),
                ("lda", ctypes.c_size_t), ("draws", ctypes.c_int), ("omega_dist", ctypes.c_int),
                ("omega_scale", ctypes.c_float), ("omega_seed", ctypes.c_ulonglong)]


class OmegaJob(ctypes.Structure):
    _fields_ = [("dst", ctypes.c_void_p), ("ld", ctypes.c_size_t), ("k", ctypes.c_size_t), ("cols", ctypes.c_size_t),
                ("seed", ctypes.c_ulonglong), ("scale", ctypes.c_float), ("dist", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_ulonglong), ("completed", ctypes.c_ulonglong), ("failed", ctypes.c_ulonglong),
                ("batches", ctypes.c_ulonglong), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double), ("flops_completed", ctypes.c_double),
                ("span_s", ctypes.c_double), ("peak_resident_bytes", ctypes.c_size_t),
                ("resident_bytes", ctypes.c_size_t), ("queued", ctypes.c_ulonglong), ("in_flight", ctypes.c_ulonglong),
                ("kernel_busy_s", ctypes.c_double), ("omega_s", ctypes.c_double), ("launches", ctypes.c_ulonglong)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


_declared = False


def _declare():
    global _declared
    if _declared:
        return lib()
    L = lib()
    vp, sz, i, d = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_double
    ull = ctypes.c_ulonglong
    sig = {
        "shgemm_b200_generate_omega": [vp, vp, sz, sz, sz, i, ull, ctypes.c_float, i],
        "shgemm_b200_generate_omega_batch": [vp, ctypes.POINTER(OmegaJob), i, i],
        "shgemm_b200_server_create": [ctypes.POINTER(vp), i, ctypes.POINTER(ServerConfig)],
        "shgemm_b200_server_destroy": [vp],
        "shgemm_b200_server_submit": [vp, ctypes.POINTER(SketchRequest), ctypes.POINTER(ull)],
        "shgemm_b200_server_poll": [vp, ull, ctypes.POINTER(i), ctypes.POINTER(vp), ctypes.POINTER(sz),
                                    ctypes.POINTER(d)],
        "shgemm_b200_server_wait": [vp, ull, d, ctypes.POINTER(i)],
        "shgemm_b200_server_drain": [vp, d],
        "shgemm_b200_server_release": [vp, ull],
        "shgemm_b200_server_get_stats": [vp, ctypes.POINTER(ServerStats)],
        "shgemm_b200_server_reset_stats": [vp],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = i
    _declared = True
    return L


def draw_seed(seed: int, j: int) -> int:
    """Seed of draw j of a request whose omega_seed is `seed` (what the server passes to generate_omega)."""
    return (seed * _SEED_STEP + j) & 0xFFFFFFFFFFFFFFFF


def generate_omega(dst, ld: int, k: int, cols: int, dist: int = GAUSSIAN, seed: int = 0, scale: float = 1.0,
                   fp32: bool = False, stream=None) -> None:
    """Writes a k x cols column-major Omega (binary16, or binary16 values widened to FP32) on `stream`."""
    _check(_declare().shgemm_b200_generate_omega(_stream_addr(stream), _addr(dst), ld, k, cols, dist,
                                                 seed & 0xFFFFFFFFFFFFFFFF, scale, int(fp32)), "generate_omega")


def generate_omega_batch(jobs, fp32: bool = False, stream=None) -> None:
    """Writes several Omegas in one launch per 64: ``jobs`` holds (dst, ld, k, cols, dist, seed,
    scale) tuples, each written exactly as ``generate_omega`` would."""
    arr = (OmegaJob * max(1, len(jobs)))()
    for q, (dst, ld, k, cols, dist, seed, scale) in zip(arr, jobs):
        q.dst, q.ld, q.k, q.cols = _addr(dst), ld, k, cols
        q.seed, q.scale, q.dist = seed & 0xFFFFFFFFFFFFFFFF, scale, dist
    _check(_declare().shgemm_b200_generate_omega_batch(_stream_addr(stream), arr, len(jobs), int(fp32)),
           "generate_omega_batch")


class SketchServer:
    """Continuous-batching sketch service on one GPU.

    ``submit(m, n, k, A, lda, draws=4, ...)`` queues Y = A [Omega_1 .. Omega_draws] and returns a
    ticket; ``wait``/``poll`` report completion and give Y's device address (m x draws*n,
    column-major, ld = m), ``release`` returns Y's memory to the budget.
    """

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 40 << 30, compute_type: int = 1,
                 max_batch: int = 512, streams: int = 3, auto_release: bool = False):
        L = _declare()
        self._s = ctypes.c_void_p()
        cfg = ServerConfig(hbm_budget_bytes, compute_type, max_batch, streams, int(auto_release))
        _check(L.shgemm_b200_server_create(ctypes.byref(self._s), device, ctypes.byref(cfg)), "server_create")
        self.device = device
        self.compute_type = compute_type

    def close(self) -> None:
        if self._s:
            _declare().shgemm_b200_server_destroy(self._s)
            self._s = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, m: int, n: int, k: int, a, lda: int, draws: int = 4, dist: int = GAUSSIAN,
               scale: float | None = None, seed: int = 0) -> int:
        req = SketchRequest(m, n, k, _addr(a), lda, draws, dist, (n ** -0.5) if scale is None else scale,
                            seed & 0xFFFFFFFFFFFFFFFF)
        t = ctypes.c_ulonglong()
        _check(_declare().shgemm_b200_server_submit(self._s, ctypes.byref(req), ctypes.byref(t)), "server_submit")
        return t.value

    def poll(self, ticket: int):
        """(state, y_address or 0, ldy, latency_ms)."""
        st, y, ld, lat = ctypes.c_int(), ctypes.c_void_p(), ctypes.c_size_t(), ctypes.c_double()
        _declare().shgemm_b200_server_poll(self._s, ticket, ctypes.byref(st), ctypes.byref(y), ctypes.byref(ld),
                                           ctypes.byref(lat))
        return st.value, (y.value or 0), ld.value, lat.value

    def wait(self, ticket: int, timeout_ms: float = 60000.0) -> int:
        st = ctypes.c_int()
        status = _declare().shgemm_b200_server_wait(self._s, ticket, timeout_ms, ctypes.byref(st))
        if status != 0:
            raise ShgemmError(status, "server_wait")
        return st.value

    def drain(self, timeout_ms: float = 600000.0) -> None:
        _check(_declare().shgemm_b200_server_drain(self._s, timeout_ms), "server_drain")

    def release(self, ticket: int) -> None:
        _check(_declare().shgemm_b200_server_release(self._s, ticket), "server_release")

    def stats(self) -> dict:
        s = ServerStats()
        _check(_declare().shgemm_b200_server_get_stats(self._s, ctypes.byref(s)), "server_get_stats")
        return s.as_dict()

    def reset_stats(self) -> None:
        _check(_declare().shgemm_b200_server_reset_stats(self._s), "server_reset_stats")
