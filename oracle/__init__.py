"""CPU oracle for SHGEMM -- test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import this package, and only as the checker / the timed CPU baseline. The
product library (``shgemm_b200``) never imports it.

Parity status: "parity unpinned" against the reference's own outputs -- the
reference's numerics live in an un-vendored submodule (wmma_extension/tcec)
and its tests store no golden values. The element conversions are pinned
bit-for-bit against independent implementations (tests/golden/), and the GEMM
modes against a restatement in exact rational arithmetic (tests/test_oracle_exact.py).
Three accumulation modes: IDEAL (the reference's algorithm with exact fragment sums),
TCMODEL (the reference's tensor-core accumulation) and B200MODEL (this library's own
kernels, down to the MMA instruction, calibrated on the B200's measured errors).

The C restatement lives in ``shgemm_oracle.c`` (each function cites the
reference file:line it follows) and is built by ``oracle/Makefile`` into
``oracle/_build/liboracle.so``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

OP_N, OP_T = 0, 1
FP16, TF32 = 0, 1


def build() -> str:
    """Compiles the C oracle with the system gcc (OpenMP)."""
    env = dict(os.environ)
    env.pop("CC", None)
    subprocess.run(["make", "-s", "-C", _HERE], check=True, env=env)
    return _LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        src = os.path.join(_HERE, "shgemm_oracle.c")
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        sz, i, f, d = ctypes.c_size_t, ctypes.c_int, ctypes.c_float, ctypes.c_double
        p = ctypes.c_void_p
        L.oracle_f32_to_f16_bits.restype = ctypes.c_uint16
        L.oracle_f32_to_f16_bits.argtypes = [f]
        L.oracle_f16_bits_to_f32.restype = f
        L.oracle_f16_bits_to_f32.argtypes = [ctypes.c_uint16]
        L.oracle_round_tf32.restype = f
        L.oracle_round_tf32.argtypes = [f]
        L.oracle_round_f16.restype = f
        L.oracle_round_f16.argtypes = [f]
        L.oracle_split.restype = None
        L.oracle_split.argtypes = [i, p, sz, p, p]
        L.oracle_shgemm.restype = i
        L.oracle_shgemm.argtypes = [i, i, i, sz, sz, sz, f, p, sz, p, sz, f, p, sz, i, sz]
        L.oracle_shgemm_tcmodel.restype = i
        L.oracle_shgemm_tcmodel.argtypes = [i, i, i, sz, sz, sz, f, p, sz, p, sz, f, p, sz, i, sz, i]
        L.oracle_shgemm_b200model.restype = i
        L.oracle_shgemm_b200model.argtypes = [i, i, i, sz, sz, sz, f, p, sz, p, sz, f, p, sz, i, sz, i]
        L.oracle_dgemm_ref.restype = i
        L.oracle_dgemm_ref.argtypes = [i, i, sz, sz, sz, d, p, sz, p, sz, d, p, sz, i, p]
        L.oracle_sgemm.restype = i
        L.oracle_sgemm.argtypes = [i, i, sz, sz, sz, f, p, sz, p, sz, f, p, sz, i]
        L.oracle_num_threads.restype = i
        L.oracle_num_threads.argtypes = []
        for fn in (L.oracle_cpu_sgemm, L.oracle_cpu_dgemm):
            fn.restype = None
            fn.argtypes = [sz, sz, sz, p, sz, p, sz, p, sz]
        _lib = L
    return _lib


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _u16(a) -> np.ndarray:
    a = np.asarray(a)
    if a.dtype == np.float16:
        a = a.view(np.uint16)
    return np.ascontiguousarray(a, dtype=np.uint16)


def f32_to_f16_bits(x) -> np.ndarray:
    x = _f32(x).ravel()
    L = lib()
    return np.fromiter((L.oracle_f32_to_f16_bits(float(v)) for v in x), dtype=np.uint16, count=x.size)


def round_tf32(x) -> np.ndarray:
    x = _f32(x).ravel()
    L = lib()
    return np.fromiter((L.oracle_round_tf32(float(v)) for v in x), dtype=np.float32, count=x.size)


def split(tc: int, x) -> tuple[np.ndarray, np.ndarray]:
    """Reference split (src/wmmae_shgemm.hpp:30-31): (hi, lo) as float32 values."""
    x = _f32(x).ravel()
    hi = np.empty_like(x)
    lo = np.empty_like(x)
    lib().oracle_split(tc, _ptr(x), x.size, _ptr(hi), _ptr(lo))
    return hi, lo


IDEAL, TCMODEL, B200MODEL = "ideal", "tcmodel", "b200model"


# Bits the B200 tensor core keeps when it aligns an MMA's products and accumulator to the
# largest nominal exponent among them (a product's is the sum of its factors' exponents;
# FP32 accumulation), as calibrated against the GPU's measured errors: with 26 the model
# reproduces twelve binary16 ones (64- and 128-k drains, all-positive and mixed-sign inputs,
# both A layouts) to their printed 4 digits, where 24, 25, 27 and 28 miss by 20-300 %, and,
# out of sample, a recorded binary16 and TF32 pair as well.
B200_ALIGN_BITS = 26


def shgemm(tc, op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, op_c=OP_N, chunk=0, model=IDEAL,
           align_bits=None):
    """Restated reference SHGEMM on column-major flat buffers; C is updated in place.

    ``B`` holds binary16 values (np.float16 or their uint16 bits). ``model``: IDEAL sums
    each hi fragment exactly and accumulates lo exactly (oracle_shgemm); TCMODEL models
    the reference's tensor-core accumulation -- hi fragments truncated to FP32 before
    their round-to-nearest add, lo in a truncating FP32 accumulator over all k
    (oracle_shgemm_tcmodel, src/wmmae_shgemm.hpp:86-124; with ``align_bits`` > 0 each fragment
    is instead one MMA modelled as B200MODEL's, i.e. the reference's algorithm on a tensor core
    that aligns like the B200's); B200MODEL models this library's
    kernels instead -- per drain of ``chunk`` k (64 binary16 / 32 TF32 by default) lo then
    hi fragments through one accumulator, one modelled MMA instruction each (terms aligned to
    the largest nominal exponent with ``align_bits`` bits kept and truncated toward zero, the
    sum truncated to FP32; or the exact sum truncated when ``align_bits`` is 0), folded by the
    2^-11 input scale, added to the running sum with round to nearest
    (oracle_shgemm_b200model).
    """
    A = _f32(A)
    B = _u16(B)
    assert C.dtype == np.float32 and C.flags.c_contiguous
    fns = {IDEAL: "oracle_shgemm", TCMODEL: "oracle_shgemm_tcmodel", B200MODEL: "oracle_shgemm_b200model"}
    if model not in fns:
        raise ValueError(model)
    if align_bits is None:
        align_bits = B200_ALIGN_BITS if model == B200MODEL else 0
    args = (tc, op_a, op_b, m, n, k, alpha, _ptr(A), lda, _ptr(B), ldb, beta, _ptr(C), ldc, op_c, chunk)
    rc = getattr(lib(), fns[model])(*(args + ((align_bits,) if model != IDEAL else ())))
    if rc == 2:
        raise ValueError("B200MODEL: chunk a multiple of the MMA fragment (16 k binary16, 8 k TF32); TCMODEL with "
                         "alignment: chunk at most 16; align_bits 0..40")
    if rc != 0:
        raise MemoryError("oracle_shgemm: allocation failed")
    return C


def hsgemm(tc, op_a, op_b, m, n, k, alpha, A_half, lda, B_float, ldb, beta, C, ldc, op_c=OP_N, chunk=0,
           model=IDEAL):
    """HSGEMM through the transposition identity of include/shgemm/shgemm.hpp:121-157."""
    inv = lambda op: OP_T if op == OP_N else OP_N  # noqa: E731
    return shgemm(tc, inv(op_b), inv(op_a), n, m, k, alpha, B_float, ldb, A_half, lda,
                  beta, C, ldc, inv(op_c), chunk, model)


def dgemm_ref(op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta=0.0, Cin=None, ldc=0, op_c=OP_N):
    """FP64 product of the same FP32/binary16 inputs; returns (m, n) float64 in logical layout."""
    A = _f32(A)
    B = _u16(B)
    out = np.empty(m * n, dtype=np.float64)
    cin = None if Cin is None else _f32(Cin)
    rc = lib().oracle_dgemm_ref(op_a, op_b, m, n, k, alpha, _ptr(A), lda, _ptr(B), ldb, beta,
                                _ptr(cin), ldc, op_c, _ptr(out))
    if rc != 0:
        raise MemoryError("oracle_dgemm_ref: allocation failed")
    return out.reshape(n, m).T


def sgemm(op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, op_c=OP_N):
    """Plain FP32 SGEMM of the same inputs; C updated in place."""
    A = _f32(A)
    B = _u16(B)
    rc = lib().oracle_sgemm(op_a, op_b, m, n, k, alpha, _ptr(A), lda, _ptr(B), ldb, beta,
                            _ptr(C), ldc, op_c)
    if rc != 0:
        raise MemoryError("oracle_sgemm: allocation failed")
    return C


def cpu_gemm(A, B, m, n, k, dtype=np.float64) -> np.ndarray:
    """Plain OpenMP GEMM C = A B (column-major flat buffers, A m x k, B k x n) in FP32 or
    FP64: the timed CPU baseline, not a checker. Returns C flat (ld = m)."""
    A = np.ascontiguousarray(A, dtype=dtype)
    B = np.ascontiguousarray(B, dtype=dtype)
    C = np.empty(m * n, dtype=dtype)
    fn = lib().oracle_cpu_dgemm if dtype == np.float64 else lib().oracle_cpu_sgemm
    fn(m, n, k, _ptr(A), m, _ptr(B), k, _ptr(C), m)
    return C


def num_threads() -> int:
    return lib().oracle_num_threads()


def logical_c(C, m, n, ldc, op_c=OP_N) -> np.ndarray:
    """(m, n) view of a column-major C buffer (op_c == op_t stores it transposed)."""
    if op_c == OP_N:
        return np.asarray(C).reshape(-1)[: ldc * n].reshape(n, ldc)[:, :m].T
    return np.asarray(C).reshape(-1)[: ldc * m].reshape(m, ldc)[:, :n]


def rel_fro(x, ref) -> float:
    """Relative Frobenius error over entries that are finite in both."""
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    mask = np.isfinite(x) & np.isfinite(ref)
    den = np.linalg.norm(ref[mask])
    num = np.linalg.norm((x - ref)[mask])
    return float(num / den) if den > 0 else float(num)
