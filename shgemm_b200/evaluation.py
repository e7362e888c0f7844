"""Error measurement on the GPU (FP64), the role mateval plays in the reference
(test/shgemm_test.cu:91-100): an FP64 GEMM of the same FP32/binary16 inputs and
FP64 norm reductions. FP64 appears only here, never in the SHGEMM kernels."""
from __future__ import annotations

import ctypes

import torch

from . import Handle, ShgemmError, _addr, lib, op_n


def fp64_product(h: Handle, op_a: int, op_b: int, m: int, n: int, k: int, a, lda: int, b, ldb: int,
                 a_is_fp32: bool = True) -> torch.Tensor:
    """op(A) op(B) in FP64 as an (m*n,) column-major tensor (ld = m) on the GPU."""
    c64 = torch.empty(m * n, dtype=torch.float64, device=f"cuda:{h.device}")
    fn = lib().shgemm_b200_eval_dgemm if a_is_fp32 else lib().shgemm_b200_eval_dgemm_hs
    st = fn(h.ptr, op_a, op_b, m, n, k, _addr(a), lda, _addr(b), ldb, _addr(c64))
    if st != 0:
        raise ShgemmError(st, "eval_dgemm")
    return c64


def error(h: Handle, m: int, n: int, c, ldc: int, c64, alpha: float = 1.0, beta: float = 0.0, c0=None,
          op_c: int = op_n) -> dict:
    """Relative Frobenius and max relative error of C against alpha*C64 + beta*C0."""
    out = (ctypes.c_double * 4)()
    st = lib().shgemm_b200_eval_error(h.ptr, m, n, _addr(c), ldc, op_c, _addr(c64), alpha, beta, _addr(c0), out)
    if st != 0:
        raise ShgemmError(st, "eval_error")
    diff, ref, mx, mismatch = out[0], out[1], out[2], out[3]
    return {"rel_fro": diff / ref if ref > 0 else diff, "max_rel": mx, "nonfinite_mismatch": int(mismatch)}
