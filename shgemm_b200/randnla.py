"""Randomized linear algebra on top of the SHGEMM sketch: a range finder and a
randomized SVD (Halko, Martinsson and Tropp, "Finding structure with randomness",
SIAM Review 2011, algorithms 4.1/4.4 and 5.1). The large products -- the sketch
Y = A Omega, the power iterations A^T Q and A Z, and the projection A^T Q -- run
through this library's SHGEMM on the GPU (FP32 A, binary16 second operand, the
error-corrected hi/lo split); only the thin QR and the small SVD use torch.

The reference (enp1s0/shgemm) motivates SHGEMM with exactly this use -- random
projections of an FP32 matrix by a low-precision Gaussian matrix (README.md) -- but
ships no such consumer; these functions are the next step on top of its hot path.

The orthonormal bases that re-enter a product as its binary16 operand are rounded to
binary16 (entries of size 1/sqrt(m), 11 significant bits); the FP32 operand A is never
rounded beyond SHGEMM's own split.
"""
from __future__ import annotations

import math

import torch

from . import Handle, fp16, op_n, op_t, shgemm
from . import server as _srv


def _omega(k: int, cols: int, seed: int, stream) -> tuple[torch.Tensor, int]:
    """k x cols Gaussian N(0, 1/cols) in binary16, column-major with a 16-byte leading dimension."""
    ld = (k + 7) // 8 * 8
    om = torch.empty(cols * ld, device="cuda", dtype=torch.float16)
    _srv.generate_omega(om, ld, k, cols, _srv.GAUSSIAN, seed, 1.0 / math.sqrt(cols), False, stream=stream)
    return om, ld


def _as_fp16_colmajor(Q: torch.Tensor) -> tuple[torch.Tensor, int]:
    """A rows x cols FP32 torch matrix as a binary16 column-major buffer with a 16-byte leading dimension."""
    rows, cols = Q.shape
    ld = (rows + 7) // 8 * 8
    buf = torch.zeros(cols, ld, device=Q.device, dtype=torch.float16)
    buf[:, :rows] = Q.T.to(torch.float16)
    return buf.reshape(-1), ld


def _orth(Ybuf: torch.Tensor, rows: int, cols: int) -> torch.Tensor:
    """Orthonormal basis (rows x cols, FP32) of a column-major rows x cols buffer."""
    Y = Ybuf.view(cols, rows).T
    return torch.linalg.qr(Y, mode="reduced")[0]


def range_finder(h: Handle, A, m: int, k: int, lda: int, rank: int, oversample: int = 10, power_iters: int = 0,
                 compute_type: int = fp16, seed: int = 0) -> torch.Tensor:
    """Orthonormal Q (m x l, l = rank + oversample) with range(Q) ~ range(A).

    A: FP32 column-major m x k device matrix (a torch CUDA tensor or address), leading
    dimension lda. Y = A Omega with a Gaussian binary16 Omega (k x l, generated on the device),
    then `power_iters` rounds of Z = A^T Q, Q = orth(A Z) (all products through SHGEMM).
    """
    stream = torch.cuda.current_stream()
    h.set_stream(stream)
    l = min(rank + oversample, m, k)
    om, ldo = _omega(k, l, seed, stream)
    Y = torch.empty(l * m, device="cuda", dtype=torch.float32)
    shgemm(h, op_n, op_n, m, l, k, 1.0, A, lda, om, ldo, 0.0, Y, m, compute_type)
    Q = _orth(Y, m, l)
    for _ in range(power_iters):
        q16, ldq = _as_fp16_colmajor(Q)
        Z = torch.empty(l * k, device="cuda", dtype=torch.float32)
        shgemm(h, op_t, op_n, k, l, m, 1.0, A, lda, q16, ldq, 0.0, Z, k, compute_type)  # A^T Q
        Zq = _orth(Z, k, l)
        z16, ldz = _as_fp16_colmajor(Zq)
        shgemm(h, op_n, op_n, m, l, k, 1.0, A, lda, z16, ldz, 0.0, Y, m, compute_type)  # A Z
        Q = _orth(Y, m, l)
    return Q


def rsvd(h: Handle, A, m: int, k: int, lda: int, rank: int, oversample: int = 10, power_iters: int = 1,
         compute_type: int = fp16, seed: int = 0):
    """Randomized truncated SVD A ~ U diag(S) V^T with `rank` terms (U: m x rank, S: rank, V: k x rank).

    Q from `range_finder`; the projection B^T = A^T Q (k x l) through SHGEMM; the small SVD of B
    with torch; U = Q U_B.
    """
    Q = range_finder(h, A, m, k, lda, rank, oversample, power_iters, compute_type, seed)
    l = Q.shape[1]
    q16, ldq = _as_fp16_colmajor(Q)
    Bt = torch.empty(l * k, device="cuda", dtype=torch.float32)
    shgemm(h, op_t, op_n, k, l, m, 1.0, A, lda, q16, ldq, 0.0, Bt, k, compute_type)  # A^T Q = B^T
    B = Bt.view(l, k)  # row-major l x k == (A^T Q)^T
    Ub, S, Vt = torch.linalg.svd(B, full_matrices=False)
    U = Q @ Ub[:, :rank]
    return U, S[:rank], Vt[:rank].T
