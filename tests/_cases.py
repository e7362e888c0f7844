"""Shared helpers of the parity tests: seeded column-major inputs, GPU calls
through the C ABI, and the oracle comparisons."""
from __future__ import annotations

import numpy as np

import oracle

# One binary32 ulp-scale floor on relative errors (tiny products can be exact
# in the oracle but not in the tensor core's accumulation order).
ULP_FLOOR = 4 * 2.0 ** -24


def stored_shape(op, rows, cols, ld):
    """Number of elements of a column-major buffer holding op(X) (rows x cols) with leading dimension ld."""
    return ld * (cols if op == oracle.OP_N else rows)


def make_inputs(rng, m, n, k, op_a, op_b, op_c, dist="uniform", pad=0):
    lda = (m if op_a == oracle.OP_N else k) + pad
    ldb = (k if op_b == oracle.OP_N else n) + pad
    ldc = (m if op_c == oracle.OP_N else n) + pad
    na = max(1, stored_shape(op_a, m, k, lda))
    nb = max(1, stored_shape(op_b, k, n, ldb))
    nc = max(1, stored_shape(op_c, m, n, ldc))
    if dist == "uniform":
        A = rng.uniform(-1, 1, na).astype(np.float32)
        B = rng.uniform(-1, 1, nb).astype(np.float16)
    elif dist == "wide":  # FP32 operand N(0,1) * 2^U(-15,15), FP16 operand N(0,1)
        A = (rng.standard_normal(na) * np.exp2(rng.uniform(-15, 15, na))).astype(np.float32)
        B = rng.standard_normal(nb).astype(np.float16)
    elif dist == "positive":  # the reference tests' curand uniform (0, 1]
        A = rng.uniform(0, 1, na).astype(np.float32)
        B = rng.uniform(0, 1, nb).astype(np.float16)
    else:
        raise ValueError(dist)
    C = rng.uniform(-1, 1, nc).astype(np.float32)
    return dict(A=A, B=B, C=C, lda=lda, ldb=ldb, ldc=ldc)


def make_inputs_with_ld(rng, m, n, k, op_a, op_b, op_c, lda, ldb, ldc, dist="uniform"):
    """make_inputs with explicit leading dimensions."""
    na = max(1, stored_shape(op_a, m, k, lda))
    nb = max(1, stored_shape(op_b, k, n, ldb))
    nc = max(1, stored_shape(op_c, m, n, ldc))
    A = rng.uniform(-1, 1, na).astype(np.float32)
    B = rng.uniform(-1, 1, nb).astype(np.float16)
    C = rng.uniform(-1, 1, nc).astype(np.float32)
    return dict(A=A, B=B, C=C, lda=lda, ldb=ldb, ldc=ldc)


def run_gpu(h, tc, op_a, op_b, m, n, k, alpha, inp, beta, op_c, hs=False):
    """Calls shgemm (or hsgemm with hs=True) on the GPU; returns the C buffer as numpy."""
    import torch

    import shgemm_b200 as sg

    dev = f"cuda:{h.device}"
    A = torch.from_numpy(inp["A"]).to(dev)
    B = torch.from_numpy(inp["B"].view(np.int16)).to(dev).view(torch.float16)
    C = torch.from_numpy(inp["C"].copy()).to(dev)
    if hs:
        # hsgemm: A binary16, B FP32 -- the caller passes them in that role
        level = sg.hsgemm(h, op_a, op_b, m, n, k, alpha, B, inp["ldb"], A, inp["lda"], beta, C, inp["ldc"], tc, op_c)
    else:
        level = sg.shgemm(h, op_a, op_b, m, n, k, alpha, A, inp["lda"], B, inp["ldb"], beta, C, inp["ldc"], tc, op_c)
    torch.cuda.synchronize()
    assert h.check_error() == 0
    return C.cpu().numpy(), level


def run_oracle(tc, op_a, op_b, m, n, k, alpha, inp, beta, op_c, chunk):
    C = inp["C"].copy()
    oracle.shgemm(tc, op_a, op_b, m, n, k, alpha, inp["A"], inp["lda"], inp["B"], inp["ldb"], beta, C, inp["ldc"],
                  op_c, chunk)
    return C


def fp64(op_a, op_b, m, n, k, alpha, inp, beta, op_c):
    return oracle.dgemm_ref(op_a, op_b, m, n, k, alpha, inp["A"], inp["lda"], inp["B"], inp["ldb"], beta, inp["C"],
                            inp["ldc"], op_c)


def sgemm(op_a, op_b, m, n, k, alpha, inp, beta, op_c):
    C = inp["C"].copy()
    oracle.sgemm(op_a, op_b, m, n, k, alpha, inp["A"], inp["lda"], inp["B"], inp["ldb"], beta, C, inp["ldc"], op_c)
    return C


def parity_report(gpu_c, oracle_c, ref64, sgemm_c, m, n, ldc, op_c):
    g = oracle.logical_c(gpu_c, m, n, ldc, op_c)
    o = oracle.logical_c(oracle_c, m, n, ldc, op_c)
    s = oracle.logical_c(sgemm_c, m, n, ldc, op_c)
    return dict(
        e_gpu=oracle.rel_fro(g, ref64),
        e_oracle=oracle.rel_fro(o, ref64),
        e_sgemm=oracle.rel_fro(s, ref64),
        d_gpu_oracle=oracle.rel_fro(g, o),
        finite_mask_equal=bool(np.array_equal(np.isfinite(g), np.isfinite(o))),
    )


def assert_parity(r):
    """Parity bar: same non-finite mask as the restated reference algorithm; the GPU's
    error against FP64 within 2x the restated algorithm's own error (plus an ulp-level
    floor); and within 2x plain FP32 SGEMM's error."""
    assert r["finite_mask_equal"], r
    assert r["e_gpu"] <= 2.0 * r["e_oracle"] + ULP_FLOOR, r
    assert r["e_gpu"] <= 2.0 * r["e_sgemm"] + ULP_FLOOR, r
