"""shgemm_b200_shgemm_host: SHGEMM on host buffers with the copies overlapping the work.

The host entry point computes C in column blocks on the device entry point, so with
the tile size fixed and split-K off every element goes through the same kernel and the
same k order as one device call on the whole problem: results must be bit-identical.
Covers every op combination, ragged blocks, default and forced block widths,
page-locked and pageable host memory, k = 0, staging growth and release.
"""
import numpy as np
import pytest

import oracle
from tests import _cases as K

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h(cuda_device):
    import shgemm_b200 as sg

    hd = sg.Handle(0)
    yield hd
    hd.close()


def _host_call(h, tc, op_a, op_b, op_c, m, n, k, inp, alpha, beta, pinned):
    import torch

    import shgemm_b200 as sg

    C = inp["C"].copy()
    if pinned:
        A = torch.from_numpy(inp["A"]).pin_memory()
        B = torch.from_numpy(inp["B"].view(np.int16)).pin_memory()
        Ct = torch.from_numpy(C).pin_memory()
        level = sg.shgemm_host(h, op_a, op_b, m, n, k, alpha, A, inp["lda"], B, inp["ldb"], beta, Ct, inp["ldc"], tc,
                               op_c)
        torch.cuda.synchronize()
        out = Ct.numpy().copy()
    else:
        level = sg.shgemm_host(h, op_a, op_b, m, n, k, alpha, inp["A"], inp["lda"], inp["B"], inp["ldb"], beta, C,
                               inp["ldc"], tc, op_c)
        torch.cuda.synchronize()
        out = C
    assert h.check_error() == 0
    return out, level


def _same_plan(h):
    """Fixed 128 x 256 tiles and no split-K: per-element work independent of n."""
    import shgemm_b200 as sg

    sg.enable_kernel_level_fixing(h, 1)
    h.set_config(sg.CFG_SPLIT_K, 1)


def _default_plan(h):
    import shgemm_b200 as sg

    sg.disable_kernel_level_fixing(h)
    h.set_config(sg.CFG_SPLIT_K, 0)
    h.set_config(sg.CFG_HOST_BLOCK_COLS, 0)


@pytest.mark.parametrize("op_c", [0, 1])
@pytest.mark.parametrize("op_a,op_b", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_host_matches_device(h, op_a, op_b, op_c):
    """Three ragged column blocks (256, 256, 188), beta = 0.5, page-locked buffers:
    bit-identical to the device entry point, and within the parity bar of the oracle."""
    import shgemm_b200 as sg

    m, n, k = 300, 700, 1000
    rng = np.random.default_rng(11 + 4 * op_a + 2 * op_b + op_c)
    inp = K.make_inputs(rng, m, n, k, op_a, op_b, op_c, dist="wide")
    _same_plan(h)
    h.set_config(sg.CFG_HOST_BLOCK_COLS, 256)
    try:
        c_dev, _ = K.run_gpu(h, oracle.FP16, op_a, op_b, m, n, k, 1.0, inp, 0.5, op_c)
        c_host, _ = _host_call(h, oracle.FP16, op_a, op_b, op_c, m, n, k, inp, 1.0, 0.5, pinned=True)
    finally:
        _default_plan(h)
    assert np.array_equal(c_dev.view(np.uint32), c_host.view(np.uint32))
    orc = K.run_oracle(oracle.FP16, op_a, op_b, m, n, k, 1.0, inp, 0.5, op_c, chunk=0)
    ref = K.fp64(op_a, op_b, m, n, k, 1.0, inp, 0.5, op_c)
    sgc = K.sgemm(op_a, op_b, m, n, k, 1.0, inp, 0.5, op_c)
    K.assert_parity(K.parity_report(c_host, orc, ref, sgc, m, n, inp["ldc"], op_c))


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
def test_host_pageable_default_blocks(h, tc):
    """Pageable numpy buffers, padded leading dimensions, the default block width
    (four blocks of 256 at n = 1000), beta = 0: bit-identical to the device call."""
    m, n, k = 513, 1000, 777
    rng = np.random.default_rng(5 + tc)
    inp = K.make_inputs(rng, m, n, k, 0, 0, 0, dist="uniform", pad=3)
    _same_plan(h)
    try:
        c_dev, _ = K.run_gpu(h, tc, 0, 0, m, n, k, 0.75, inp, 0.0, 0)
        c_host, _ = _host_call(h, tc, 0, 0, 0, m, n, k, inp, 0.75, 0.0, pinned=False)
    finally:
        _default_plan(h)
    assert np.array_equal(c_dev.view(np.uint32), c_host.view(np.uint32))


def test_host_k0_and_staging_growth(h):
    """k = 0 gives C = beta C on the host buffer; a larger call afterwards grows the
    staging and two calls in a row agree; release frees it and the next call works."""
    import shgemm_b200 as sg

    m, n = 64, 96
    rng = np.random.default_rng(3)
    inp0 = K.make_inputs(rng, m, n, 0, 0, 0, 0)
    c0, _ = _host_call(h, oracle.FP16, 0, 0, 0, m, n, 0, inp0, 1.0, -2.0, pinned=True)
    want = (np.float32(-2.0) * inp0["C"]).astype(np.float32)
    assert np.array_equal(c0.view(np.uint32), want.view(np.uint32))

    m, n, k = 1024, 1536, 2048
    inp = K.make_inputs(rng, m, n, k, 1, 0, 0, dist="uniform")
    c1, _ = _host_call(h, oracle.FP16, 1, 0, 0, m, n, k, inp, 1.0, 0.5, pinned=True)
    c2, _ = _host_call(h, oracle.FP16, 1, 0, 0, m, n, k, inp, 1.0, 0.5, pinned=False)
    assert np.array_equal(c1.view(np.uint32), c2.view(np.uint32))
    c_dev, _ = K.run_gpu(h, oracle.FP16, 1, 0, m, n, k, 1.0, inp, 0.5, 0)
    rel = np.linalg.norm(c1 - c_dev) / np.linalg.norm(c_dev)
    assert rel < 1e-6  # the default plan may pick other split-K slices per block than for the whole C
    sg.release_host_staging(h)
    c3, _ = _host_call(h, oracle.FP16, 1, 0, 0, m, n, k, inp, 1.0, 0.5, pinned=True)
    assert np.array_equal(c1.view(np.uint32), c3.view(np.uint32))


def test_host_rejects_device_tensor(h):
    import torch

    import shgemm_b200 as sg

    a = torch.zeros(16, device="cuda")
    with pytest.raises(ValueError):
        sg.shgemm_host(h, 0, 0, 4, 4, 4, 1.0, a, 4, a, 4, 0.0, a, 4, oracle.FP16)


@pytest.mark.parametrize("op_a,op_b", [(0, 0), (1, 1)])
def test_hsgemm_host_matches_device(h, op_a, op_b):
    """hsgemm (A binary16, B FP32) on host buffers, two blocks: bit-identical to the
    device hsgemm under the same fixed plan."""
    import torch

    import shgemm_b200 as sg

    rng = np.random.default_rng(41 + op_a)
    m, n, k = 384, 200, 520
    lda = m if op_a == 0 else k
    ldb = k if op_b == 0 else n
    Ah = rng.uniform(-1, 1, lda * (k if op_a == 0 else m)).astype(np.float16)
    Bf = rng.uniform(-1, 1, ldb * (n if op_b == 0 else k)).astype(np.float32)
    inp = dict(A=Bf, B=Ah, C=rng.uniform(-1, 1, m * n).astype(np.float32), lda=ldb, ldb=lda, ldc=m)
    _same_plan(h)
    h.set_config(sg.CFG_HOST_BLOCK_COLS, 256)  # the internal shgemm's n is this call's m: blocks 256 + 128
    try:
        c_dev, _ = K.run_gpu(h, oracle.FP16, op_a, op_b, m, n, k, 1.0, inp, 0.5, 0, hs=True)
        Ch = torch.from_numpy(inp["C"].copy()).pin_memory()
        sg.hsgemm_host(h, op_a, op_b, m, n, k, 1.0, Ah, lda, Bf, ldb, 0.5, Ch, m, oracle.FP16)
        torch.cuda.synchronize()
        assert h.check_error() == 0
    finally:
        _default_plan(h)
    assert np.array_equal(c_dev.view(np.uint32), Ch.numpy().view(np.uint32))
