"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Mirrors the reference's test programs (test/shgemm_test.cu: every op_a x op_b x
op_c x compute type; test/exponent_test.cu: exponent ranges; test/
shgemm_k_slicing_test.cu: long k), at sizes the oracle finishes in seconds,
plus the edge cases they do not cover (ragged shapes, alpha/beta, padded
leading dimensions, k = 0, hsgemm).
"""
import os

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


def _parity(h, tc, op_a, op_b, op_c, m, n, k, alpha=1.0, beta=0.0, dist="uniform", pad=0, seed=0):
    rng = np.random.default_rng(seed)
    inp = K.make_inputs(rng, m, n, k, op_a, op_b, op_c, dist=dist, pad=pad)
    gpu_c, level = K.run_gpu(h, tc, op_a, op_b, m, n, k, alpha, inp, beta, op_c)
    orc = K.run_oracle(tc, op_a, op_b, m, n, k, alpha, inp, beta, op_c, chunk=0)
    ref = K.fp64(op_a, op_b, m, n, k, alpha, inp, beta, op_c)
    sg_c = K.sgemm(op_a, op_b, m, n, k, alpha, inp, beta, op_c)
    r = K.parity_report(gpu_c, orc, ref, sg_c, m, n, inp["ldc"], op_c)
    r["level"] = level
    return r, gpu_c, inp


OPS = [(a, b) for a in (0, 1) for b in (0, 1)]


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
@pytest.mark.parametrize("op_a,op_b", OPS)
@pytest.mark.parametrize("op_c", [0, 1])
def test_square_1024(h, tc, op_a, op_b, op_c):
    """Config 1 shape (1024^3) for every op combination (test/shgemm_test.cu:276-306)."""
    r, _, _ = _parity(h, tc, op_a, op_b, op_c, 1024, 1024, 1024)
    K.assert_parity(r)


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
@pytest.mark.parametrize("op_a,op_b", OPS)
@pytest.mark.parametrize("mnk", [(1, 1, 1), (7, 5, 3), (33, 17, 70), (129, 65, 257), (200, 300, 1000),
                                 (128, 128, 64), (257, 130, 4097)])
def test_ragged_shapes(h, tc, op_a, op_b, mnk):
    m, n, k = mnk
    r, _, _ = _parity(h, tc, op_a, op_b, (op_a + op_b) % 2, m, n, k, seed=m + n + k)
    K.assert_parity(r)


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
def test_alpha_beta_padded_ld(h, tc):
    r, _, _ = _parity(h, tc, 0, 1, 0, 300, 200, 500, alpha=-1.5, beta=0.5, pad=8, seed=3)
    K.assert_parity(r)
    r, _, _ = _parity(h, tc, 1, 0, 1, 300, 200, 500, alpha=0.25, beta=2.0, pad=16, seed=4)
    K.assert_parity(r)


def test_beta_zero_does_not_read_c(h):
    import torch

    import shgemm_b200 as sg

    m = n = k = 256
    rng = np.random.default_rng(9)
    A = torch.from_numpy(rng.uniform(-1, 1, m * k).astype(np.float32)).cuda()
    B = torch.from_numpy(rng.uniform(-1, 1, k * n).astype(np.float16).view(np.int16)).cuda().view(torch.float16)
    C = torch.full((m * n,), float("nan"), device="cuda")
    sg.shgemm(h, 0, 0, m, n, k, 1.0, A, m, B, k, 0.0, C, m, sg.fp16)
    torch.cuda.synchronize()
    assert torch.isfinite(C).all()


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
def test_permutation_b_is_bit_exact(h, tc):
    """B = a column permutation: every C entry is one split element folded back,
    hi + lo * 2^-11, so the GPU must equal the oracle bit for bit."""
    rng = np.random.default_rng(21)
    m, k = 300, 192
    n = k
    A = (rng.standard_normal(m * k) * np.exp2(rng.uniform(-20, 10, m * k))).astype(np.float32)
    perm = rng.permutation(k)
    Bm = np.zeros((k, n), np.float16)
    Bm[perm, np.arange(n)] = 1.0
    inp = dict(A=A, B=Bm.ravel(order="F"), C=np.zeros(m * n, np.float32), lda=m, ldb=k, ldc=m)
    gpu_c, _ = K.run_gpu(h, tc, 0, 0, m, n, k, 1.0, inp, 0.0, 0)
    orc = K.run_oracle(tc, 0, 0, m, n, k, 1.0, inp, 0.0, 0, chunk=64 if tc == oracle.FP16 else 32)
    same = (gpu_c.view(np.uint32) == orc.view(np.uint32)) | (np.isnan(gpu_c) & np.isnan(orc))
    assert same.all(), np.argwhere(~same)[:5]


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
def test_exact_gemm_fixture(h, tc):
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "gemm_exact.npz"))
    m, n, k = int(g["m"]), int(g["n"]), int(g["k"])
    inp = dict(A=g["A"], B=g["B"].view(np.float16), C=np.zeros(m * n, np.float32), lda=m, ldb=k, ldc=m)
    gpu_c, _ = K.run_gpu(h, tc, 0, 0, m, n, k, 1.0, inp, 0.0, 0)
    assert np.array_equal(gpu_c.astype(np.float64), g["C"])


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
@pytest.mark.parametrize("op_a,op_b", OPS)
def test_wide_exponent_nonfinite_mask(h, tc, op_a, op_b):
    """Config 2's FP32 distribution N(0,1) 2^U(-15,15): in fp16 mode elements past
    65504 overflow to inf in hi (no rescaling, like the reference) and the
    non-finite pattern must match the oracle exactly."""
    r, _, _ = _parity(h, tc, op_a, op_b, 0, 256, 192, 640, dist="wide", beta=0.5, seed=17)
    K.assert_parity(r)


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
@pytest.mark.parametrize("lo_e,hi_e", [(-15, 14), (-36, -15), (-100, -36)])
def test_exponent_ranges(h, tc, lo_e, hi_e):
    """test/exponent_test.cu:249-252: A = 2^U(lo, hi), B uniform (0, 1]; the lo term
    carries the value once hi underflows and the GPU must follow the oracle."""
    rng = np.random.default_rng(lo_e & 0xFF)
    m, n, k = 256, 256, 256
    A = np.exp2(rng.uniform(lo_e, hi_e, m * k)).astype(np.float32)
    B = rng.uniform(0, 1, k * n).astype(np.float16)
    inp = dict(A=A, B=B, C=np.zeros(m * n, np.float32), lda=m, ldb=k, ldc=m)
    gpu_c, _ = K.run_gpu(h, tc, 0, 0, m, n, k, 1.0, inp, 0.0, 0)
    orc = K.run_oracle(tc, 0, 0, m, n, k, 1.0, inp, 0.0, 0, chunk=0)
    ref = K.fp64(0, 0, m, n, k, 1.0, inp, 0.0, 0)
    e_g = oracle.rel_fro(oracle.logical_c(gpu_c, m, n, m), ref)
    e_o = oracle.rel_fro(oracle.logical_c(orc, m, n, m), ref)
    # where the split loses bits (deep underflow) both lose the same ones
    assert e_g <= 2.0 * e_o + K.ULP_FLOOR, (e_g, e_o)


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
@pytest.mark.parametrize("op_a,op_b", OPS)
def test_hsgemm(h, tc, op_a, op_b):
    """hsgemm through the transposition identity (include/shgemm/shgemm.hpp:121-157)."""
    rng = np.random.default_rng(31)
    m, n, k = 96, 160, 320
    lda = m if op_a == 0 else k
    ldb = k if op_b == 0 else n
    Ah = rng.uniform(-1, 1, lda * (k if op_a == 0 else m)).astype(np.float16)
    Bf = rng.uniform(-1, 1, ldb * (n if op_b == 0 else k)).astype(np.float32)
    inp = dict(A=Bf, B=Ah, C=np.zeros(m * n, np.float32), lda=ldb, ldb=lda, ldc=m)
    gpu_c, _ = K.run_gpu(h, tc, op_a, op_b, m, n, k, 1.0, inp, 0.0, 0, hs=True)
    C = np.zeros(m * n, np.float32)
    oracle.hsgemm(tc, op_a, op_b, m, n, k, 1.0, Ah, lda, Bf, ldb, 0.0, C, m, 0)
    Am = Ah.astype(np.float64).reshape(-1, lda).T  # columns of the stored buffer
    Aop = Am[:m, :k] if op_a == 0 else Am[:k, :m].T
    Bm = Bf.astype(np.float64).reshape(-1, ldb).T
    Bop = Bm[:k, :n] if op_b == 0 else Bm[:n, :k].T
    ref = Aop @ Bop
    e_g = oracle.rel_fro(oracle.logical_c(gpu_c, m, n, m), ref)
    e_o = oracle.rel_fro(oracle.logical_c(C, m, n, m), ref)
    assert e_g <= 2.0 * e_o + K.ULP_FLOOR, (e_g, e_o)


def test_k_zero_scales_c(h):
    r, gpu_c, inp = _parity(h, oracle.FP16, 0, 0, 0, 64, 48, 0, beta=0.5)
    assert np.array_equal(gpu_c, (inp["C"] * np.float32(0.5)).astype(np.float32))


@pytest.mark.parametrize("level", [0, 1])
def test_kernel_level_fixing(h, level):
    import shgemm_b200 as sg

    sg.enable_kernel_level_fixing(h, level)
    try:
        r, _, _ = _parity(h, oracle.FP16, 0, 0, 0, 320, 192, 384, seed=level)
    finally:
        sg.disable_kernel_level_fixing(h)
    assert r["level"] == level
    K.assert_parity(r)


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
def test_unaligned_operands_go_through_staging(h, tc):
    """Leading dimensions / base addresses TMA cannot address (the reference accepts
    any ld, src/dmem_accessor.hpp:15-146) are staged into the workspace."""
    import torch

    import shgemm_b200 as sg

    rng = np.random.default_rng(41)
    m, n, k = 75, 61, 333
    inp = K.make_inputs(rng, m, n, k, 0, 0, 0, pad=3)  # lda = 78, ldb = 336: unaligned A
    A = np.concatenate([[np.float32(0)], inp["A"]])  # shift the base by 4 bytes
    B = np.concatenate([[np.float16(0)], inp["B"]])  # and B's by 2 bytes
    dA = torch.from_numpy(A).cuda()
    dB = torch.from_numpy(B.view(np.int16)).cuda().view(torch.float16)
    dC = torch.from_numpy(inp["C"].copy()).cuda()
    sg.shgemm(h, 0, 0, m, n, k, 1.0, dA.data_ptr() + 4, inp["lda"], dB.data_ptr() + 2, inp["ldb"], 0.25, dC,
              inp["ldc"], tc)
    torch.cuda.synchronize()
    gpu_c = dC.cpu().numpy()
    orc = K.run_oracle(tc, 0, 0, m, n, k, 1.0, inp, 0.25, 0, chunk=0)
    ref = K.fp64(0, 0, m, n, k, 1.0, inp, 0.25, 0)
    sgc = K.sgemm(0, 0, m, n, k, 1.0, inp, 0.25, 0)
    K.assert_parity(K.parity_report(gpu_c, orc, ref, sgc, m, n, inp["ldc"], 0))


def test_staging_in_k_slabs_with_small_workspace(cuda_device):
    """With a workspace too small for the whole staged operand the product runs in
    k-slabs accumulated into C."""
    import shgemm_b200 as sg

    hd = sg.Handle(0)
    try:
        hd.set_workspace_size(1 << 20)
        r, _, _ = _parity(hd, oracle.FP16, 1, 0, 0, 301, 77, 3001, beta=0.5, seed=8)
        K.assert_parity(r)
    finally:
        hd.close()


def test_bounded_wait_times_out_and_context_survives(h):
    """A wait on an mbarrier that nothing arrives at gives up after its limit, the
    host reads the timeout status, and the context keeps working."""
    st, code = h.selftest_wait_timeout(20000)
    assert st == 5 and code != 0
    r, _, _ = _parity(h, oracle.FP16, 0, 0, 0, 128, 128, 128)
    K.assert_parity(r)


def test_launch_count_increments(h):
    before = h.launch_count()
    _parity(h, oracle.FP16, 0, 0, 0, 64, 64, 64)
    assert h.launch_count() > before


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
@pytest.mark.parametrize("op_a,op_b", [(1, 0), (0, 0)])
def test_split_k_deterministic_and_matches(h, tc, op_a, op_b):
    """Long-k, few-tile shapes take the deterministic split-K path (the reference's
    k-slicing, src/shgemm.cu:532-609, which reduces with atomics): results are
    bit-identical across runs and within the parity bar; beta != 0 is supported."""
    import shgemm_b200 as sg

    m, n, k = 256, 192, 16384
    rng = np.random.default_rng(77)
    inp = K.make_inputs(rng, m, n, k, op_a, op_b, 1)
    c1, _ = K.run_gpu(h, tc, op_a, op_b, m, n, k, 1.0, inp, 0.5, 1)
    c2, _ = K.run_gpu(h, tc, op_a, op_b, m, n, k, 1.0, inp, 0.5, 1)
    assert np.array_equal(c1.view(np.uint32), c2.view(np.uint32))
    orc = K.run_oracle(tc, op_a, op_b, m, n, k, 1.0, inp, 0.5, 1, chunk=0)
    ref = K.fp64(op_a, op_b, m, n, k, 1.0, inp, 0.5, 1)
    sgc = K.sgemm(op_a, op_b, m, n, k, 1.0, inp, 0.5, 1)
    K.assert_parity(K.parity_report(c1, orc, ref, sgc, m, n, inp["ldc"], 1))
    # forcing one slice (no split-K) gives a result within the same bar
    h.set_config(sg.CFG_SPLIT_K, 1)
    try:
        c3, _ = K.run_gpu(h, tc, op_a, op_b, m, n, k, 1.0, inp, 0.5, 1)
    finally:
        h.set_config(sg.CFG_SPLIT_K, 0)
    K.assert_parity(K.parity_report(c3, orc, ref, sgc, m, n, inp["ldc"], 1))
    assert not np.array_equal(c1.view(np.uint32), c3.view(np.uint32))  # the split path really ran


@pytest.mark.parametrize("op_a", [0, 1])
@pytest.mark.parametrize("mnk", [(1000, 700, 3000), (128, 256, 64), (385, 513, 1111), (1000, 700, 2080), (385, 513, 1024)])
def test_tensor_memory_kernel_matches_shared_memory_kernel(h, op_a, mnk):
    """The 128x256 binary16 kernel that keeps hi/lo in tensor memory computes the same
    products in the same order as the shared-memory operand kernel: bit-identical C,
    and within the parity bar of the restated reference. With op_a = T and k a multiple
    of 32 (2080: an odd count of 32-wide halves, the last step half past k) the FP32
    operand arrives through the paired 3-D box; other k take the two 2-D boxes."""
    import shgemm_b200 as sg

    m, n, k = mnk
    sg.enable_kernel_level_fixing(h, 1)  # 128 x 256 tiles
    try:
        r_tm, c_tm, inp = _parity(h, oracle.FP16, op_a, 0, 0, m, n, k, beta=0.5, dist="wide", seed=m + op_a)
        h.set_config(sg.CFG_TILE_KERNEL, 1)
        try:
            r_sm, c_sm, _ = _parity(h, oracle.FP16, op_a, 0, 0, m, n, k, beta=0.5, dist="wide", seed=m + op_a)
        finally:
            h.set_config(sg.CFG_TILE_KERNEL, 0)
    finally:
        sg.disable_kernel_level_fixing(h)
    K.assert_parity(r_tm)
    K.assert_parity(r_sm)
    assert np.array_equal(c_tm.view(np.uint32), c_sm.view(np.uint32))


@pytest.mark.parametrize("op_a", [0, 1])
@pytest.mark.parametrize("k", [1000, 8224])
def test_wide_pitch_b_k_blocks(h, op_a, k):
    """A binary16 operand whose columns lie >= 1 MiB apart is re-laid out as contiguous
    k-blocks in the workspace before the tensor-memory kernel runs (ragged last block
    zero-filled, n below one tile, split-K at k = 8224): C is bit-identical to the same
    values stored with a compact leading dimension, which loads B in place."""
    import shgemm_b200 as sg

    m, n = 300, 136
    rng = np.random.default_rng(k + op_a)
    inp = K.make_inputs(rng, m, n, k, op_a, 0, 0, dist="wide")
    ld_wide = (1 << 19) + 8  # 1 MiB + 16 bytes between columns
    wide = np.zeros(n * ld_wide, dtype=np.float16)
    wide.reshape(n, ld_wide)[:, :k] = inp["B"].reshape(n, k)
    inp_w = dict(inp, B=wide, ldb=ld_wide)
    sg.enable_kernel_level_fixing(h, 1)  # 128 x 256 tiles: the tensor-memory kernel
    try:
        c_compact, _ = K.run_gpu(h, oracle.FP16, op_a, 0, m, n, k, 1.0, inp, 0.5, 0)
        c_wide, _ = K.run_gpu(h, oracle.FP16, op_a, 0, m, n, k, 1.0, inp_w, 0.5, 0)
    finally:
        sg.disable_kernel_level_fixing(h)
    assert np.array_equal(c_compact.view(np.uint32), c_wide.view(np.uint32))
    orc = K.run_oracle(oracle.FP16, op_a, 0, m, n, k, 1.0, inp, 0.5, 0, chunk=0)
    ref = K.fp64(op_a, 0, m, n, k, 1.0, inp, 0.5, 0)
    sgc = K.sgemm(op_a, 0, m, n, k, 1.0, inp, 0.5, 0)
    K.assert_parity(K.parity_report(c_wide, orc, ref, sgc, m, n, inp["ldc"], 0))


@pytest.mark.parametrize("dist", ["uniform", "wide", "positive"])
@pytest.mark.parametrize("op_a", [0, 1])
def test_k_chunk_128(h, dist, op_a):
    """SHGEMM_CFG_K_CHUNK = 128 (one FP32 drain per 128 k in the tensor-memory kernel, an odd
    step count included): same non-finite mask as the restated reference and relative error
    within 2x plain FP32 SGEMM's (the library's accuracy target); the 64-k default meets the tighter
    2x-the-restated-algorithm bar as well."""
    import shgemm_b200 as sg

    m, n, k = 1000, 700, 4000  # 63 k-steps: the last chunk has one step
    sg.enable_kernel_level_fixing(h, 1)
    try:
        r64, c64, inp = _parity(h, oracle.FP16, op_a, 0, 0, m, n, k, beta=0.5, dist=dist, seed=5 + op_a)
        h.set_config(sg.CFG_K_CHUNK, 128)
        try:
            r128, c128, _ = _parity(h, oracle.FP16, op_a, 0, 0, m, n, k, beta=0.5, dist=dist, seed=5 + op_a)
        finally:
            h.set_config(sg.CFG_K_CHUNK, 64)
    finally:
        sg.disable_kernel_level_fixing(h)
    K.assert_parity(r64)
    assert r128["finite_mask_equal"], r128
    assert r128["e_gpu"] <= 2.0 * r128["e_sgemm"] + K.ULP_FLOOR, r128
    print(f"\n{dist} op_a={op_a}: e(64)={r64['e_gpu']:.3e} e(128)={r128['e_gpu']:.3e} "
          f"oracle={r64['e_oracle']:.3e} sgemm={r64['e_sgemm']:.3e}")
    # The oracle's model of these kernels' arithmetic (B200MODEL: each MMA truncating its terms
    # to 26 bits below the largest nominal exponent) on the same inputs and drain: the GPU's
    # error equals the model's (the model reproduced the twelve errors of this test to their
    # printed four digits); the share of bit-identical entries is printed.
    ref = K.fp64(op_a, 0, m, n, k, 1.0, inp, 0.5, 0)
    for chunk, r, c_gpu in ((64, r64, c64), (128, r128, c128)):
        cm = inp["C"].copy()
        oracle.shgemm(oracle.FP16, op_a, 0, m, n, k, 1.0, inp["A"], inp["lda"], inp["B"], inp["ldb"], 0.5, cm,
                      inp["ldc"], 0, chunk, oracle.B200MODEL)
        e_model = oracle.rel_fro(oracle.logical_c(cm, m, n, inp["ldc"]), ref)
        same = float(np.mean(np.asarray(c_gpu, dtype=np.float32).view(np.uint32) == cm.view(np.uint32)))
        print(f"{dist} op_a={op_a} {chunk}-k drain: error gpu/model {r['e_gpu'] / e_model:.5f}, "
              f"{100 * same:.2f} % of entries bit-identical to the model")
        assert abs(r["e_gpu"] / e_model - 1) < 2e-3, (chunk, r["e_gpu"], e_model)


@pytest.mark.parametrize("op_a", [0, 1])
def test_tf32_widened_b_route(h, op_a):
    """TF32 calls whose 128x256 tiles fill the GPU widen B into the workspace and run the
    TF32 kernel that loads it unconverted: two launches, parity with the restated
    reference, and the same bar as the in-kernel-widening tile kernel."""
    import shgemm_b200 as sg

    m, n, k = 2048, 2560, 700
    before = h.launch_count()
    r, c_route, _ = _parity(h, oracle.TF32, op_a, 0, 0, m, n, k, beta=0.5, dist="wide", seed=31 + op_a)
    assert h.launch_count() - before == 2  # widen + TF32 kernel
    K.assert_parity(r)
    h.set_config(sg.CFG_TILE_KERNEL, 1)  # the tile kernel that widens B itself
    try:
        r_old, _, _ = _parity(h, oracle.TF32, op_a, 0, 0, m, n, k, beta=0.5, dist="wide", seed=31 + op_a)
    finally:
        h.set_config(sg.CFG_TILE_KERNEL, 0)
    K.assert_parity(r_old)
