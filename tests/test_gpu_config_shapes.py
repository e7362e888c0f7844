"""Parity at the workload shapes themselves, not only at sizes the oracle runs whole.

* Large square SHGEMM / HSGEMM, m = n = k = 16384, op_n and op_t, binary16 and TF32
  compute, alpha = 1, beta = 0.5 with C uniform[-1, 1]; FP32 operand N(0,1) 2^U(-15,15)
  (the wide exponent range that exercises the lo term), binary16 operand N(0,1). With
  binary16 compute almost every row of that FP32 operand holds an entry >= 65520, whose hi
  part overflows (the reference's behaviour, checked through the non-finite mask), so the
  binary16 cases also run the reference's widest exponent-test range, +-2^U(-15,14)
  (test/exponent_test.cu:202-250, random signs), where every entry stays finite. The whole
  product runs on the GPU; a 256 x 256 block of C (rows and columns off the tile grid) is
  recomputed by the oracle from the same rows of op(A) and columns of op(B) over the full
  k = 16384 -- each entry of C depends on nothing else.
* The long-k sketch aspect: HSGEMM Y = Omega^T A with m = 256, n = 128, k = 2^20 (the
  internal SHGEMM is one tile row with split-K), whole, with and without the workspace that
  lets the long binary16 operand be re-laid out as k-blocks.

The bar is the one of the other parity tests, against the oracle that models the
reference's tensor-core accumulation (oracle.TCMODEL: each 16-k / 8-k hi fragment truncated
before its round-to-nearest add, lo in a truncating FP32 accumulator over all k,
src/wmmae_shgemm.hpp:86-124): same non-finite mask; relative Frobenius error against FP64
within 2x the model's and within 2x plain FP32 SGEMM's. Each test prints the GPU error
over both, the headroom of the 64-k drain at these k.
"""
import numpy as np
import pytest

import oracle
from tests import _cases as K

pytestmark = pytest.mark.gpu

N = 16384
R0, C0_ = 8000, 12000  # block origin: not a multiple of the 128 / 256 tile sizes
BLK = 256


@pytest.fixture(scope="module")
def square_inputs(cuda_device):
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(2)
    F = torch.randn(N * N, generator=g, device="cuda")
    F.mul_(torch.exp2(torch.empty(N * N, device="cuda").uniform_(-15, 15, generator=g)))
    H = torch.randn(N * N, generator=g, device="cuda").to(torch.float16)
    Cin = torch.empty(N * N, device="cuda").uniform_(-1, 1, generator=g)
    X = torch.exp2(torch.empty(N * N, device="cuda").uniform_(-15, 14, generator=g))
    X.mul_(torch.randn(N * N, generator=g, device="cuda").sign_())
    yield {"wide": F, "exp14": X}, H, Cin
    del F, H, Cin, X
    torch.cuda.empty_cache()


@pytest.fixture(scope="module")
def hbig(cuda_device):
    import shgemm_b200 as sg

    hd = sg.Handle(0)
    # room for the widened B of the TF32 route (n * k FP32) and for B's k-block re-layout
    hd.set_workspace_size(N * N * 4 + (64 << 20))
    yield hd
    hd.close()


def _logical(buf, op):
    """(rows x cols) logical view of a square column-major N x N buffer stored for op."""
    v = buf.view(N, N)  # v[j, i] = stored element (i, j)
    return v.T if op == 0 else v


def _colmajor_np(mat):
    """A (rows x cols) torch matrix as a flat column-major numpy array (ld = rows)."""
    return mat.T.contiguous().reshape(-1).cpu().numpy()


def _report(gpu_blk, tcm, ideal, ref, sgc):
    r = dict(
        e_gpu=oracle.rel_fro(gpu_blk, ref),
        e_oracle=oracle.rel_fro(tcm, ref),
        e_ideal=oracle.rel_fro(ideal, ref) if ideal is not None else float("nan"),
        e_sgemm=oracle.rel_fro(sgc, ref),
        finite_mask_equal=bool(np.array_equal(np.isfinite(gpu_blk), np.isfinite(tcm))),
        finite_fraction=float(np.isfinite(gpu_blk).mean()),
    )
    r["d_gpu_oracle"] = oracle.rel_fro(gpu_blk, tcm)
    return r


def _print(tag, r):
    hm = r["e_gpu"] / r["e_oracle"] if r["e_oracle"] else float("nan")
    hs = r["e_gpu"] / r["e_sgemm"] if r["e_sgemm"] else float("nan")
    print(f"\n{tag}: finite {r['finite_fraction']:.4f}  e_gpu {r['e_gpu']:.3e}  e_tcmodel {r['e_oracle']:.3e}  "
          f"e_ideal {r['e_ideal']:.3e}  e_sgemm {r['e_sgemm']:.3e}  gpu/tcmodel {hm:.3f}  gpu/sgemm {hs:.3f}")


@pytest.mark.parametrize("tc,dist", [(oracle.FP16, "wide"), (oracle.TF32, "wide"), (oracle.FP16, "exp14")],
                         ids=["fp16", "tf32", "fp16-exp14"])
@pytest.mark.parametrize("op", [0, 1])
@pytest.mark.parametrize("hs", [False, True], ids=["shgemm", "hsgemm"])
def test_square_16384_block(square_inputs, hbig, tc, dist, op, hs):
    import torch

    import shgemm_b200 as sg

    Fs, H, Cin = square_inputs
    F = Fs[dist]
    C = Cin.clone()
    alpha, beta = 1.0, 0.5
    if hs:  # A binary16 (m x k), B FP32 (k x n)
        sg.hsgemm(hbig, op, op, N, N, N, alpha, H, N, F, N, beta, C, N, tc)
    else:  # A FP32, B binary16
        sg.shgemm(hbig, op, op, N, N, N, alpha, F, N, H, N, beta, C, N, tc)
    torch.cuda.synchronize()
    assert hbig.check_error() == 0
    rows, cols = slice(R0, R0 + BLK), slice(C0_, C0_ + BLK)
    a_buf, b_buf = (H, F) if hs else (F, H)
    a_sub = _colmajor_np(_logical(a_buf, op)[rows, :])  # BLK x N, ld = BLK
    b_sub = _colmajor_np(_logical(b_buf, op)[:, cols])  # N x BLK, ld = N
    c0 = _colmajor_np(_logical(Cin, 0)[rows, cols])
    gpu_blk = _logical(C, 0)[rows, cols].cpu().numpy().astype(np.float64)
    del C

    def run(model):
        out = c0.copy()
        if hs:
            oracle.hsgemm(tc, 0, 0, BLK, BLK, N, alpha, a_sub, BLK, b_sub, N, beta, out, BLK, 0, 0, model)
        else:
            oracle.shgemm(tc, 0, 0, BLK, BLK, N, alpha, a_sub, BLK, b_sub, N, beta, out, BLK, 0, 0, model)
        return oracle.logical_c(out, BLK, BLK, BLK)

    tcm, ideal = run(oracle.TCMODEL), run(oracle.IDEAL)
    if hs:  # the FP64 product of binary16 A and FP32 B, through the same identity
        ref = oracle.dgemm_ref(1, 1, BLK, BLK, N, alpha, b_sub, N, a_sub, BLK, beta, c0, BLK, 1).T
    else:
        ref = oracle.dgemm_ref(0, 0, BLK, BLK, N, alpha, a_sub, BLK, b_sub, N, beta, c0, BLK, 0)
    if hs:
        sgc_buf = c0.copy()
        oracle.sgemm(1, 1, BLK, BLK, N, alpha, b_sub, N, a_sub, BLK, beta, sgc_buf, BLK, 1)
    else:
        sgc_buf = c0.copy()
        oracle.sgemm(0, 0, BLK, BLK, N, alpha, a_sub, BLK, b_sub, N, beta, sgc_buf, BLK, 0)
    sgc = oracle.logical_c(sgc_buf, BLK, BLK, BLK)
    r = _report(gpu_blk, tcm, ideal, ref, sgc)
    _print(f"{'hsgemm' if hs else 'shgemm'} {'NT'[op]}{'NT'[op]} {['fp16', 'tf32'][tc]} {dist} 16384^3 block", r)
    assert r["finite_mask_equal"], r
    if tc == oracle.TF32 or dist == "exp14":
        assert r["finite_fraction"] == 1.0  # no overflow: the check covers every entry
    assert r["e_gpu"] <= 2.0 * r["e_oracle"] + K.ULP_FLOOR, r
    assert r["e_gpu"] <= 2.0 * r["e_sgemm"] + K.ULP_FLOOR, r


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
@pytest.mark.parametrize("workspace", ["default", "k_blocks"])
def test_sketch_k_2_20(cuda_device, tc, workspace):
    """Y = Omega^T A by HSGEMM(op_t, op_n), m = 256, n = 128, k = 2^20: A low rank (rank 128,
    sigma_j = j^-2) plus N(0, 1e-6), Omega N(0, 1/256) binary16. The internal SHGEMM is
    shgemm(op_t, op_n, 128, 256, 2^20) with op_c = op_t: one tile row, deterministic split-K.
    "k_blocks": a workspace that also holds Omega re-laid out as contiguous 64-deep k-blocks
    (its columns lie 2 MiB apart), as the sketch benchmark sets it up."""
    import torch

    import shgemm_b200 as sg

    m, n, k = 256, 128, 1 << 20
    g = torch.Generator(device="cuda")
    g.manual_seed(3 + tc)
    U = torch.randn(k, n, generator=g, device="cuda") / np.sqrt(k)
    V = torch.randn(n, n, generator=g, device="cuda") / np.sqrt(n)
    sig = torch.arange(1, n + 1, device="cuda", dtype=torch.float32).pow(-2.0)
    A = (U * sig) @ V.T  # k x n, column j of A = row j of A.T
    A.add_(torch.randn(k, n, generator=g, device="cuda"), alpha=1e-6)
    A_cm = A.T.contiguous().reshape(-1)  # column-major k x n, ld = k
    Om = (torch.randn(m * k, generator=g, device="cuda") / 16.0).to(torch.float16)  # k x m col-major, ld = k
    del U, V, A
    hd = sg.Handle(0)
    try:
        if workspace == "k_blocks":
            hd.set_workspace_size((64 << 20) + m * k * 2)
        Y = torch.zeros(m * n, device="cuda")
        lvl = sg.hsgemm(hd, 1, 0, m, n, k, 1.0, Om, k, A_cm, k, 0.0, Y, m, tc)
        torch.cuda.synchronize()
        assert hd.check_error() == 0
        assert lvl == sg.P0  # split-K reports the small level, like the reference's k-slicing
    finally:
        hd.close()
    om_np = Om.view(torch.int16).cpu().numpy().view(np.float16)
    a_np = A_cm.cpu().numpy()
    gpu = oracle.logical_c(Y.cpu().numpy(), m, n, m)
    del Om, A_cm, Y

    def run(model):
        out = np.zeros(m * n, np.float32)
        oracle.hsgemm(tc, 1, 0, m, n, k, 1.0, om_np, k, a_np, k, 0.0, out, m, 0, 0, model)
        return oracle.logical_c(out, m, n, m)

    tcm, ideal = run(oracle.TCMODEL), None
    # FP64: Y^T (n x m) = A^T Omega with A^T as the FP32 operand
    ref = oracle.dgemm_ref(1, 0, n, m, k, 1.0, a_np, k, om_np, k).T
    sgc_buf = np.zeros(m * n, np.float32)
    oracle.sgemm(1, 0, n, m, k, 1.0, a_np, k, om_np, k, 0.0, sgc_buf, m, 1)
    sgc = oracle.logical_c(sgc_buf, m, n, m)
    r = _report(gpu, tcm, ideal, ref, sgc)
    _print(f"sketch 256x128x2^20 {['fp16', 'tf32'][tc]} ({workspace})", r)
    assert r["finite_mask_equal"] and r["finite_fraction"] == 1.0, r
    assert r["e_gpu"] <= 2.0 * r["e_oracle"] + K.ULP_FLOOR, r
    assert r["e_gpu"] <= 2.0 * r["e_sgemm"] + K.ULP_FLOOR, r
