"""alpha and beta in device memory (shgemm_b200_shgemm_device_scalars). The reference reads
them on the host at call time (src/shgemm.cu:532,600,603); with device scalars the kernels
read them, so results must be bit-identical to the host-scalar call with the same values,
on every path a call can take, and a captured graph replays with whatever the scalars hold."""
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


def _dev(inp, shift_a=0, shift_b=0):
    import torch

    A = torch.from_numpy(np.concatenate([np.zeros(shift_a, np.float32), inp["A"]])).cuda()
    B = torch.from_numpy(np.concatenate([np.zeros(shift_b, np.float16), inp["B"]]).view(np.int16)).cuda()
    return A, B.view(torch.float16)


def _both(h, tc, op_a, op_b, op_c, m, n, k, alpha, beta, inp, shift=0):
    """C from the host-scalar call and from the device-scalar call, as numpy arrays."""
    import torch

    import shgemm_b200 as sg

    A, B = _dev(inp, shift, shift)
    a_addr, b_addr = A.data_ptr() + 4 * shift, B.data_ptr() + 2 * shift
    C_host = torch.from_numpy(inp["C"].copy()).cuda()
    C_dev = C_host.clone()
    lv_h = sg.shgemm(h, op_a, op_b, m, n, k, alpha, a_addr, inp["lda"], b_addr, inp["ldb"], beta, C_host, inp["ldc"],
                     tc, op_c)
    scal = torch.tensor([alpha, beta], dtype=torch.float32, device="cuda")
    lv_d = sg.shgemm_device_scalars(h, op_a, op_b, m, n, k, scal[0:1], a_addr, inp["lda"], b_addr, inp["ldb"],
                                    scal[1:2], C_dev, inp["ldc"], tc, op_c)
    torch.cuda.synchronize()
    assert h.check_error() == 0
    assert lv_h == lv_d
    return C_host.cpu().numpy(), C_dev.cpu().numpy()


CASES = [
    # (tc, op_a, op_b, op_c, m, n, k): 128 x 256 tensor-memory tiles, shared-memory tiles,
    # split-K, k = 0, a TF32 call that takes the widened-B route, op_c = op_t
    (oracle.FP16, 0, 0, 0, 1000, 700, 1000),
    (oracle.FP16, 1, 1, 1, 300, 200, 500),
    (oracle.TF32, 0, 1, 0, 300, 200, 500),
    (oracle.FP16, 1, 0, 0, 256, 192, 16384),
    (oracle.TF32, 0, 0, 1, 256, 192, 16384),
    (oracle.FP16, 0, 0, 0, 64, 48, 0),
    (oracle.TF32, 0, 0, 0, 2048, 2560, 700),
]


@pytest.mark.parametrize("case", CASES, ids=[f"{c}" for c in CASES])
def test_device_scalars_match_host_scalars(h, case):
    tc, op_a, op_b, op_c, m, n, k = case
    rng = np.random.default_rng(m + k)
    inp = K.make_inputs(rng, m, n, k, op_a, op_b, op_c, dist="wide" if tc == oracle.TF32 else "uniform")
    c_h, c_d = _both(h, tc, op_a, op_b, op_c, m, n, k, -1.25, 0.5, inp)
    assert np.array_equal(c_h.view(np.uint32), c_d.view(np.uint32))
    if k > 0:
        orc = K.run_oracle(tc, op_a, op_b, m, n, k, -1.25, inp, 0.5, op_c, chunk=0)
        ref = K.fp64(op_a, op_b, m, n, k, -1.25, inp, 0.5, op_c)
        sgc = K.sgemm(op_a, op_b, m, n, k, -1.25, inp, 0.5, op_c)
        K.assert_parity(K.parity_report(c_d, orc, ref, sgc, m, n, inp["ldc"], op_c))


def test_device_scalars_through_staging(h):
    """Unaligned operands go through the k-slab staging path: beta applies to the first slab,
    alpha to every slab."""
    m, n, k = 75, 61, 333
    rng = np.random.default_rng(5)
    inp = K.make_inputs(rng, m, n, k, 0, 0, 0, pad=3)
    c_h, c_d = _both(h, oracle.FP16, 0, 0, 0, m, n, k, 0.75, -2.0, inp, shift=1)
    assert np.array_equal(c_h.view(np.uint32), c_d.view(np.uint32))


def test_device_beta_zero_does_not_read_c(h):
    import torch

    import shgemm_b200 as sg

    m = n = k = 256
    rng = np.random.default_rng(9)
    inp = K.make_inputs(rng, m, n, k, 0, 0, 0)
    A, B = _dev(inp)
    C = torch.full((m * n,), float("nan"), device="cuda")
    scal = torch.tensor([1.0, 0.0], device="cuda")
    sg.shgemm_device_scalars(h, 0, 0, m, n, k, scal[0:1], A, m, B, k, scal[1:2], C, m, sg.fp16)
    torch.cuda.synchronize()
    assert torch.isfinite(C).all()


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
def test_graph_replay_picks_up_new_scalars(cuda_device, tc):
    """One captured call replayed after the device scalars are rewritten: each replay equals
    the host-scalar call with the values stored at that time."""
    import torch

    import shgemm_b200 as sg

    hd = sg.Handle(0)
    s = torch.cuda.Stream()
    hd.set_stream(s)
    try:
        m, n, k = 384, 320, 4096  # long k, few tiles: split-K, whose reduction reads the scalars too
        rng = np.random.default_rng(17)
        inp = K.make_inputs(rng, m, n, k, 0, 0, 0)
        A, B = _dev(inp)
        C0 = torch.from_numpy(inp["C"].copy()).cuda()
        C = C0.clone()
        scal = torch.tensor([1.0, 0.0], device="cuda")
        with torch.cuda.stream(s):  # warm-up outside the capture
            sg.shgemm_device_scalars(hd, 0, 0, m, n, k, scal[0:1], A, m, B, k, scal[1:2], C, m, tc)
        s.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            sg.shgemm_device_scalars(hd, 0, 0, m, n, k, scal[0:1], A, m, B, k, scal[1:2], C, m, tc)
        for alpha, beta in ((2.0, 0.0), (-0.5, 1.5), (1.0, -3.0)):
            scal.copy_(torch.tensor([alpha, beta]))
            C.copy_(C0)
            torch.cuda.synchronize()
            with torch.cuda.stream(s):
                g.replay()
            torch.cuda.synchronize()
            ref = C0.clone()
            sg.shgemm(hd, 0, 0, m, n, k, alpha, A, m, B, k, beta, ref, m, tc)
            torch.cuda.synchronize()
            assert torch.equal(C, ref), (alpha, beta)
        assert hd.check_error() == 0
        del g
    finally:
        hd.close()
