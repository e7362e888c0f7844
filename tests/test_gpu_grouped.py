"""Grouped launches (many uneven problems, one persistent kernel) and their CUDA-graph
replay with new tables. The reference has no grouped path; its equivalent is a host
loop of shgemm calls, which is what every result here is checked against (through
the oracle and the single-problem entry point)."""
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


def _batch(rng, count, op_a, k_max=1500):
    shapes = []
    ns = [1, 17, 32, 33, 64, 100, 128, 200, 256, 300]
    for i in range(count):
        m = int(rng.integers(1, 700))
        n = ns[i % len(ns)]
        k = int(rng.integers(0, k_max)) if i % 7 else 0
        shapes.append((m, n, k))
    return shapes


def _run_batch(h, shapes, tc, op_a, rng, beta=0.0, stream_capture=False):
    import torch

    import shgemm_b200 as sg

    inputs, dev, probs = [], [], []
    for (m, n, k) in shapes:
        # leading dimensions TMA can address: lda a multiple of 4 floats, ldb of 8 halves
        lda = ((m if op_a == 0 else k) + 4 + 3) // 4 * 4
        ldb = (k + 8 + 7) // 8 * 8
        inp = K.make_inputs_with_ld(rng, m, n, k, op_a, 0, 0, lda, ldb, m + 3)
        A = torch.from_numpy(inp["A"]).cuda()
        B = torch.from_numpy(inp["B"].view(np.int16)).cuda().view(torch.float16)
        C = torch.from_numpy(inp["C"].copy()).cuda()
        inputs.append(inp)
        dev.append((A, B, C))
        probs.append((m, n, k, A, inp["lda"], B, inp["ldb"], C, inp["ldc"], 1.0, beta))
    return inputs, dev, probs


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
@pytest.mark.parametrize("op_a", [0, 1])
def test_grouped_matches_oracle(h, tc, op_a):
    import torch

    import shgemm_b200 as sg

    rng = np.random.default_rng(100 + tc * 10 + op_a)
    shapes = _batch(rng, 24, op_a)
    inputs, dev, probs = _run_batch(h, shapes, tc, op_a, rng, beta=0.5)
    sg.shgemm_grouped(h, probs, tc, op_a=op_a)
    torch.cuda.synchronize()
    assert h.check_error() == 0
    for (m, n, k), inp, (_, _, C) in zip(shapes, inputs, dev):
        gpu_c = C.cpu().numpy()
        orc = K.run_oracle(tc, op_a, 0, m, n, k, 1.0, inp, 0.5, 0, chunk=0)
        ref = K.fp64(op_a, 0, m, n, k, 1.0, inp, 0.5, 0)
        sgc = K.sgemm(op_a, 0, m, n, k, 1.0, inp, 0.5, 0)
        K.assert_parity(K.parity_report(gpu_c, orc, ref, sgc, m, n, inp["ldc"], 0))


@pytest.mark.parametrize("op_a", [0, 1])
def test_grouped_tf32_widened_b_matches_oracle(h, op_a):
    """TF32 batches whose B is handed over already widened to FP32 (exact binary16 values)."""
    import torch

    import shgemm_b200 as sg

    rng = np.random.default_rng(300 + op_a)
    shapes = _batch(rng, 24, op_a)
    inputs, dev, probs = _run_batch(h, shapes, oracle.TF32, op_a, rng, beta=0.5)
    wide = []
    for (m, n, k, A, lda, B, ldb, C, ldc, al, be) in probs:
        ldb4 = (k + 3) // 4 * 4 + 4  # a 16-byte multiple of FP32
        Bw = torch.zeros(max(1, n * ldb4), device=B.device, dtype=torch.float32)
        if k > 0:
            Bw.view(n, ldb4)[:, :k] = B.view(n, ldb)[:, :k].float()
        wide.append((m, n, k, A, lda, Bw, ldb4, C, ldc, al, be))
    h.set_config(sg.CFG_GROUPED_B_FP32, 1)
    try:
        sg.shgemm_grouped(h, wide, sg.tf32, op_a=op_a)
        torch.cuda.synchronize()
    finally:
        h.set_config(sg.CFG_GROUPED_B_FP32, 0)
    assert h.check_error() == 0
    for (m, n, k), inp, (_, _, C) in zip(shapes, inputs, dev):
        gpu_c = C.cpu().numpy()
        orc = K.run_oracle(oracle.TF32, op_a, 0, m, n, k, 1.0, inp, 0.5, 0, chunk=0)
        ref = K.fp64(op_a, 0, m, n, k, 1.0, inp, 0.5, 0)
        sgc = K.sgemm(op_a, 0, m, n, k, 1.0, inp, 0.5, 0)
        K.assert_parity(K.parity_report(gpu_c, orc, ref, sgc, m, n, inp["ldc"], 0))


@pytest.mark.parametrize("op_a", [0, 1])
def test_generated_b_matches_materialised_b(h, op_a):
    """Problems whose B is the block-sign Rademacher operand generated by the kernel's B
    producer give C bit-identical to the same batch with that operand materialised by
    shgemm_b200_generate_omega (scale 1) and loaded by TMA -- ragged n and k, k = 0, tiles
    past n, mixed with ordinary problems -- and stay within the parity bar of the oracle."""
    import torch

    import shgemm_b200 as sg
    from shgemm_b200 import server as srv

    rng = np.random.default_rng(500 + op_a)
    shapes = [(300, 64, 512), (129, 256, 1000), (640, 32, 320), (64, 100, 2049), (77, 17, 63), (200, 48, 0),
              (1000, 250, 4096)]
    inputs, dev, probs_gen, probs_mat, oms = [], [], [], [], []
    for i, (m, n, k) in enumerate(shapes):
        lda = ((m if op_a == 0 else k) + 4 + 3) // 4 * 4
        ldb = (k + 8 + 7) // 8 * 8
        inp = K.make_inputs_with_ld(rng, m, n, k, op_a, 0, 0, lda, ldb, m + 3)
        A = torch.from_numpy(inp["A"]).cuda()
        C1 = torch.from_numpy(inp["C"].copy()).cuda()
        C2 = C1.clone()
        seed = 1000 + i
        Om = torch.zeros(n * ldb + 8, device="cuda", dtype=torch.float16)
        if k > 0:
            srv.generate_omega(Om, ldb, k, n, srv.RADEMACHER_BLOCKS, seed, 1.0)
        alpha = float(n) ** -0.5
        if i == 1:  # one ordinary problem in the mix: B given, loaded by TMA in both batches
            Bg = torch.from_numpy(inp["B"].view(np.int16)).cuda().view(torch.float16)
            probs_gen.append((m, n, k, A, lda, Bg, ldb, C1, m + 3, alpha, 0.5))
            probs_mat.append((m, n, k, A, lda, Bg, ldb, C2, m + 3, alpha, 0.5))
        else:
            probs_gen.append((m, n, k, A, lda, None, 0, C1, m + 3, alpha, 0.5, srv.RADEMACHER_BLOCKS, seed))
            probs_mat.append((m, n, k, A, lda, Om, ldb, C2, m + 3, alpha, 0.5))
        inputs.append(inp)
        dev.append((A, C1, C2))
        oms.append((Om, ldb))
    torch.cuda.synchronize()
    sg.shgemm_grouped(h, probs_gen, sg.fp16, op_a=op_a)
    sg.shgemm_grouped(h, probs_mat, sg.fp16, op_a=op_a)
    torch.cuda.synchronize()
    assert h.check_error() == 0
    for i, ((m, n, k), inp, (A, C1, C2), (Om, ldb)) in enumerate(zip(shapes, inputs, dev, oms)):
        assert torch.equal(C1.view(torch.int32), C2.view(torch.int32)), (i, m, n, k)
        if i == 1 or k == 0:
            continue
        om_np = Om[:n * ldb].view(torch.int16).cpu().numpy().view(np.float16)
        vals = np.unique(om_np.reshape(n, ldb)[:, :k].astype(np.float32))
        assert set(vals.tolist()) <= {-1.0, 1.0}
        ref_inp = dict(inp, B=om_np, ldb=ldb)
        alpha = float(n) ** -0.5
        orc = K.run_oracle(oracle.FP16, op_a, 0, m, n, k, alpha, ref_inp, 0.5, 0, chunk=0)
        ref = K.fp64(op_a, 0, m, n, k, alpha, ref_inp, 0.5, 0)
        sgc = K.sgemm(op_a, 0, m, n, k, alpha, ref_inp, 0.5, 0)
        K.assert_parity(K.parity_report(C1.cpu().numpy(), orc, ref, sgc, m, n, m + 3, 0))


def test_grouped_result_same_alone_and_in_the_mix(h):
    """A problem's result does not depend on the batch it runs in (bit for bit)."""
    import torch

    import shgemm_b200 as sg

    rng = np.random.default_rng(5)
    shapes = _batch(rng, 16, 0)
    inputs, dev, probs = _run_batch(h, shapes, oracle.FP16, 0, rng)
    initial = [C.clone() for (_, _, C) in dev]
    sg.shgemm_grouped(h, probs, sg.fp16)
    torch.cuda.synchronize()
    mixed = [C.clone() for (_, _, C) in dev]
    for i, q in enumerate(probs):
        dev[i][2].copy_(initial[i])
        sg.shgemm_grouped(h, [q], sg.fp16)
        torch.cuda.synchronize()
        assert torch.equal(dev[i][2], mixed[i]), i


def test_grouped_graph_replay_with_new_tables(h):
    """One captured grouped launch replayed with two different batches."""
    import torch

    import shgemm_b200 as sg

    rng = np.random.default_rng(9)
    s = torch.cuda.Stream()
    h.set_stream(s)
    try:
        shapes1 = [(300, 64, 512), (129, 256, 1000), (640, 32, 320), (64, 128, 2048)]
        in1, dev1, pr1 = _run_batch(h, shapes1, oracle.FP16, 0, rng)
        # warm-up outside the capture, then capture the same call
        with torch.cuda.stream(s):
            sg.shgemm_grouped(h, pr1, sg.fp16)
        s.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            sg.shgemm_grouped(h, pr1, sg.fp16)
        for (_, _, C) in dev1:
            C.zero_()
        torch.cuda.synchronize()
        with torch.cuda.stream(s):
            g.replay()
        torch.cuda.synchronize()
        for (m, n, k), inp, (_, _, C) in zip(shapes1, in1, dev1):
            orc = K.run_oracle(oracle.FP16, 0, 0, m, n, k, 1.0, inp, 0.0, 0, chunk=0)
            ref = K.fp64(0, 0, m, n, k, 1.0, inp, 0.0, 0)
            sgc = K.sgemm(0, 0, m, n, k, 1.0, inp, 0.0, 0)
            K.assert_parity(K.parity_report(C.cpu().numpy(), orc, ref, sgc, m, n, inp["ldc"], 0))
        # a different batch (fewer problems, other sizes and buffers) through the same graph
        shapes2 = [(500, 200, 700), (77, 17, 1500), (1000, 256, 128)]
        in2, dev2, pr2 = _run_batch(h, shapes2, oracle.FP16, 0, rng)
        sg.grouped_update(h, pr2, sg.fp16)
        with torch.cuda.stream(s):
            g.replay()
        torch.cuda.synchronize()
        assert h.check_error() == 0
        for (m, n, k), inp, (_, _, C) in zip(shapes2, in2, dev2):
            orc = K.run_oracle(oracle.FP16, 0, 0, m, n, k, 1.0, inp, 0.0, 0, chunk=0)
            ref = K.fp64(0, 0, m, n, k, 1.0, inp, 0.0, 0)
            sgc = K.sgemm(0, 0, m, n, k, 1.0, inp, 0.0, 0)
            K.assert_parity(K.parity_report(C.cpu().numpy(), orc, ref, sgc, m, n, inp["ldc"], 0))
        del g
    finally:
        h.set_stream(torch.cuda.current_stream())


def test_eager_tf32_call_between_replays_leaves_captured_batch_intact(cuda_device):
    """An eager TF32 shgemm that takes the widened-B route (its own one-problem grouped
    table) between two replays of a captured grouped launch on the same handle: the second
    replay still computes the captured batch, and the eager call its own product."""
    import torch

    import shgemm_b200 as sg

    hd = sg.Handle(0)
    s = torch.cuda.Stream()
    hd.set_stream(s)
    try:
        rng = np.random.default_rng(77)
        shapes = [(300, 64, 512), (129, 256, 1000), (640, 32, 320)]
        ins, dev, probs = _run_batch(hd, shapes, oracle.FP16, 0, rng)
        with torch.cuda.stream(s):
            sg.shgemm_grouped(hd, probs, sg.fp16)
        s.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            sg.shgemm_grouped(hd, probs, sg.fp16)
        # eager TF32 call whose 128 x 256 tiles fill the GPU: widened B, one-problem table
        m, n, k = 2048, 2560, 700
        hd.set_workspace_size(max(64 << 20, n * (k + 3) // 4 * 4 * 4 + (1 << 20)))
        inp = K.make_inputs(rng, m, n, k, 0, 0, 0, dist="uniform")
        A = torch.from_numpy(inp["A"]).cuda()
        B = torch.from_numpy(inp["B"].view(np.int16)).cuda().view(torch.float16)
        Ce = torch.from_numpy(inp["C"].copy()).cuda()
        before = hd.launch_count()
        with torch.cuda.stream(s):
            sg.shgemm(hd, 0, 0, m, n, k, 1.0, A, inp["lda"], B, inp["ldb"], 0.0, Ce, inp["ldc"], sg.tf32)
        s.synchronize()
        assert hd.launch_count() - before == 2  # widen + the TF32 grouped kernel: the route was taken
        for (_, _, C) in dev:
            C.zero_()
        torch.cuda.synchronize()
        with torch.cuda.stream(s):
            g.replay()
        torch.cuda.synchronize()
        assert hd.check_error() == 0
        for (mm, nn, kk), ip, (_, _, C) in zip(shapes, ins, dev):
            orc = K.run_oracle(oracle.FP16, 0, 0, mm, nn, kk, 1.0, ip, 0.0, 0, chunk=0)
            ref = K.fp64(0, 0, mm, nn, kk, 1.0, ip, 0.0, 0)
            sgc = K.sgemm(0, 0, mm, nn, kk, 1.0, ip, 0.0, 0)
            K.assert_parity(K.parity_report(C.cpu().numpy(), orc, ref, sgc, mm, nn, ip["ldc"], 0))
        orc = K.run_oracle(oracle.TF32, 0, 0, m, n, k, 1.0, inp, 0.0, 0, chunk=0)
        ref = K.fp64(0, 0, m, n, k, 1.0, inp, 0.0, 0)
        sgc = K.sgemm(0, 0, m, n, k, 1.0, inp, 0.0, 0)
        K.assert_parity(K.parity_report(Ce.cpu().numpy(), orc, ref, sgc, m, n, inp["ldc"], 0))
        del g
    finally:
        hd.close()


def test_grouped_rejects_unsupported(h):
    import torch

    import shgemm_b200 as sg

    A = torch.zeros(64 * 64 + 8, device="cuda")
    B = torch.zeros(64 * 64 + 8, device="cuda", dtype=torch.float16)
    C = torch.zeros(64 * 64, device="cuda")
    with pytest.raises(sg.ShgemmError) as ei:  # op_b = op_t is not supported by grouped launches
        sg.shgemm_grouped(h, [(64, 64, 64, A, 64, B, 64, C, 64)], sg.fp16, op_b=sg.op_t)
    assert ei.value.status == 2
    with pytest.raises(sg.ShgemmError) as ei:  # lda not 16-byte aligned
        sg.shgemm_grouped(h, [(61, 64, 64, A, 61, B, 64, C, 64)], sg.fp16)
    assert ei.value.status == 2


def _mix64(z):
    """splitmix64's finaliser on numpy uint64 (wrapping arithmetic)."""
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def _block_sign_bit(r):
    """Bit of a block's hash that signs entry r (0..63) of the block: entries 2p and 2p + 1
    take bits (p mod 16) and (p mod 16) + 16 of 32-bit half p / 16."""
    p = r >> 1
    return 32 * (p >> 4) + (p & 15) + 16 * (r & 1)


def test_block_sign_bit_order_is_a_permutation():
    assert sorted(_block_sign_bit(r) for r in range(64)) == list(range(64))


def test_block_sign_stream_is_the_documented_one(cuda_device):
    """shgemm_b200_generate_omega(RADEMACHER_BLOCKS): entry (r, c) negative exactly when bit
    b(r mod 64) of splitmix64(seed * 0x9E3779B97F4A7C15 + c * ceil(k / 64) + r / 64 + 1) is set,
    b(r) = 32 (r / 32) + (r / 2 mod 16) + 16 (r mod 2)."""
    import torch

    from shgemm_b200 import server as srv

    k, n, seed, ld = 200, 5, 77, 208
    Om = torch.zeros(n * ld, device="cuda", dtype=torch.float16)
    srv.generate_omega(Om, ld, k, n, srv.RADEMACHER_BLOCKS, seed, 0.5)
    got = Om.view(n, ld)[:, :k].float().cpu().numpy()
    kb = (k + 63) // 64
    with np.errstate(over="ignore"):
        base = np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15)
    for c in range(n):
        for r in range(k):
            with np.errstate(over="ignore"):
                x = _mix64(base + np.uint64(c * kb + r // 64 + 1))
            neg = (int(x) >> _block_sign_bit(r % 64)) & 1
            assert got[c, r] == (-0.5 if neg else 0.5), (c, r)
