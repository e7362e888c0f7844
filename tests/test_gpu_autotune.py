"""The autotuner: per-bucket entries, their use by later calls (same results as the
heuristic plan, within the parity bar), the tune-on-first-use mode and the cache file.
No reference counterpart (the reference's tile tables are fixed at compile time,
src/shgemm.cu:429-488)."""
import numpy as np
import pytest

import oracle
from tests import _cases as K

pytestmark = pytest.mark.gpu


@pytest.fixture()
def h(cuda_device):
    import shgemm_b200 as sg

    hd = sg.Handle(0)
    yield hd
    hd.close()


def _dev(inp):
    import torch

    A = torch.from_numpy(inp["A"]).cuda()
    B = torch.from_numpy(inp["B"].view(np.int16)).cuda().view(torch.float16)
    C = torch.from_numpy(inp["C"].copy()).cuda()
    return A, B, C


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
def test_autotune_entry_used_and_correct(h, tc):
    import torch

    import shgemm_b200 as sg

    m, n, k = 512, 384, 4096
    rng = np.random.default_rng(7 + tc)
    inp = K.make_inputs(rng, m, n, k, 0, 0, 0)
    A, B, C = _dev(inp)
    assert h.autotune_lookup(0, 0, m, n, k, tc) is None
    best = h.autotune(0, 0, m, n, k, A, inp["lda"], B, inp["ldb"], C, inp["ldc"], tc)
    assert best["tile_n"] in ((64, 128, 256) if tc == oracle.FP16 else (64, 128))
    assert best["slices"] >= 1 and best["group_m"] >= 1 and best["time_us"] > 0
    assert h.autotune_lookup(0, 0, m + 100, n + 100, k + 1000, tc) == best  # same log2 bucket
    outs = []
    for _ in range(2):
        C.copy_(torch.from_numpy(inp["C"]))
        sg.shgemm(h, 0, 0, m, n, k, 1.0, A, inp["lda"], B, inp["ldb"], 0.5, C, inp["ldc"], tc)
        torch.cuda.synchronize()
        assert h.check_error() == 0
        outs.append(C.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    orc = K.run_oracle(tc, 0, 0, m, n, k, 1.0, inp, 0.5, 0, chunk=0)
    ref = K.fp64(0, 0, m, n, k, 1.0, inp, 0.5, 0)
    sgc = K.sgemm(0, 0, m, n, k, 1.0, inp, 0.5, 0)
    K.assert_parity(K.parity_report(outs[0], orc, ref, sgc, m, n, inp["ldc"], 0))


def test_autotune_on_first_use(h):
    import torch

    import shgemm_b200 as sg

    m, n, k = 256, 1024, 2048
    rng = np.random.default_rng(70)
    inp = K.make_inputs(rng, m, n, k, 1, 0, 0)
    A, B, C = _dev(inp)
    h.set_config(sg.CFG_AUTOTUNE, 2)
    sg.shgemm(h, 1, 0, m, n, k, 1.0, A, inp["lda"], B, inp["ldb"], 0.0, C, inp["ldc"], sg.fp16)
    torch.cuda.synchronize()
    assert h.autotune_lookup(1, 0, m, n, k, sg.fp16) is not None
    gpu = C.cpu().numpy()
    orc = K.run_oracle(oracle.FP16, 1, 0, m, n, k, 1.0, inp, 0.0, 0, chunk=0)
    ref = K.fp64(1, 0, m, n, k, 1.0, inp, 0.0, 0)
    sgc = K.sgemm(1, 0, m, n, k, 1.0, inp, 0.0, 0)
    K.assert_parity(K.parity_report(gpu, orc, ref, sgc, m, n, inp["ldc"], 0))


def test_autotune_cache_file(h, tmp_path):
    import shgemm_b200 as sg

    m, n, k = 300, 200, 1000
    rng = np.random.default_rng(71)
    inp = K.make_inputs(rng, m, n, k, 0, 0, 0)
    A, B, C = _dev(inp)
    best = h.autotune(0, 0, m, n, k, A, inp["lda"], B, inp["ldb"], C, inp["ldc"], sg.fp16)
    path = str(tmp_path / "tune.txt")
    h.autotune_save(path)
    h.autotune_clear()
    assert h.autotune_lookup(0, 0, m, n, k, sg.fp16) is None
    h.autotune_load(path)
    got = h.autotune_lookup(0, 0, m, n, k, sg.fp16)
    assert got["tile_n"] == best["tile_n"] and got["slices"] == best["slices"] and got["group_m"] == best["group_m"]
    bad = tmp_path / "bad.txt"
    bad.write_text("0 0 0 8 7 9 96 1 8 1.0\n")  # tile N 96 does not exist
    with pytest.raises(sg.ShgemmError):
        h.autotune_load(str(bad))


def test_autotune_entry_has_ring_and_k_chunk(h):
    """128 x 256 binary16 tiles: the tuner also chooses the tensor-memory kernel's operand ring
    and, behind the accuracy gate, the k-chunk; either way the tuned plan stays within the
    parity bar."""
    import torch

    import shgemm_b200 as sg

    m, n, k = 2048, 2048, 2048
    rng = np.random.default_rng(72)
    inp = K.make_inputs(rng, m, n, k, 0, 0, 0)
    A, B, C = _dev(inp)
    best = h.autotune(0, 0, m, n, k, A, inp["lda"], B, inp["ldb"], C, inp["ldc"], sg.fp16)
    assert best["stages"] in (0, 1) and best["k_chunk"] in (64, 128)
    C.copy_(torch.from_numpy(inp["C"]))
    sg.shgemm(h, 0, 0, m, n, k, 1.0, A, inp["lda"], B, inp["ldb"], 0.5, C, inp["ldc"], sg.fp16)
    torch.cuda.synchronize()
    assert h.check_error() == 0
    orc = K.run_oracle(oracle.FP16, 0, 0, m, n, k, 1.0, inp, 0.5, 0, chunk=0)
    ref = K.fp64(0, 0, m, n, k, 1.0, inp, 0.5, 0)
    sgc = K.sgemm(0, 0, m, n, k, 1.0, inp, 0.5, 0)
    K.assert_parity(K.parity_report(C.cpu().numpy(), orc, ref, sgc, m, n, inp["ldc"], 0))


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
def test_autotune_grouped_tiles_used_and_correct(h, tc, tmp_path):
    """Grouped launches: tile N tuned per n bucket on a batch; the next launch of the batch
    uses the entries and every problem stays within the parity bar; the entries survive the
    cache file."""
    import torch

    import shgemm_b200 as sg

    rng = np.random.default_rng(80 + tc)
    shapes = [(int(rng.integers(64, 900)), int(n), int(rng.integers(256, 2500)))
              for n in (20, 40, 48, 100, 100, 200, 240, 250)]
    inputs, dev, probs = [], [], []
    for (m, n, k) in shapes:
        lda, ldb = (m + 3) // 4 * 4, (k + 7) // 8 * 8
        inp = K.make_inputs_with_ld(rng, m, n, k, 0, 0, 0, lda, ldb, m)
        A, B, C = _dev(inp)
        inputs.append(inp)
        dev.append((A, B, C))
        probs.append((m, n, k, A, lda, B, ldb, C, m, 1.0, 0.0))
    tuned = h.autotune_grouped(probs, tc)
    assert tuned == len({int(np.floor(np.log2(n))) for (_, n, _) in shapes})
    for (_, n, _) in shapes:
        bn = h.autotune_grouped_lookup(n, tc)
        assert bn in ((32, 64, 128, 256) if tc == oracle.FP16 else (32, 64, 128))
    for (_, _, C) in dev:
        C.zero_()
    sg.shgemm_grouped(h, probs, tc)
    torch.cuda.synchronize()
    assert h.check_error() == 0
    for (m, n, k), inp, (_, _, C) in zip(shapes, inputs, dev):
        orc = K.run_oracle(tc, 0, 0, m, n, k, 1.0, inp, 0.0, 0, chunk=0)
        ref = K.fp64(0, 0, m, n, k, 1.0, inp, 0.0, 0)
        sgc = K.sgemm(0, 0, m, n, k, 1.0, inp, 0.0, 0)
        K.assert_parity(K.parity_report(C.cpu().numpy(), orc, ref, sgc, m, n, m, 0))
    path = str(tmp_path / "tune.txt")
    h.autotune_save(path)
    text = open(path).read()
    assert "autotune v2" in text and any(ln.startswith("1 ") for ln in text.splitlines())
    got = {n: h.autotune_grouped_lookup(n, tc) for (_, n, _) in shapes}
    h.autotune_clear()
    assert h.autotune_grouped_lookup(shapes[0][1], tc) is None
    h.autotune_load(path)
    assert {n: h.autotune_grouped_lookup(n, tc) for (_, n, _) in shapes} == got
