"""The allocation-free entry point, for callers that cannot call cudaMalloc
(code inside an allocator callback, or a memory manager that owns all device
memory): it must give the same result as the handle-based entry point, call
after call, with its scratch in a fixed device array.

Collected last on purpose, so that a run stopping at the first failure has
already run every other test; it also passes when run alone in a fresh process.
"""
import numpy as np
import pytest

import oracle
from tests import _cases as K

pytestmark = pytest.mark.gpu


def _device_inputs(inp):
    import torch

    A = torch.from_numpy(inp["A"]).cuda()
    B = torch.from_numpy(inp["B"].view(np.int16)).cuda().view(torch.float16)
    return A, B


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
def test_noalloc_matches_handle_entry_on_two_calls(cuda_device, tc):
    import torch

    import shgemm_b200 as sg

    m, n, k = 256, 192, 16384  # long k, few tiles: the split-K path, which uses the scratch
    rng = np.random.default_rng(123)
    inp = K.make_inputs(rng, m, n, k, 1, 0, 0)
    A, B = _device_inputs(inp)
    stream = torch.cuda.current_stream()

    h = sg.Handle(0)
    try:
        h.set_stream(stream)
        C_ref = torch.from_numpy(inp["C"].copy()).cuda()
        sg.shgemm(h, 1, 0, m, n, k, 1.0, A, inp["lda"], B, inp["ldb"], 0.5, C_ref, inp["ldc"], tc)
        torch.cuda.synchronize()
        assert h.check_error() == 0
    finally:
        h.close()
    ref_np = C_ref.cpu().numpy()

    orc = K.run_oracle(tc, 1, 0, m, n, k, 1.0, inp, 0.5, 0, chunk=0)
    ref64 = K.fp64(1, 0, m, n, k, 1.0, inp, 0.5, 0)
    sgc = K.sgemm(1, 0, m, n, k, 1.0, inp, 0.5, 0)
    C0 = torch.from_numpy(inp["C"].copy()).cuda()
    Cs = [C0.clone(), C0.clone()]  # outputs made before any call, so the calls themselves allocate nothing
    torch.cuda.synchronize()
    for i in range(2):
        C = Cs[i]
        if i == 1:  # the first call did the one-time set-up; the second must not allocate at all
            free0, torch0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
        sg.shgemm_noalloc(stream, 1, 0, m, n, k, 1.0, A, inp["lda"], B, inp["ldb"], 0.5, C, inp["ldc"], tc)
        assert sg.noalloc_check_error(stream) == 0
        if i == 1:
            assert torch.cuda.mem_get_info()[0] == free0
            assert torch.cuda.memory_allocated() == torch0
        out = C.cpu().numpy()
        # the tolerance of the parity tests, against the oracle and the FP64 product ...
        K.assert_parity(K.parity_report(out, orc, ref64, sgc, m, n, inp["ldc"], 0))
        # ... and against the handle-based entry point's result
        diff = oracle.rel_fro(oracle.logical_c(out, m, n, m), oracle.logical_c(ref_np, m, n, m))
        assert diff <= K.ULP_FLOOR, diff


def test_noalloc_rejects_problems_beyond_its_scratch(cuda_device):
    import torch

    import shgemm_b200 as sg

    limit = sg.noalloc_scratch_bytes() // 8  # two slices of FP32 partials
    m, n, k = 4096, limit // 4096 + 64, 64
    A = torch.zeros(m * k, device="cuda")
    B = torch.zeros(k * n, device="cuda", dtype=torch.float16)
    C = torch.full((m * n,), 3.0, device="cuda")
    with pytest.raises(sg.ShgemmError) as ei:
        sg.shgemm_noalloc(torch.cuda.current_stream(), 0, 0, m, n, k, 1.0, A, m, B, k, 0.0, C, m, sg.fp16)
    assert ei.value.status == 7  # SHGEMM_STATUS_SCRATCH_TOO_SMALL
    torch.cuda.synchronize()
    assert bool((C == 3.0).all())  # nothing was launched
