"""TF32 calls with a K-contiguous binary16 B and n > 64 whose workspace holds B widened to FP32
(the sketch shapes: few tiles, long k): B is widened once per call and the 128 x 256 (n > 128)
or 128 x 128 TF32 kernel that loads FP32 B directly runs with split-K. Parity with the restated reference
algorithm, and the debug line shows that this path ran. Shapes keep the operands
TMA-addressable (16-byte leading dimensions) and ragged against the 128 x 256 x 32 tiles."""
import ctypes

import numpy as np
import pytest

import oracle
from tests import _cases as K

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h(cuda_device):
    import shgemm_b200 as sg

    hd = sg.Handle(0)
    hd.set_config(sg.CFG_AUTOTUNE, 0)
    yield hd
    hd.close()


@pytest.mark.parametrize("op_a,op_c", [(1, 1), (0, 0), (1, 0)])
@pytest.mark.parametrize("mnk", [(512, 256, 32768), (300, 200, 20008), (132, 257, 4104), (1024, 384, 8192),
                                 (700, 100, 16384), (256, 128, 8200)])
def test_tf32_widened_b_split_k(h, capfd, op_a, op_c, mnk):
    import shgemm_b200 as sg

    m, n, k = mnk
    rng = np.random.default_rng(m + n + k + op_a)
    inp = K.make_inputs(rng, m, n, k, op_a, 0, op_c, dist="wide")
    ldw = (k + 3) // 4 * 4
    h.set_workspace_size(ldw * n * 4 + (64 << 20))
    sg.set_debug_mode(h, 1)
    try:
        gpu_c, _ = K.run_gpu(h, oracle.TF32, op_a, 0, m, n, k, 1.0, inp, 0.5, op_c)
    finally:
        sg.set_debug_mode(h, 0)
        h.set_workspace_size(64 << 20)
    ctypes.CDLL(None).fflush(None)
    out = capfd.readouterr().out
    assert "B widened to FP32" in out, out  # the widened-B tile kernel ran
    assert h.check_error() == 0
    orc = K.run_oracle(oracle.TF32, op_a, 0, m, n, k, 1.0, inp, 0.5, op_c, chunk=0)
    ref = K.fp64(op_a, 0, m, n, k, 1.0, inp, 0.5, op_c)
    sgc = K.sgemm(op_a, 0, m, n, k, 1.0, inp, 0.5, op_c)
    K.assert_parity(K.parity_report(gpu_c, orc, ref, sgc, m, n, inp["ldc"], op_c))


def test_tf32_small_workspace_keeps_the_other_path(h, capfd):
    """Without room for the widened B the call takes the kernel that widens B tile by tile."""
    import shgemm_b200 as sg

    m, n, k = 256, 256, 16384
    rng = np.random.default_rng(9)
    inp = K.make_inputs(rng, m, n, k, 1, 0, 0)
    h.set_workspace_size(1 << 20)
    sg.set_debug_mode(h, 1)
    try:
        gpu_c, _ = K.run_gpu(h, oracle.TF32, 1, 0, m, n, k, 1.0, inp, 0.0, 0)
    finally:
        sg.set_debug_mode(h, 0)
        h.set_workspace_size(64 << 20)
    ctypes.CDLL(None).fflush(None)
    assert "B widened to FP32" not in capfd.readouterr().out
    orc = K.run_oracle(oracle.TF32, 1, 0, m, n, k, 1.0, inp, 0.0, 0, chunk=0)
    ref = K.fp64(1, 0, m, n, k, 1.0, inp, 0.0, 0)
    sgc = K.sgemm(1, 0, m, n, k, 1.0, inp, 0.0, 0)
    K.assert_parity(K.parity_report(gpu_c, orc, ref, sgc, m, n, inp["ldc"], 0))
