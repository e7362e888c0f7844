"""The tensor-memory kernel in CTA pairs (SHGEMM_CFG_PAIR_TILES = 1: 256 x 256 tiles over two
SMs, tcgen05.mma.cta_group::2, each CTA loading half of B) computes the same products in the
same order as the one-CTA form: C must be bit-identical, on ragged shapes (rows past a pair
tile, columns past a tile), an odd number of pair tiles, op_a = T, beta != 0 and split-K, and
within the parity bar of the restated reference."""
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
    yield hd
    hd.close()


@pytest.mark.parametrize("op_a", [0, 1])
@pytest.mark.parametrize("mnk", [(1000, 700, 3000), (300, 512, 256), (2048, 1024, 1024), (129, 300, 4224),
                                 (384, 256, 64), (256, 256, 16384)])
def test_pair_tiles_bit_identical(h, capfd, op_a, mnk):
    import shgemm_b200 as sg

    m, n, k = mnk
    sg.enable_kernel_level_fixing(h, 1)  # 128 x 256 tiles: the tensor-memory kernel
    try:
        r1, c1, inp = _run(h, op_a, m, n, k, pair=0)
        sg.set_debug_mode(h, 1)
        try:
            r2, c2, _ = _run(h, op_a, m, n, k, pair=1)
        finally:
            sg.set_debug_mode(h, 0)
        ctypes.CDLL(None).fflush(None)
        assert "CTA pairs" in capfd.readouterr().out  # the pair kernel really ran
    finally:
        sg.disable_kernel_level_fixing(h)
    K.assert_parity(r1)
    K.assert_parity(r2)
    assert np.array_equal(c1.view(np.uint32), c2.view(np.uint32))


def _run(h, op_a, m, n, k, pair):
    import shgemm_b200 as sg

    h.set_config(sg.CFG_PAIR_TILES, pair)
    try:
        rng = np.random.default_rng(m + k + op_a)
        inp = K.make_inputs(rng, m, n, k, op_a, 0, 0, dist="wide")
        gpu_c, _ = K.run_gpu(h, oracle.FP16, op_a, 0, m, n, k, 1.0, inp, 0.5, 0)
    finally:
        h.set_config(sg.CFG_PAIR_TILES, 0)
    orc = K.run_oracle(oracle.FP16, op_a, 0, m, n, k, 1.0, inp, 0.5, 0, chunk=0)
    ref = K.fp64(op_a, 0, m, n, k, 1.0, inp, 0.5, 0)
    sgc = K.sgemm(op_a, 0, m, n, k, 1.0, inp, 0.5, 0)
    return K.parity_report(gpu_c, orc, ref, sgc, m, n, inp["ldc"], 0), gpu_c, inp
