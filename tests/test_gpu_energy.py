"""The energy harness on the GPU: a short version of the reference's power sweep
(test/power_consumption_test.cu:251-286) -- one size, both compute types -- gives a
positive energy per call and a board power inside the B200's range."""
import pytest

pytestmark = pytest.mark.gpu


def test_power_sweep_short(cuda_device):
    import shgemm_b200 as sg
    from shgemm_b200 import energy

    h = sg.Handle(0)
    try:
        rows = energy.power_sweep(h, log_sizes=[12], compute_types=(1, 0), seconds=0.5)
    finally:
        h.close()
    assert [r["compute_type"] for r in rows] == ["tf32", "fp16"]
    for r in rows:
        assert r["calls"] >= 1 and r["seconds"] > 0.2
        assert r["joules_per_call"] > 0
        assert 30.0 < r["avg_power_w"] < 1500.0, r
        assert r["tflops"] > 1.0, r
