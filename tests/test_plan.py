"""The host planner (no GPU): kernel level, tile N and split-K slices of a call, against the
rule it documents -- the reference's level choice (large tile when it fills the machine or
split-K will, src/shgemm.cu:643-656) and deterministic split-K only where tiles leave SMs idle,
k is long and the workspace holds the partials, with the slice count that maximises the busy
fraction over the waves."""
import math

import pytest

import shgemm_b200 as sg

SMS = 148


def _waves(units, sms=SMS):
    return units / (math.ceil(units / sms) * sms)


def _expected(m, n, k, tc, ws):
    small, big = (128, 256) if tc == sg.fp16 else (64, 128)
    bk = 64 if tc == sg.fp16 else 32
    steps = math.ceil(k / bk)
    tiles_m = math.ceil(m / 128)
    fit = min(ws // (m * n * 4), 1024)
    can_split = fit >= 2 and k >= 4096
    level = 1 if n > small and (tiles_m * math.ceil(n / big) >= SMS or can_split) else 0
    bn = big if level else small
    if n <= 64:
        bn = 64
    tiles = tiles_m * math.ceil(n / bn)
    slices = 1
    if can_split and tiles < SMS:
        best = _waves(tiles)
        for s in range(2, min(fit, 64) + 1):
            if steps // s < 8:
                break
            e = _waves(tiles * s)
            if e > best + 0.02:
                best, slices = e, s
    slices = max(1, min(slices, steps))
    per = math.ceil(steps / slices)
    return {"level": level, "tile_n": bn, "slices": math.ceil(steps / per)}


CASES = [
    (16384, 16384, 16384, 0, 64 << 20),   # square: large tiles fill the machine, no split
    (1024, 1024, 1024, 0, 64 << 20),      # config 1: 32 large tiles, k too short to split
    (4096, 256, 1 << 20, 0, 64 << 20),    # the sketch: few tiles, long k -> split-K
    (4096, 256, 1 << 20, 0, 0),           # no workspace: no split
    (256, 128, 1 << 20, 1, 64 << 20),     # HSGEMM sketch aspect in TF32
    (300, 48, 5000, 0, 64 << 20),         # n <= 64: tile N 64
    (8192, 8192, 8192, 1, 64 << 20),      # TF32 square
    (129, 300, 4224, 0, 1 << 20),         # ragged, little workspace
    (2048, 512, 65536, 1, 256 << 20),     # TF32, many slices possible
]


@pytest.mark.parametrize("m,n,k,tc,ws", CASES)
def test_plan_follows_the_rule(m, n, k, tc, ws):
    assert sg.plan_preview(SMS, m, n, k, tc, ws) == _expected(m, n, k, tc, ws)


def test_plan_properties():
    p = sg.plan_preview(SMS, 16384, 16384, 16384, sg.fp16, 64 << 20)
    assert p == {"level": 1, "tile_n": 256, "slices": 1}
    p = sg.plan_preview(SMS, 4096, 256, 1 << 20, sg.fp16, 64 << 20)
    assert p["tile_n"] == 256 and p["slices"] > 1
    assert (32 * p["slices"]) % SMS == 0 or _waves(32 * p["slices"]) > 0.9
    assert sg.plan_preview(SMS, 4096, 256, 1 << 20, sg.fp16, 0)["slices"] == 1
    assert sg.plan_preview(SMS, 100, 40, 100, sg.tf32, 0)["tile_n"] == 64


def test_plan_preview_rejects_bad_arguments():
    with pytest.raises(sg.ShgemmError):
        sg.plan_preview(0, 16, 16, 16, sg.fp16, 0)
    with pytest.raises(sg.ShgemmError):
        sg.plan_preview(SMS, 16, 16, 16, 7, 0)
    with pytest.raises(sg.ShgemmError):
        sg.plan_preview(SMS, 0, 16, 16, sg.fp16, 0)
