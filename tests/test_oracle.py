"""The CPU oracle against the golden fixtures (independent implementations)."""
import os

import numpy as np
import pytest

import oracle

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _same_float(a, b):
    a = np.asarray(a, dtype=np.float32)
    b = np.asarray(b, dtype=np.float32)
    both_nan = np.isnan(a) & np.isnan(b)
    return np.all(both_nan | (a.view(np.uint32) == b.view(np.uint32)))


def test_split_fp16_matches_numpy_ieee_cast():
    g = np.load(os.path.join(GOLD, "split_fp16.npz"))
    hi, lo = oracle.split(oracle.FP16, g["v"])
    assert _same_float(hi, g["hi"].view(np.float16).astype(np.float32))
    assert _same_float(lo, g["lo"].view(np.float16).astype(np.float32))


def test_f16_bits_roundtrip_all_halves():
    bits = np.arange(0, 1 << 16, dtype=np.uint32).astype(np.uint16)
    vals = bits.view(np.float16).astype(np.float32)
    finite = np.isfinite(vals)
    back = oracle.f32_to_f16_bits(vals[finite])
    assert np.array_equal(back, bits[finite])


def test_split_tf32_matches_exact_rounding():
    g = np.load(os.path.join(GOLD, "split_tf32.npz"))
    hi, lo = oracle.split(oracle.TF32, g["v"])
    assert _same_float(hi, g["hi"])
    assert _same_float(lo, g["lo"])


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
def test_split_recovers_22_bits(tc):
    rng = np.random.default_rng(1)
    v = rng.uniform(-1, 1, 20000).astype(np.float32)
    v = v[np.abs(v) > 2.0 ** -10]
    hi, lo = oracle.split(tc, v)
    rec = hi.astype(np.float64) + lo.astype(np.float64) / 2048.0
    rel = np.abs(rec - v) / np.abs(v)
    assert rel.max() <= 2.0 ** -21


def test_fp16_overflow_and_underflow_handling():
    # 7e4 overflows binary16: hi = inf and lo = -inf (reference behaviour, no rescaling)
    hi, lo = oracle.split(oracle.FP16, np.array([7e4], np.float32))
    assert np.isinf(hi[0]) and np.isinf(lo[0]) and hi[0] > 0 > lo[0]
    # 2^-30 is below binary16's range: hi = 0 and it survives only in lo (x 2^11)
    hi, lo = oracle.split(oracle.FP16, np.array([2.0 ** -30], np.float32))
    assert hi[0] == 0.0 and lo[0] == np.float32(2.0 ** -19)


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
@pytest.mark.parametrize("chunk", [0, 64, 256])
def test_gemm_exact_fixture(tc, chunk):
    g = np.load(os.path.join(GOLD, "gemm_exact.npz"))
    m, n, k = int(g["m"]), int(g["n"]), int(g["k"])
    C = np.zeros(m * n, np.float32)
    oracle.shgemm(tc, 0, 0, m, n, k, 1.0, g["A"], m, g["B"], k, 0.0, C, m, 0, chunk)
    assert np.array_equal(C.astype(np.float64), g["C"])


def _rand_case(rng, m, n, k, op_a, op_b):
    A = rng.uniform(-1, 1, m * k).astype(np.float32)
    B = rng.uniform(-1, 1, k * n).astype(np.float16)
    lda = m if op_a == 0 else k
    ldb = k if op_b == 0 else n
    return A, lda, B, ldb


@pytest.mark.parametrize("op_a", [0, 1])
@pytest.mark.parametrize("op_b", [0, 1])
@pytest.mark.parametrize("op_c", [0, 1])
def test_shgemm_error_well_below_sgemm(op_a, op_b, op_c):
    rng = np.random.default_rng(7)
    m, n, k = 45, 38, 300
    A, lda, B, ldb = _rand_case(rng, m, n, k, op_a, op_b)
    ldc = m if op_c == 0 else n
    ref = oracle.dgemm_ref(op_a, op_b, m, n, k, 1.0, A, lda, B, ldb)
    errs = {}
    for tc in (oracle.FP16, oracle.TF32):
        C = np.zeros(m * n, np.float32)
        oracle.shgemm(tc, op_a, op_b, m, n, k, 1.0, A, lda, B, ldb, 0.0, C, ldc, op_c)
        errs[tc] = oracle.rel_fro(oracle.logical_c(C, m, n, ldc, op_c), ref)
    S = np.zeros(m * n, np.float32)
    oracle.sgemm(op_a, op_b, m, n, k, 1.0, A, lda, B, ldb, 0.0, S, ldc, op_c)
    e_s = oracle.rel_fro(oracle.logical_c(S, m, n, ldc, op_c), ref)
    assert errs[oracle.FP16] < 2 * e_s and errs[oracle.TF32] < 2 * e_s
    assert e_s < 1e-6


def test_alpha_beta_and_beta_zero_ignores_c():
    rng = np.random.default_rng(3)
    m, n, k = 20, 12, 50
    A, lda, B, ldb = _rand_case(rng, m, n, k, 0, 0)
    C0 = rng.uniform(-1, 1, m * n).astype(np.float32)
    C = C0.copy()
    oracle.shgemm(oracle.FP16, 0, 0, m, n, k, 2.0, A, lda, B, ldb, 0.5, C, m, 0)
    ref = oracle.dgemm_ref(0, 0, m, n, k, 2.0, A, lda, B, ldb, 0.5, C0, m, 0)
    assert oracle.rel_fro(oracle.logical_c(C, m, n, m), ref) < 1e-6
    Cn = np.full(m * n, np.nan, np.float32)  # beta == 0: C must not be read
    oracle.shgemm(oracle.FP16, 0, 0, m, n, k, 1.0, A, lda, B, ldb, 0.0, Cn, m, 0)
    assert np.isfinite(Cn).all()


def test_hsgemm_identity():
    rng = np.random.default_rng(5)
    m, n, k = 23, 31, 64
    Ah = rng.uniform(-1, 1, m * k).astype(np.float16)  # m x k col-major
    Bf = rng.uniform(-1, 1, k * n).astype(np.float32)  # k x n col-major
    C = np.zeros(m * n, np.float32)
    oracle.hsgemm(oracle.FP16, 0, 0, m, n, k, 1.0, Ah, m, Bf, k, 0.0, C, m, 0)
    ref = Ah.astype(np.float64).reshape(k, m).T @ Bf.astype(np.float64).reshape(n, k).T
    assert oracle.rel_fro(oracle.logical_c(C, m, n, m), ref) < 1e-6


def test_wide_exponent_lo_term_underflow():
    """Exponent-range probe (reference test/exponent_test.cu:249-252): A = 2^U(lo,hi)."""
    rng = np.random.default_rng(11)
    m = n = k = 64
    B = rng.uniform(0, 1, k * n).astype(np.float16)
    res = {}
    for lo_e, hi_e in [(-15, 14), (-36, -15), (-100, -36)]:
        A = np.exp2(rng.uniform(lo_e, hi_e, m * k)).astype(np.float32)
        ref = oracle.dgemm_ref(0, 0, m, n, k, 1.0, A, m, B, k)
        C = np.zeros(m * n, np.float32)
        oracle.shgemm(oracle.FP16, 0, 0, m, n, k, 1.0, A, m, B, k, 0.0, C, m, 0)
        res[(lo_e, hi_e)] = oracle.rel_fro(oracle.logical_c(C, m, n, m), ref)
    assert res[(-15, 14)] < 1e-6
    # below binary16's range the hi term vanishes and only the lo term carries
    # the value, with ever fewer bits: the error grows, as in the reference
    assert res[(-36, -15)] > res[(-15, 14)]
    assert res[(-100, -36)] > 0.5


def test_tcmodel_truncates_each_hi_fragment():
    """Known answer of the tensor-core model: one 16-k fragment whose exact sum is
    1 + 3 * 2^-25 (three quarters of an FP32 ulp above 1). The idealised oracle rounds it
    to nearest (1 + 2^-23); the model truncates it before the round-to-nearest add (1)."""
    k = 16
    A = np.zeros(k, np.float32)
    B = np.zeros(k, np.float16)
    A[0], B[0] = 1.0, 1.0
    for j in (1, 2, 3):  # 2^-13 * 2^-12 = 2^-25, each exact in binary16 and in the product
        A[j], B[j] = 2.0 ** -13, 2.0 ** -12
    out = {}
    for model in (oracle.IDEAL, oracle.TCMODEL):
        C = np.zeros(1, np.float32)
        oracle.shgemm(oracle.FP16, 0, 0, 1, 1, k, 1.0, A, 1, B, k, 0.0, C, 1, 0, 0, model)
        out[model] = float(C[0])
    assert out[oracle.IDEAL] == 1.0 + 2.0 ** -23
    assert out[oracle.TCMODEL] == 1.0


def test_tcmodel_lo_accumulator_truncates_across_k():
    """Known answer for the lo term, carried across two 16-k fragments. a1 = 2^-25 splits
    into hi = 0 (a binary16 tie, rounded to even) and lo = 2^-14; a2 = 3 * 2^-35 into hi = 0
    and lo = 3 * 2^-24 (subnormal). With b = (1, 2^-14) the lo sum is 2^-14 + 1.5 ulp: the
    idealised oracle rounds it to nearest (even: + 2 ulp), the truncating FP32 accumulator
    of the model keeps + 1 ulp. The fold scales by 2^-11 exactly."""
    k = 32
    A = np.zeros(k, np.float32)
    B = np.zeros(k, np.float16)
    A[0], B[0] = 2.0 ** -25, 1.0
    A[16], B[16] = 3 * 2.0 ** -35, 2.0 ** -14
    hi, lo = oracle.split(oracle.FP16, A[[0, 16]])
    assert hi[0] == 0.0 and hi[1] == 0.0 and lo[0] == 2.0 ** -14 and lo[1] == 3 * 2.0 ** -24
    out = {}
    for model in (oracle.IDEAL, oracle.TCMODEL):
        C = np.zeros(1, np.float32)
        oracle.shgemm(oracle.FP16, 0, 0, 1, 1, k, 1.0, A, 1, B, k, 0.0, C, 1, 0, 0, model)
        out[model] = float(C[0])
    assert out[oracle.IDEAL] == 2.0 ** -25 + 2.0 ** -47
    assert out[oracle.TCMODEL] == 2.0 ** -25 + 2.0 ** -48


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
def test_tcmodel_error_close_to_idealised(tc):
    """The modelled truncation costs little against the idealised sums, and both stay well
    inside 2x FP32 SGEMM's error (the bar the CUDA path is held to)."""
    rng = np.random.default_rng(12)
    m, n, k = 48, 40, 2048
    A, lda, B, ldb = _rand_case(rng, m, n, k, 0, 0)
    ref = oracle.dgemm_ref(0, 0, m, n, k, 1.0, A, lda, B, ldb)
    e = {}
    for model in (oracle.IDEAL, oracle.TCMODEL):
        C = np.zeros(m * n, np.float32)
        oracle.shgemm(tc, 0, 0, m, n, k, 1.0, A, lda, B, ldb, 0.0, C, m, 0, 0, model)
        e[model] = oracle.rel_fro(oracle.logical_c(C, m, n, m), ref)
    S = np.zeros(m * n, np.float32)
    oracle.sgemm(0, 0, m, n, k, 1.0, A, lda, B, ldb, 0.0, S, m, 0)
    e_s = oracle.rel_fro(oracle.logical_c(S, m, n, m), ref)
    assert 0.9 * e[oracle.IDEAL] <= e[oracle.TCMODEL] <= 1.5 * e[oracle.IDEAL]
    assert e[oracle.TCMODEL] < 0.5 * e_s


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
def test_b200_accumulation_model_against_the_reference_model(tc):
    """The B200 kernels' accumulation (B200MODEL: one round-to-nearest add to the running sum
    per 64 k in binary16 / 32 k in TF32, truncation only inside a drain, lo folded in by the
    2^-11 input scale) against the reference's (TCMODEL: one add per 16 / 8 k, lo truncated
    over all k), both on the CPU: the modelled error against FP64 is no larger at k = 1024 and
    about half at k = 16384 (fewer roundings of the large running sum)."""
    rng = np.random.default_rng(3)
    m = n = 64
    for k, lo_bound, hi_bound in ((1024, 0.6, 1.1), (16384, 0.4, 0.65)):
        signs = np.where(rng.random(m * k) < 0.5, -1.0, 1.0)
        A = (signs * 2.0 ** rng.uniform(-15, 14, m * k)).astype(np.float32)  # binary16-safe range
        B = rng.standard_normal(k * n).astype(np.float16)
        ref = oracle.dgemm_ref(0, 0, m, n, k, 1.0, A, m, B, k)
        err = {}
        for model in (oracle.TCMODEL, oracle.B200MODEL):
            C = np.zeros(m * n, np.float32)
            oracle.shgemm(tc, 0, 0, m, n, k, 1.0, A, m, B, k, 0.0, C, m, 0, 0, model)
            err[model] = oracle.rel_fro(oracle.logical_c(C, m, n, m), ref)
        ratio = err[oracle.B200MODEL] / err[oracle.TCMODEL]
        print(f"tc={tc} k={k}: B200 model / reference model error = {ratio:.2f}")
        assert lo_bound <= ratio <= hi_bound, (k, ratio)


def test_b200_model_rejects_a_partial_fragment_chunk():
    A = np.ones(16 * 16, np.float32)
    B = np.ones(16 * 16, np.float16)
    with pytest.raises(ValueError):
        oracle.shgemm(oracle.FP16, 0, 0, 16, 16, 16, 1.0, A, 16, B, 16, 0.0, np.zeros(256, np.float32), 16, 0, 24,
                      oracle.B200MODEL)


def test_b200_model_short_k_all_positive_data():
    """Where the method loses to the reference (the B200 model against the reference's model
    of the same tensor core, all-positive binary16 data): with the 64-k drain the alignment
    truncation inside the growing accumulator costs 2-3x the reference's error at k = 256 and
    1.3-2x at k = 1024, and wins from k ~ 4096 on; a 32-k drain would stay within 1.3x."""
    rng = np.random.default_rng(3)
    m = n = 64
    bounds = {256: ((2.0, 3.0), (0.8, 1.3)), 1024: ((1.3, 2.0), (0.8, 1.2)), 16384: ((0.5, 0.8), (0.6, 0.85))}
    for k, ((lo64, hi64), (lo32, hi32)) in bounds.items():
        A = rng.uniform(0, 1, m * k).astype(np.float32)
        B = rng.uniform(0, 1, k * n).astype(np.float16)
        ref = oracle.dgemm_ref(0, 0, m, n, k, 1.0, A, m, B, k)

        def err(model, chunk, bits):
            C = np.zeros(m * n, np.float32)
            oracle.shgemm(oracle.FP16, 0, 0, m, n, k, 1.0, A, m, B, k, 0.0, C, m, 0, chunk, model, align_bits=bits)
            return oracle.rel_fro(oracle.logical_c(C, m, n, m), ref)

        e_ref = err(oracle.TCMODEL, 0, oracle.B200_ALIGN_BITS)  # the reference's algorithm, same MMA model
        r64 = err(oracle.B200MODEL, 64, oracle.B200_ALIGN_BITS) / e_ref
        r32 = err(oracle.B200MODEL, 32, oracle.B200_ALIGN_BITS) / e_ref
        print(f"k={k}: 64-k drain {r64:.2f}x, 32-k drain {r32:.2f}x the reference's error")
        assert lo64 <= r64 <= hi64 and lo32 <= r32 <= hi32, (k, r64, r32)
