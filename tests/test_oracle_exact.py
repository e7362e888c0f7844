"""The C oracle's GEMM against a second restatement of the same algorithm in exact rational
arithmetic, with every IEEE rounding done on the rationals (no FP32 or FP64 sums at all).

Pins what the element-conversion fixtures do not: the operand indexing of every op
combination, the k-fragment walk with a ragged last fragment, the three accumulation models
(the idealised one, the reference's tensor-core model of src/wmmae_shgemm.hpp:86-124, and
the model of this library's kernels: a truncating accumulator per drain with lo folded in by
the 2^-11 input scale), the fold hi + lo * 2^-11 (tcec store, src/shgemm.cu:87-99) and the
alpha/beta epilogue (src/dmem_accessor.hpp:199-214, 267-271), bit for bit.

The oracle forms each fragment sum in FP64, which is exact while the products' bits fit in
53 bits; the inputs here keep every |value| within [2^-3, 2^3) (A) and [2^-2, 2^2) (B), so
every partial sum is exact and the two restatements must agree on every bit.
"""
from fractions import Fraction

import numpy as np
import pytest

import oracle

TWO = Fraction(2)


def _round(x, mode, prec=24, emin=-126, emax=127):
    """x rounded to a binary floating-point format with `prec` significand bits, subnormals
    below 2^emin, and overflow (to inf, or to the largest finite value when rounding toward
    zero). mode: "rne" (nearest, ties to even), "rna" (nearest, ties away), "rz"."""
    if x == 0:
        return Fraction(0)
    neg = x < 0
    a = -x if neg else x
    e = a.numerator.bit_length() - a.denominator.bit_length()
    if TWO ** e > a:
        e -= 1
    e = max(e, emin)
    q = TWO ** (e - prec + 1)
    n, rem = divmod(a, q)
    if mode == "rne" and (2 * rem > q or (2 * rem == q and n % 2 == 1)):
        n += 1
    elif mode == "rna" and 2 * rem >= q:
        n += 1
    r = n * q
    if r >= TWO ** (emax + 1):
        if mode == "rz":
            r = (TWO - TWO ** (1 - prec)) * TWO ** emax
        else:
            return float("-inf") if neg else float("inf")
    return -r if neg else r


def rn(x):
    return _round(x, "rne")


def rz(x):
    return _round(x, "rz")


def _f32(x):
    return np.float32(float(x))


def _split(tc, v):
    """hi = T(v), lo = T(2^11 (v - hi)) with FP32 subtraction and scaling
    (src/wmmae_shgemm.hpp:30-31). binary16 through numpy's IEEE cast, TF32 through the
    rational rounder (10 stored bits, ties away, binary32's exponent range)."""
    v = np.float32(v)
    if tc == oracle.FP16:
        hi = np.float32(np.float16(v))
        lo = np.float32(np.float16(np.float32(2048.0) * np.float32(v - hi)))
    else:
        hi = _f32(_round(Fraction(float(v)), "rna", prec=11))
        lo = _f32(_round(Fraction(float(np.float32(2048.0) * np.float32(v - hi))), "rna", prec=11))
    return Fraction(float(hi)), Fraction(float(lo))


def _exponent(x):
    """floor(log2 |x|) of a nonzero rational."""
    x = abs(x)
    e = x.numerator.bit_length() - x.denominator.bit_length()
    return e - 1 if TWO ** e > x else e


def _mma(c, pairs, p):
    """One modelled MMA instruction on the accumulator c and the factor pairs (a, b): with
    p > 0 every term gets a nominal exponent (a product the sum of its factors' exponents, c
    its own), E is the largest among the nonzero terms, each term is truncated toward zero to a
    multiple of 2^(E - p + 1), the terms are summed exactly and the sum truncated to FP32; with
    p = 0 the exact sum is truncated."""
    terms = [c] + [a * b for a, b in pairs]
    if p > 0:
        nominal = ([_exponent(c)] if c != 0 else []) + [_exponent(a) + _exponent(b) for a, b in pairs
                                                         if a != 0 and b != 0]
        if nominal:
            q = TWO ** (max(nominal) - p + 1)
            terms = [(abs(t) // q) * q * (1 if t >= 0 else -1) for t in terms]
    return rz(sum(terms, Fraction(0)))


def _b200_element(h, l, bv, k, frag, nfrag, p):
    """One element as the B200 kernels accumulate it (the oracle's B200MODEL): per drain of
    nfrag fragments, D from zero goes through one modelled MMA per lo fragment, then per hi
    fragment, the first with D scaled by 2^-11; the drain is added to the running sum with
    round to nearest."""
    acc = Fraction(0)
    for k0 in range(0, k, frag * nfrag):
        d = Fraction(0)
        for part, src in ((0, l), (1, h)):
            for f in range(nfrag):
                kb = k0 + f * frag
                if kb >= k:
                    break
                pairs = [(src[kk], bv[kk]) for kk in range(kb, min(kb + frag, k))]
                d = _mma(d / 2048 if part == 1 and f == 0 else d, pairs, p)
        acc = rn(acc + d)
    return acc


def _exact_shgemm(tc, op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, op_c, chunk, model,
                  align_bits=oracle.B200_ALIGN_BITS):
    if model == oracle.B200MODEL:
        frag = 16 if tc == oracle.FP16 else 8
        chunk = chunk or (64 if tc == oracle.FP16 else 32)
    chunk = chunk or (16 if tc == oracle.FP16 else 8)
    a = lambda i, kk: A[i + kk * lda] if op_a == oracle.OP_N else A[kk + i * lda]  # noqa: E731
    b = lambda kk, j: B[kk + j * ldb] if op_b == oracle.OP_N else B[j + kk * ldb]  # noqa: E731
    split = {}
    out = C.copy()
    al, be = Fraction(float(np.float32(alpha))), Fraction(float(np.float32(beta)))
    for j in range(n):
        for i in range(m):
            if model == oracle.B200MODEL:
                for kk in range(k):
                    if (i, kk) not in split:
                        split[(i, kk)] = _split(tc, a(i, kk))
                h = [split[(i, kk)][0] for kk in range(k)]
                l = [split[(i, kk)][1] for kk in range(k)]
                bv = [Fraction(float(np.float16(b(kk, j)))) for kk in range(k)]
                c = _b200_element(h, l, bv, k, frag, chunk // frag, align_bits)
                idx = i + j * ldc if op_c == oracle.OP_N else j + i * ldc
                res = rn(c * al) if beta == 0 else rn(c * al + rn(be * Fraction(float(out[idx]))))
                out[idx] = _f32(res)
                continue
            acc, lo_acc, lo_exact = Fraction(0), Fraction(0), Fraction(0)
            for k0 in range(0, k, chunk):
                s = t = Fraction(0)
                for kk in range(k0, min(k0 + chunk, k)):
                    key = (i, kk)
                    if key not in split:
                        split[key] = _split(tc, a(i, kk))
                    h, l = split[key]
                    bv = Fraction(float(np.float16(b(kk, j))))
                    s += h * bv
                    t += l * bv
                lo_exact += t
                if model == oracle.IDEAL:
                    acc = rn(acc + rn(s))
                else:
                    acc = rn(acc + rz(s))
                    lo_acc = rz(lo_acc + t)
            lo = rn(lo_exact) if model == oracle.IDEAL else lo_acc
            c = rn(acc + rn(lo / 2048))
            idx = i + j * ldc if op_c == oracle.OP_N else j + i * ldc
            if beta == 0:
                res = rn(c * al)
            else:
                res = rn(c * al + rn(be * Fraction(float(out[idx]))))
            out[idx] = _f32(res)
    return out


def _inputs(rng, m, n, k, op_a, op_b, op_c):
    lda = (m if op_a == oracle.OP_N else k) + 3
    ldb = (k if op_b == oracle.OP_N else n) + 2
    ldc = (m if op_c == oracle.OP_N else n) + 1
    ka = lda * (k if op_a == oracle.OP_N else m)
    kb = ldb * (n if op_b == oracle.OP_N else k)
    kc = ldc * (n if op_c == oracle.OP_N else m)
    sgn = lambda s: np.where(rng.random(s) < 0.5, -1.0, 1.0)  # noqa: E731
    A = (sgn(ka) * (1 + rng.random(ka)) * 2.0 ** rng.integers(-3, 3, ka)).astype(np.float32)
    B = (sgn(kb) * (1 + rng.random(kb)) * 2.0 ** rng.integers(-2, 2, kb)).astype(np.float16)
    C = rng.standard_normal(kc).astype(np.float32)
    return A, lda, B, ldb, C, ldc


CASES = [(0, 0, 0), (1, 0, 0), (0, 1, 1), (1, 1, 1)]


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
@pytest.mark.parametrize("model", [oracle.IDEAL, oracle.TCMODEL, oracle.B200MODEL])
@pytest.mark.parametrize("ops", CASES)
@pytest.mark.parametrize("chunk,k", [(0, 37), (64, 150)])
def test_oracle_matches_exact_restatement(tc, model, ops, chunk, k):
    op_a, op_b, op_c = ops
    m, n = 5, 4
    rng = np.random.default_rng(1000 * tc + 100 * op_a + 10 * op_b + op_c + k)
    A, lda, B, ldb, C, ldc = _inputs(rng, m, n, k, op_a, op_b, op_c)
    for alpha, beta in ((1.0, 0.0), (-1.25, 0.5)):
        got = C.copy()
        oracle.shgemm(tc, op_a, op_b, m, n, k, alpha, A, lda, B.view(np.uint16), ldb, beta, got, ldc, op_c,
                      chunk, model)
        want = _exact_shgemm(tc, op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, op_c, chunk, model)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (alpha, beta)


def test_rational_rounder_agrees_with_numpy():
    """The rounder itself against numpy's IEEE float32 cast (round to nearest even) and the
    binary16 cast, including subnormals and overflow."""
    rng = np.random.default_rng(5)
    xs = rng.standard_normal(300) * 2.0 ** rng.integers(-160, 130, 300)
    ys = rng.standard_normal(300) * 2.0 ** rng.integers(-28, 17, 300)
    with np.errstate(over="ignore"):
        for x in xs:
            r, want = rn(Fraction(float(x))), np.float32(x)
            assert np.isinf(float(r)) if np.isinf(want) else _f32(r) == want
        for y in ys:
            r, want = _round(Fraction(float(y)), "rne", prec=11, emin=-14, emax=15), np.float16(y)
            assert np.isinf(float(r)) if np.isinf(want) else float(r) == float(want)


@pytest.mark.parametrize("tc", [oracle.FP16, oracle.TF32])
@pytest.mark.parametrize("align_bits", [0, 20, oracle.B200_ALIGN_BITS])
def test_b200_model_alignment_matches_exact_restatement(tc, align_bits):
    """The modelled MMA's alignment and truncation, bit for bit, on inputs whose products span
    a wide range within a fragment (so that alignment drops bits) and with a ragged drain."""
    m, n, k = 4, 3, 70
    rng = np.random.default_rng(40 + align_bits + tc)
    lda, ldb, ldc = m, k, m
    A = (np.where(rng.random(lda * k) < 0.5, -1.0, 1.0) * (1 + rng.random(lda * k))
         * 2.0 ** rng.integers(-3, 3, lda * k)).astype(np.float32)
    B = ((1 + rng.random(ldb * n)) * 2.0 ** rng.integers(-2, 2, ldb * n)).astype(np.float16)
    C = rng.standard_normal(ldc * n).astype(np.float32)
    got = C.copy()
    oracle.shgemm(tc, 0, 0, m, n, k, 1.0, A, lda, B.view(np.uint16), ldb, 0.5, got, ldc, 0, 0, oracle.B200MODEL,
                  align_bits=align_bits)
    want = _exact_shgemm(tc, 0, 0, m, n, k, 1.0, A, lda, B, ldb, 0.5, C, ldc, 0, 0, oracle.B200MODEL, align_bits)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
