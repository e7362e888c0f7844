"""Generates the golden fixtures in this directory.

The reference keeps no golden values (its test programs only print errors) and
its arithmetic module is not vendored, so these vectors come from independent
implementations of the documented conversions the reference's split uses
(src/wmmae_shgemm.hpp:30-31, scale 2^11):

* split_fp16.npz -- numpy's IEEE-754 binary16 cast (round to nearest even,
  gradual underflow, overflow to inf) applied to the split formula.
* split_tf32.npz -- exact rational (fractions.Fraction) rounding to an 11-bit
  significand, ties away from zero (cvt.rna.tf32.f32 semantics).
* gemm_exact.npz -- a small product whose every partial sum is exact, so the
  full algorithm's result is known exactly in float64.

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def edge_values() -> np.ndarray:
    v = [0.0, -0.0, 1.0, -1.0, 1.0 / 3.0, -2.0 / 3.0, 65504.0, 65519.99, 65520.0, -65520.0,
         70000.0, 1e-8, -1e-8, 2.0 ** -24, 2.0 ** -25, 3 * 2.0 ** -26, 2.0 ** -14, 2.0 ** -15 * 1.5,
         2.0 ** -30, 2.0 ** -35, 2.0 ** -40, 1.0000001, 3.1415927, 1e30, -1e-30, 2.0 ** -126,
         2.0 ** -130, float("inf"), float("-inf")]
    return np.array(v, dtype=np.float32)


def random_values(rng, n) -> np.ndarray:
    a = rng.standard_normal(n).astype(np.float32)
    e = rng.uniform(-15, 15, n)
    wide = (rng.standard_normal(n) * np.exp2(e)).astype(np.float32)
    tiny = (rng.uniform(-1, 1, n) * np.exp2(rng.uniform(-40, -14, n))).astype(np.float32)
    bits = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32).view(np.float32)
    bits = bits[np.isfinite(bits)]
    return np.concatenate([a, wide, tiny, bits])


def split_fp16(v: np.ndarray):
    with np.errstate(over="ignore", invalid="ignore"):
        hi = v.astype(np.float16)
        lo = ((v - hi.astype(np.float32)) * np.float32(2048.0)).astype(np.float16)
    return hi.view(np.uint16), lo.view(np.uint16)


def _rna_tf32(x: float) -> float:
    if not np.isfinite(x) or x == 0.0:
        return float(np.float32(x))
    fr = Fraction(abs(x))
    e = fr.numerator.bit_length() - fr.denominator.bit_length()
    if Fraction(2) ** e > fr:
        e -= 1
    e = max(e, -126)  # binary32 subnormals keep the 2^-136 quantum of the lowest binade
    q = Fraction(2) ** (e - 10)
    n = fr / q
    r = int(n)
    if n - r >= Fraction(1, 2):
        r += 1
    val = r * q
    if val >= Fraction(2) ** 128:
        out = float("inf")
    else:
        out = float(val)
    return -out if x < 0 else out


def split_tf32(v: np.ndarray):
    hi = np.array([_rna_tf32(float(x)) for x in v], dtype=np.float32)
    with np.errstate(over="ignore", invalid="ignore"):
        d = (v - hi) * np.float32(2048.0)
    lo = np.array([_rna_tf32(float(x)) for x in d], dtype=np.float32)
    return hi, lo


def gemm_exact(rng):
    """A holds 12-bit fixed-point values (one bit more than an FP16/TF32 significand),
    B small integers: hi + lo recovers A exactly and every partial sum is exact in
    binary32, so the algorithm's result equals the float64 product bit for bit.
    Rounding A to the compute type alone (no lo term) would not."""
    m, n, k = 37, 19, 96
    N = rng.integers(-4095, 4096, (m, k))
    A = (N / 4096.0).astype(np.float32)
    B = rng.integers(-8, 9, (k, n)).astype(np.float16)
    C64 = A.astype(np.float64) @ B.astype(np.float64)
    return dict(m=m, n=n, k=k, A=A.ravel(order="F"),
                B=B.ravel(order="F").view(np.uint16), C=C64.ravel(order="F"))


def main():
    rng = np.random.default_rng(20240611)
    v = np.concatenate([edge_values(), random_values(rng, 4000)])
    hi16, lo16 = split_fp16(v)
    np.savez_compressed(os.path.join(HERE, "split_fp16.npz"), v=v, hi=hi16, lo=lo16)
    vt = np.concatenate([edge_values(), random_values(rng, 1500)])
    hit, lot = split_tf32(vt)
    np.savez_compressed(os.path.join(HERE, "split_tf32.npz"), v=vt, hi=hit, lo=lot)
    np.savez_compressed(os.path.join(HERE, "gemm_exact.npz"), **gemm_exact(rng))
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
