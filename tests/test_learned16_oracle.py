"""The binary16 restatement of the packed-half learned decoder: its rounding
primitives against independent references (numpy's correctly rounded
double -> half conversion, exact rational arithmetic), and its decoder
against the float learned decoder on the same frames and weights."""
import math
from fractions import Fraction

import numpy as np

import inputs
from test_learned_oracle import random_weights

HALF_MAX = 65504.0


def round_half_exact(v: Fraction) -> float:
    """nearest binary16 value of an exact rational (ties to even)."""
    if v == 0:
        return 0.0
    sign = -1.0 if v < 0 else 1.0
    a = abs(v)
    e = a.numerator.bit_length() - a.denominator.bit_length()
    while Fraction(2) ** e > a:
        e -= 1
    while Fraction(2) ** (e + 1) <= a:
        e += 1
    q = e - 10 if e >= -14 else -24
    sc = a / Fraction(2) ** q
    fl = sc.numerator // sc.denominator
    rem = sc - fl
    if rem > Fraction(1, 2) or (rem == Fraction(1, 2) and fl % 2 == 1):
        fl += 1
    val = fl * Fraction(2) ** q
    return sign * math.inf if val > HALF_MAX else sign * float(val)


def random_halves(rng, count, lo, hi):
    return np.clip(rng.uniform(lo, hi, count), lo, hi).astype(np.float16).astype(np.float64)


def test_half_round_matches_numpy(oracle):
    rng = np.random.default_rng(1)
    xs = np.concatenate([
        rng.standard_normal(20000) * 10.0 ** rng.uniform(-9, 5, 20000),
        # exact sums and differences of two binary16 numbers (what the decoder rounds)
        random_halves(rng, 5000, -3000, 3000) + random_halves(rng, 5000, -40, 40),
        random_halves(rng, 5000, -1e-3, 1e-3) - random_halves(rng, 5000, -1e-5, 1e-5),
        # ties: midpoints between neighbouring binary16 values, subnormal and normal
        (np.arange(1, 4000, dtype=np.float64) + 0.5) * 2.0 ** -24,
        (np.arange(1024, 2048, dtype=np.float64) + 0.5) * 2.0 ** -3,
        np.array([65504.0, 65519.99, 65520.0, 70000.0, -65520.0, 2.0 ** -25, -2.0 ** -25, 3 * 2.0 ** -26]),
    ])
    got = np.array([oracle.half_round(x) for x in xs])
    with np.errstate(over="ignore"):
        want = xs.astype(np.float16).astype(np.float64)
    assert np.array_equal(got, want, equal_nan=True)
    assert math.copysign(1.0, oracle.half_round(-2.0 ** -26)) == -1.0   # rounds to -0


def test_half_fma_relu_matches_exact_rounding(oracle):
    rng = np.random.default_rng(2)
    a = random_halves(rng, 4000, -2.0, 2.0)
    b = random_halves(rng, 4000, 0.0, 2048.0)
    c = random_halves(rng, 4000, -1024.0, 1024.0)
    cases = list(zip(a, b, c))
    # a*b + c exactly on a binary16 tie (1 + 2^-11 between 1 and 1 + 2^-10), and near the top
    cases += [(1.0, 1.0, 2.0 ** -11), (1.0, 1.0 + 2.0 ** -10, 2.0 ** -11), (-1.0, 1.0, -(2.0 ** -11)),
              (2.0, 2048.0, -0.5), (0.8149, 2048.0, -0.12), (1.5, 2047.0, 1000.0), (0.5, 3.0, -1.5)]
    for x, y, w in cases:
        want = round_half_exact(Fraction(x) * Fraction(y) + Fraction(w))
        want = 0.0 if want < 0 else want
        assert oracle.half_fma_relu(x, y, w) == want, (x, y, w)


def test_learned16_decoder_tracks_the_float_decoder(oracle):
    """Same weights, same frames: the binary16 decoder is the float decoder
    rounded to binary16, so it decodes (nearly) the same frames and its
    posteriors are binary16 values."""
    rate, z, T = 0, 48, 8
    w, _, _ = random_weights(oracle, rate, z, T, 11)
    info, cw, llr = inputs.frames(oracle, rate, z, 512, 2.0, seed=21)
    p32, d32, i32, s32 = oracle.learned_decode(rate, z, T, w, llr, cap=10)
    p16, d16, i16, s16 = oracle.learned16_decode(rate, z, T, w, llr, cap=10)
    assert np.array_equal(p16.astype(np.float16).astype(np.float32), p16)
    k = info.shape[1]
    fe32 = int((d32[:, :k] != info).any(axis=1).sum())
    fe16 = int((d16[:, :k] != info).any(axis=1).sum())
    assert fe16 <= fe32 + 2, (fe16, fe32)
    assert (d16 == d32).all(axis=1).mean() >= 0.98
    assert abs(float(i16.mean()) - float(i32.mean())) < 0.1
    assert (s16 == 0).sum() >= (s32 == 0).sum() - 2


def test_learned16_clamps_and_zero_signs(oracle):
    """Input handling: LLRs beyond +-2048 (and inf, NaN) clamp, -0 and tiny
    negatives stage as +0 (hard bit 1), and a valid codeword stops at 0
    iterations with its posteriors equal to the staged inputs."""
    rate, z, T = 0, 24, 8
    w, _, _ = random_weights(oracle, rate, z, T, 12)
    n = 24 * z
    _, cw, _ = inputs.frames(oracle, rate, z, 1, 3.0, seed=31)
    llr = np.where(cw == 1, 5.0, -5.0).astype(np.float32)
    llr[0, 0] = 1e6 if cw[0, 0] else -1e6
    llr[0, 1] = np.inf if cw[0, 1] else -np.inf
    post, dec, it, sf = oracle.learned16_decode(rate, z, T, w, llr, cap=10)
    assert it[0] == 0 and sf[0] == 0 and (dec == cw).all()
    assert abs(post[0, 0]) == 2048.0 and abs(post[0, 1]) == 2048.0
    zeros = np.full((1, n), -0.0, np.float32)
    zeros[0, 1::2] = -1e-9
    post, dec, it, sf = oracle.learned16_decode(rate, z, T, w, zeros, cap=0)
    assert (dec == 1).all() and not np.signbit(post).any()
