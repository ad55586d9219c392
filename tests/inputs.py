"""Deterministic synthetic inputs shared by the tests and tests/golden/make_golden.py.

Everything is derived from PCG64 raw 64-bit outputs (a fixed algorithm) and
basic IEEE-754 double operations, so the same seed gives bit-identical inputs
on every machine; golden fixtures can therefore store digests of outputs
instead of the inputs themselves.

Channel model (the reference's, lib/BER_runner.cc:172-191): BPSK bit*2-1
(positive = bit 1), AWGN with sigma^2 = 1/(2 R Eb/N0), LLR = 2y/sigma^2. The
Gaussian is approximated by an Irwin-Hall sum of four uniforms, which needs no
transcendental function and is exact to reproduce.
"""
from __future__ import annotations

import hashlib

import numpy as np

N_BASE_ROWS = [12, 8, 8, 6, 6, 4]


def code_dims(rate: int, z: int):
    n = 24 * z
    m = N_BASE_ROWS[rate] * z
    return n, m, n - m


def raw(seed: int, count: int) -> np.ndarray:
    return np.random.Generator(np.random.PCG64(seed)).bit_generator.random_raw(count).astype(np.uint64)


def info_bits(seed: int, frames: int, k: int) -> np.ndarray:
    words = (k + 63) // 64
    r = raw(seed, frames * words).reshape(frames, words)
    bits = ((r[:, :, None] >> np.arange(64, dtype=np.uint64)) & np.uint64(1)).astype(np.uint8)
    return bits.reshape(frames, words * 64)[:, :k].copy()


def gaussian(seed: int, shape) -> np.ndarray:
    count = int(np.prod(shape))
    r = raw(seed, 2 * count).reshape(count, 2)
    u = np.empty((count, 4), np.float64)
    u[:, 0] = (r[:, 0] & np.uint64(0xFFFFFFFF)).astype(np.float64)
    u[:, 1] = (r[:, 0] >> np.uint64(32)).astype(np.float64)
    u[:, 2] = (r[:, 1] & np.uint64(0xFFFFFFFF)).astype(np.float64)
    u[:, 3] = (r[:, 1] >> np.uint64(32)).astype(np.float64)
    u = (u + 0.5) * (1.0 / 4294967296.0)
    s = ((u[:, 0] + u[:, 1]) + (u[:, 2] + u[:, 3])) - 2.0
    return (s * 1.7320508075688772).reshape(shape)


def awgn_llr(cw: np.ndarray, rate_r: float, ebno_db: float, seed: int) -> np.ndarray:
    sigma2 = 1.0 / (2.0 * rate_r * 10.0 ** (ebno_db / 10.0))
    sigma = np.sqrt(sigma2)
    y = (cw.astype(np.float64) * 2.0 - 1.0) + sigma * gaussian(seed, cw.shape)
    return (y * (2.0 / sigma2)).astype(np.float32)


def frames(oracle, rate: int, z: int, count: int, ebno_db: float, seed: int):
    """(info, codeword, llr) for `count` frames; rate 3/4B (no encoder) uses
    the all-zero codeword, which is a codeword of every linear code."""
    n, m, k = code_dims(rate, z)
    if rate == 4:
        info = np.zeros((count, k), np.uint8)
        cw = np.zeros((count, n), np.uint8)
    else:
        info = info_bits(seed, count, k)
        cw = oracle.encode(rate, z, info)
    return info, cw, awgn_llr(cw, k / n, ebno_db, seed + 1)


def edge_llr(kind: str, rate: int, z: int, count: int, seed: int, oracle=None) -> np.ndarray:
    """Hand-made edge cases: exact +-0 LLRs, many ties, magnitudes beyond the
    decoder's 10000 clamp, valid codewords, pure noise."""
    n, m, k = code_dims(rate, z)
    g = gaussian(seed, (count, n))
    if kind == "zeros":
        x = g.astype(np.float32)
        x[:, ::7] = 0.0
        x[:, 3::11] = -0.0
        return x
    if kind == "ties":
        return np.clip(np.round(g * 1.5), -3, 3).astype(np.float32)
    if kind == "huge":
        return (g * 30000.0).astype(np.float32)
    if kind == "valid":
        info = info_bits(seed, count, k)
        cw = oracle.encode(rate, z, info) if rate != 4 else np.zeros((count, n), np.uint8)
        return ((cw.astype(np.float32) * 2 - 1) * 3).astype(np.float32)
    if kind == "noise":
        return (g * 0.3).astype(np.float32)
    raise ValueError(kind)


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:16]


def frame_digests(posterior: np.ndarray, decoded: np.ndarray):
    return [digest(posterior[f], decoded[f]) for f in range(posterior.shape[0])]


# Eb/N0 per rate for the all-variants sweep: mid-waterfall so that frames need
# several iterations and some fail.
SWEEP_EBNO = {0: 2.0, 1: 2.5, 2: 2.5, 3: 3.0, 4: 3.0, 5: 3.5}
