"""Packed-half (f16x2) learned decoder on the GPU: bit-exact against the
oracle's binary16 restatement (posteriors, hard bits, iterations, syndrome
flags) for several codes, odd batch sizes (a frame without a partner), caps
below and past the trained iterations, clamped and signed-zero inputs, the
device and host entry points, the weight-range check, and its frame error
rate against the plain decoder on the shipped weights."""
import json
import os

import numpy as np
import pytest

import inputs
from test_learned_oracle import random_weights as random_weights_any

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def random_weights(oracle, rate, z, T, seed):
    """random weights in the packed-half decoder's range (offsets b >= 0)"""
    w, rs, cols = random_weights_any(oracle, rate, z, T, seed)
    w[1] = np.abs(w[1])
    return w, rs, cols


def check_equal(out, ref):
    post, hard, st = out
    po, do, io, so = ref
    assert (post.view(np.uint32) == po.view(np.uint32)).all(), "posterior"
    assert (hard == do).all(), "hard bits"
    assert ((st & 0xFFFF) == io).all(), "iterations"
    assert (((st >> 16) & 1) == so).all(), "syndrome flag"


# every code the learned decoder supports (6 rates x z = 24, 48, 96), odd and even batch sizes
CODES16 = [(0, 96, 257), (0, 48, 131), (0, 24, 203), (1, 96, 64), (1, 48, 41), (1, 24, 66), (2, 96, 39),
           (2, 48, 75), (2, 24, 50), (3, 96, 45), (3, 48, 52), (3, 24, 97), (4, 96, 33), (4, 48, 70),
           (4, 24, 81), (5, 96, 36), (5, 48, 129), (5, 24, 58)]


@pytest.mark.parametrize("rate,z,frames", CODES16)
def test_learned16_decode_matches_oracle(wl, cuda, oracle, rate, z, frames):
    T = 8
    w, _, _ = random_weights(oracle, rate, z, T, 40 + rate * 3 + z)
    _, _, llr = inputs.frames(oracle, rate, z, frames, inputs.SWEEP_EBNO[rate] - 0.25, seed=900 + z + rate)
    ref = oracle.learned16_decode(rate, z, T, w, llr, cap=10)
    lms = wl.LearnedDecoder(rate, z, T, weights=w, cap=10, precision=wl.LMS_F16X2)
    post, hard, _, st = lms.decode_host(llr)
    check_equal((post, hard, st), ref)
    assert ref[2].max() > 1   # frames decode for several iterations


@pytest.mark.parametrize("cap", [1, 3, 12])
def test_learned16_caps_match_oracle(wl, cuda, oracle, cap):
    rate, z, T = 0, 96, 4
    w, _, _ = random_weights(oracle, rate, z, T, 9)
    _, _, llr = inputs.frames(oracle, rate, z, 96, 1.5, seed=13)
    ref = oracle.learned16_decode(rate, z, T, w, llr, cap=cap)
    post, hard, _, st = wl.LearnedDecoder(rate, z, T, weights=w, cap=cap, precision=wl.LMS_F16X2).decode_host(llr)
    check_equal((post, hard, st), ref)


def test_learned16_device_entry_and_edge_inputs(wl, cuda, oracle):
    """Device buffers, the float learned decoder's own test frames plus edge
    inputs: huge, infinite and NaN LLRs, -0 and tiny negatives, a valid
    codeword (0 iterations) and pure noise (cap reached)."""
    torch = cuda
    rate, z, T = 0, 24, 8
    w, _, _ = random_weights(oracle, rate, z, T, 77)
    _, cw, llr = inputs.frames(oracle, rate, z, 12, 2.0, seed=71)
    llr = llr.copy()
    llr[0] *= 1e5
    llr[1, ::7] = np.inf
    llr[2, ::5] = -np.inf
    llr[3, ::3] = np.nan
    llr[4] = -0.0
    llr[5, ::2] = -1e-9
    llr[6] = np.where(cw[6] == 1, 4.0, -4.0)
    rng = np.random.default_rng(5)
    llr[7] = rng.standard_normal(llr.shape[1]).astype(np.float32)
    ref = oracle.learned16_decode(rate, z, T, w, llr, cap=10)
    lms = wl.LearnedDecoder(rate, z, T, weights=w, cap=10, precision=wl.LMS_F16X2)
    d_llr = torch.from_numpy(llr).cuda()
    hard = torch.empty(llr.shape, dtype=torch.int8, device="cuda")
    post = torch.empty_like(d_llr)
    st = torch.empty(llr.shape[0], dtype=torch.int32, device="cuda")
    lms.decode_device(d_llr, hard, post, st)
    torch.cuda.synchronize()
    check_equal((post.cpu().numpy(), hard.cpu().numpy(), st.cpu().numpy()), ref)
    assert ref[2][6] == 0 and ref[3][7] == 1


def test_learned16_rejects_out_of_range_weights(wl, cuda, oracle):
    rate, z, T = 0, 48, 2
    w, rs, cols = random_weights(oracle, rate, z, T, 3)
    lms = wl.LearnedDecoder(rate, z, T, weights=w)
    lms.set_precision(wl.LMS_F16X2)
    bad = w.copy()
    bad[0, 0, 0, cols[0]] = 2.5
    lms.set_weights(bad)
    with pytest.raises(wl.LdpcError):
        lms.decode_host(np.zeros((2, 24 * z), np.float32))
    lms2 = wl.LearnedDecoder(rate, z, T, weights=bad)
    with pytest.raises(wl.LdpcError):
        lms2.set_precision(wl.LMS_F16X2)
    neg = w.copy()
    neg[1, 1, 2, cols[rs[2]]] = -0.01          # offsets must be >= 0
    lms3 = wl.LearnedDecoder(rate, z, T, weights=neg)
    with pytest.raises(wl.LdpcError):
        lms3.set_precision(wl.LMS_F16X2)
    with pytest.raises(wl.LdpcError):
        lms2.set_precision(7)


def test_learned16_shipped_weights_fer(wl, cuda):
    """The shipped r1/2 z=96 weights decoded in binary16: on held-out frames
    at 2.0 dB and the reference's cap of 10 the frame error rate is no worse
    than the plain normalized min-sum's and within a few frames of the fp32
    learned decoder's."""
    path = os.path.join(ROOT, "wimax_ldpc_lib_b200", "weights", "lms_r0_z96_T8.json")
    meta = json.load(open(path))
    w = np.array(meta["weights"], np.float32)
    torch = cuda
    frames, rate, z = 131072, 0, 96
    llr = torch.empty((frames, 2304), dtype=torch.float32, device="cuda")
    info = torch.empty((frames, 1152), dtype=torch.uint8, device="cuda")
    wl.framegen_device(rate, z, 0xF16, 1 << 41, frames, 2.0, 2.0, info=info, llr=llr)
    errs = {}
    for name, dec in [("f16x2", wl.LearnedDecoder(rate, z, 8, weights=w, cap=10, precision=wl.LMS_F16X2)),
                      ("f32", wl.LearnedDecoder(rate, z, 8, weights=w, cap=10)),
                      ("plain", wl.Decoder(rate, z, 10))]:
        hard = torch.empty((frames, 2304), dtype=torch.int8, device="cuda")
        st = torch.empty(frames, dtype=torch.int32, device="cuda")
        dec.decode_device(llr, hard, None, st)
        torch.cuda.synchronize()
        errs[name] = int((hard[:, :1152].view(torch.uint8) != info).any(dim=1).sum().item())
    assert errs["f16x2"] <= errs["plain"], errs
    assert errs["f16x2"] <= errs["f32"] + max(5, errs["f32"] // 10), errs
