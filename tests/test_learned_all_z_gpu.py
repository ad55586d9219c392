"""The learned decoders at every one of the 114 codes (6 rates x 19 z): the
fp32 and packed-binary16 kernels bit-exact against the oracle's
restatements, the fp32 kernel with unit weights bit-exact against the
reference's own min-sum build at z values that are not multiples of 32 (CTAs
of several frames with a partial last warp), the training gradient at such z
against the oracle's, and the shipped-weight lookup for codes without a
table of their own."""
import numpy as np
import pytest

import inputs
from oracle.oracle import MS, Reference, reference_available
from test_learned_oracle import random_weights

pytestmark = pytest.mark.gpu

ALL_CODES = [(r, z) for r in range(6) for z in range(24, 97, 4)]


@pytest.mark.parametrize("rate,z", ALL_CODES)
def test_learned_fp32_and_f16x2_match_oracle_at_every_code(wl, cuda, oracle, rate, z):
    T = 8
    w, _, _ = random_weights(oracle, rate, z, T, 1000 + 31 * rate + z)
    w[1] = np.abs(w[1])                          # in the binary16 decoder's range
    frames = 24 + (z // 4) % 7                   # odd and even counts: a binary16 frame without a partner
    _, _, llr = inputs.frames(oracle, rate, z, frames, inputs.SWEEP_EBNO[rate] - 0.25, seed=5000 + 31 * rate + z)
    po, do, io, so = oracle.learned_decode(rate, z, T, w, llr, cap=10)
    post, hard, _, st = wl.LearnedDecoder(rate, z, T, weights=w, cap=10).decode_host(llr)
    assert (post.view(np.uint32) == po.view(np.uint32)).all(), "fp32 posterior"
    assert (hard == do).all() and ((st & 0xFFFF) == io).all() and (((st >> 16) & 1) == so).all(), "fp32"
    po, do, io, so = oracle.learned16_decode(rate, z, T, w, llr, cap=10)
    post, hard, _, st = wl.LearnedDecoder(rate, z, T, weights=w, cap=10, precision=wl.LMS_F16X2).decode_host(llr)
    assert (post.view(np.uint32) == po.view(np.uint32)).all(), "binary16 posterior"
    assert (hard == do).all() and ((st & 0xFFFF) == io).all() and (((st >> 16) & 1) == so).all(), "binary16"


@pytest.mark.skipif(not reference_available(MS), reason="oracle/_ref (reference MS build) not built")
@pytest.mark.parametrize("rate,z", [(0, 28), (1, 92), (2, 60), (3, 44), (4, 76), (5, 36), (0, 84), (3, 52)])
def test_unit_weight_learned_decoder_equals_reference_at_odd_z(wl, cuda, oracle, rate, z):
    w = np.zeros((2, 8, 12, 24), np.float32)
    w[0] = 1.0
    _, _, llr = inputs.frames(oracle, rate, z, 150, inputs.SWEEP_EBNO[rate] - 0.25, seed=7700 + z + rate)
    po, do, ro = Reference(MS).decode(rate, z, llr, 10)
    post, hard, ne, st = wl.LearnedDecoder(rate, z, 8, weights=w, cap=10).decode_host(llr)
    assert (post.view(np.uint32) == po.view(np.uint32)).all() and (hard == do).all() and (ne == ro).all()


@pytest.mark.parametrize("rate,z", [(0, 28), (3, 92), (5, 60)])
def test_learned_gradient_matches_oracle_at_odd_z(wl, cuda, oracle, rate, z):
    T = 8
    w, _, _ = random_weights(oracle, rate, z, T, 17)
    _, cw, llr = inputs.frames(oracle, rate, z, 24, 1.75, seed=78)
    loss_o, g_o = oracle.learned_loss_grad(rate, z, T, w, llr, cw)
    loss_g, g_g = wl.LearnedDecoder(rate, z, T, weights=w).loss_grad(llr, cw)
    g_o = g_o.reshape(g_g.shape)
    assert abs(loss_g - loss_o) <= 1e-5 * abs(loss_o)
    assert np.linalg.norm(g_g - g_o) <= 1e-4 * np.linalg.norm(g_o)


def test_transferred_weights_decode_every_code(wl, cuda):
    """Every code gets a weight table (its own or its rate's nearest trained
    z), and the learned decoder runs with it on generated frames."""
    import torch
    for rate in range(6):
        for z in (24, 60, 92):
            meta, w, src_z = wl.learned_weights(rate, z, evaluated_only=False)
            assert w is not None and src_z in (48, 96)
            n = 24 * z
            llr = torch.empty((512, n), dtype=torch.float32, device="cuda")
            cw = torch.empty((512, n), dtype=torch.uint8, device="cuda")
            wl.framegen_nullspace_device(rate, z, 5, 0, 512, 4.5, 4.5, codeword=cw, llr=llr)
            hard = torch.empty((512, n), dtype=torch.int8, device="cuda")
            dec = wl.LearnedDecoder(rate, z, meta["iterations"], weights=w, cap=10)
            dec.decode_device(llr, hard)
            torch.cuda.synchronize()
            assert (hard.view(torch.uint8) != cw).any(dim=1).float().mean().item() < 0.01
