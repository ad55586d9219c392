"""Learned min-sum on the GPU: inference bit-exact against the oracle's
float restatement, the training kernels' loss and gradient against the
oracle, training lowering the loss, and the shipped weights' gain over the
plain normalized min-sum at the same iteration budget."""
import json
import os

import numpy as np
import pytest

import inputs
from test_learned_oracle import random_weights

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("rate,z", [(0, 96), (0, 24), (5, 48), (2, 96), (3, 24)])
def test_learned_decode_matches_oracle(wl, cuda, oracle, rate, z):
    T = 8
    w, _, _ = random_weights(oracle, rate, z, T, rate * 7 + z)
    _, _, llr = inputs.frames(oracle, rate, z, 256, inputs.SWEEP_EBNO[rate] - 0.25, seed=600 + z + rate)
    po, do, io, so = oracle.learned_decode(rate, z, T, w, llr)
    lms = wl.LearnedDecoder(rate, z, T, weights=w)
    assert np.array_equal(lms.get_weights(), w)
    post, hard, ne, st = lms.decode_host(llr)
    assert (post.view(np.uint32) == po.view(np.uint32)).all()
    assert (hard == do).all()
    assert ((st & 0xFFFF) == io).all() and (((st >> 16) & 1) == so).all()


def test_learned_decode_past_trained_iterations_matches_oracle(wl, cuda, oracle):
    rate, z, T = 0, 96, 4
    w, _, _ = random_weights(oracle, rate, z, T, 3)
    _, _, llr = inputs.frames(oracle, rate, z, 256, 1.75, seed=5)
    po, do, io, so = oracle.learned_decode(rate, z, T, w, llr, cap=10)
    post, hard, ne, st = wl.LearnedDecoder(rate, z, T, weights=w, cap=10).decode_host(llr)
    assert (post.view(np.uint32) == po.view(np.uint32)).all() and (hard == do).all()
    assert ((st & 0xFFFF) == io).all() and io.max() > T


@pytest.mark.parametrize("rate,z", [(0, 96), (0, 24), (4, 48), (5, 96)])
def test_learned_gradient_matches_oracle(wl, cuda, oracle, rate, z):
    T = 8
    w, _, _ = random_weights(oracle, rate, z, T, 5)
    _, cw, llr = inputs.frames(oracle, rate, z, 32, 1.75, seed=77)
    loss_o, g_o = oracle.learned_loss_grad(rate, z, T, w, llr, cw)
    lms = wl.LearnedDecoder(rate, z, T, weights=w)
    loss_g, g_g = lms.loss_grad(llr, cw)
    g_o = g_o.reshape(g_g.shape)
    # float accumulation on the GPU vs double in the oracle, same decisions
    assert abs(loss_g - loss_o) <= 1e-5 * abs(loss_o)
    assert np.linalg.norm(g_g - g_o) <= 1e-4 * np.linalg.norm(g_o)


@pytest.mark.parametrize("rate,z,ebno", [(0, 24, 1.0), (4, 24, 2.0), (5, 48, 2.75)])
def test_training_lowers_the_loss(wl, cuda, rate, z, ebno):
    """Device training (frames from the encoder, or null-space codewords for
    3/4B, which has no encoder) lowers the BCE loss."""
    lms = wl.LearnedDecoder(rate, z, 8)
    hist = lms.train(steps=60, batch=512, ebno_lo=ebno, ebno_hi=ebno + 2.0, seed=9, lr=1e-2)
    assert hist[-10:].mean() < hist[:10].mean()
    w = lms.get_weights()
    assert np.isfinite(w).all() and not np.all(w[0][w[0] != 0] == np.float32(0.815))


def test_shipped_weights_gain_over_plain(wl, cuda):
    """The trained network against the method without it: at the same budget
    of 8 iterations, on held-out frames at 2.0 dB, the learned decoder's FER is
    no worse than plain normalized min-sum's and it needs fewer iterations."""
    path = os.path.join(ROOT, "wimax_ldpc_lib_b200", "weights", "lms_r0_z96_T8.json")
    if not os.path.exists(path):
        pytest.skip("no trained weights shipped")
    meta = json.load(open(path))
    torch = cuda
    frames, rate, z = 131072, 0, 96
    llr = torch.empty((frames, 2304), dtype=torch.float32, device="cuda")
    info = torch.empty((frames, 1152), dtype=torch.uint8, device="cuda")
    wl.framegen_device(rate, z, 0xE7A1, 1 << 40, frames, 2.0, 2.0, info=info, llr=llr)
    res = {}
    for name, dec in [("learned", wl.LearnedDecoder(rate, z, 8, weights=np.array(meta["weights"], np.float32))),
                      ("plain8", wl.Decoder(rate, z, 8))]:
        hard = torch.empty((frames, 2304), dtype=torch.int8, device="cuda")
        st = torch.empty(frames, dtype=torch.int32, device="cuda")
        dec.decode_device(llr, hard, None, st)
        torch.cuda.synchronize()
        fer = (hard[:, :1152].view(torch.uint8) != info).any(dim=1).double().mean().item()
        res[name] = (fer, (st & 0xFFFF).double().mean().item())
    assert res["learned"][0] <= res["plain8"][0], res
    assert res["learned"][1] < res["plain8"][1], res


def test_split_training_step_equals_train(wl, cuda):
    """wldpc_lms_step_grad + wldpc_lms_apply_grad (the data-parallel pieces)
    give bit-identical weights to wldpc_lms_train on the same frames."""
    torch = cuda
    a, b = wl.LearnedDecoder(0, 24, 8), wl.LearnedDecoder(0, 24, 8)
    g = torch.zeros(b.grad_size(), dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    for s in range(3):
        a.train(1, 256, 1.0, 3.0, 17, first_frame=s * 256, lr=1e-2)
        b.step_grad(256, 1.0, 3.0, 17, s * 256, g, loss)
        b.apply_grad(g, 1e-2)
    assert np.array_equal(a.get_weights(), b.get_weights())
    assert float(loss.item()) > 0


def test_rank_gradients_average_to_the_job_gradient(wl, cuda):
    """Two ranks' half batches (frames [0, 256) and [256, 512)) average to the
    gradient of the whole batch, as the all-reduce in data-parallel training
    assumes (float sums in a different order: 1e-5 relative)."""
    torch = cuda
    h = wl.LearnedDecoder(0, 48, 8)
    n = h.grad_size()
    full, r0, r1 = (torch.zeros(n, dtype=torch.float32, device="cuda") for _ in range(3))
    h.step_grad(512, 1.0, 3.0, 5, 0, full)
    h.step_grad(256, 1.0, 3.0, 5, 0, r0)
    h.step_grad(256, 1.0, 3.0, 5, 256, r1)
    avg = (r0 + r1) / 2
    assert torch.linalg.norm(avg - full) <= 1e-5 * torch.linalg.norm(full)
