"""The learned min-sum kernels pinned to the reference itself.

With every scale a = 1 and every offset b = 0 the learned message
s * relu(fma(a, mu, -b)) is s * mu, which is exactly the reference's plain
min-sum branch (reference lib/ldpc_decoder.cc:233-235: m_LMN = iter_sign *
minimum; rx = LNM + iter_sign * minimum, all float), with the same layer
order, sign rule, stopping rule and cap (lib/ldpc_decoder.cc:122-262). The
reference built with that branch selected (oracle/_ref/libwldpc_ref_ms.so,
its own sources with the NMS switch flipped) must therefore agree with the
fp32 learned kernel bit for bit -- posteriors, hard bits, return values and
iteration counts -- on AWGN frames, where no LLR is -0 and no magnitude
reaches the reference's 10000 clamp (the two places the learned model
deliberately differs). This ties the learned kernel's control flow to the
reference rather than to a restatement written alongside it."""
import numpy as np
import pytest

import inputs
from oracle.oracle import MS, Reference, reference_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not reference_available(MS), reason="oracle/_ref (reference MS build) not built")]

T = 8


def unit_weights():
    w = np.zeros((2, T, 12, 24), np.float32)
    w[0] = 1.0
    return w


@pytest.mark.parametrize("z", [24, 48, 96])
@pytest.mark.parametrize("rate", range(6))
def test_unit_weight_learned_decoder_equals_reference_min_sum(wl, cuda, oracle, rate, z):
    ref = Reference(MS)
    frames = 96 if z == 96 else 160
    # mid-waterfall, so frames take several iterations and some reach the cap
    _, _, llr = inputs.frames(oracle, rate, z, frames, inputs.SWEEP_EBNO[rate] - 0.25, seed=9100 + 10 * z + rate)
    assert np.abs(llr).max() < 1000 and not (llr == 0).any()
    po, do, ro = ref.decode(rate, z, llr, 10)
    io = ref.iterations(rate, z, llr, 10)
    lms = wl.LearnedDecoder(rate, z, T, weights=unit_weights(), cap=10)
    post, hard, ne, st = lms.decode_host(llr)
    assert (post.view(np.uint32) == po.view(np.uint32)).all(), "posterior differs from the reference"
    assert (hard == do).all(), "hard decisions differ from the reference"
    assert (ne == ro).all(), "return values differ from the reference"
    it = st & 0xFFFF
    # the reference's iteration count: 0 if the input already satisfies the
    # syndrome, else the first cap at which it succeeds, cap + 1 on failure
    assert (np.where((st >> 16) & 1, 11, it) == io).all(), "iteration counts differ from the reference"
    assert it.max() >= 3                                        # the decoder actually iterated


def test_unit_weight_learned_decoder_device_call_equals_reference(wl, cuda, oracle):
    """The device-pointer entry point on a larger r1/2 z=96 batch near the FER
    knee (some frames fail at the cap)."""
    rate, z = 0, 96
    ref = Reference(MS)
    _, _, llr = inputs.frames(oracle, rate, z, 1024, 1.5, seed=9999)
    po, do, ro = ref.decode(rate, z, llr, 10)
    lms = wl.LearnedDecoder(rate, z, T, weights=unit_weights(), cap=10)
    d_llr = cuda.from_numpy(llr).cuda()
    hard = cuda.empty(d_llr.shape, dtype=cuda.int8, device="cuda")
    post = cuda.empty_like(d_llr)
    status = cuda.empty(llr.shape[0], dtype=cuda.int32, device="cuda")
    lms.decode_device(d_llr, hard, post, status)
    cuda.cuda.synchronize()
    st = status.cpu().numpy()
    assert (post.cpu().numpy().view(np.uint32) == po.view(np.uint32)).all()
    assert (hard.cpu().numpy() == do).all()
    assert (((st >> 16) & 1) == ro).all() and ro.sum() > 0
