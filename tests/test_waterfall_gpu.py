"""The full-device sweep (wimax_ldpc_lib_b200.waterfall) on the GPU, checked
against the oracle decoding the same generated frames.

sweep() generates, decodes and counts on the device. The test replays its
frame source (same seed and frame counters, so the same device-generated
LLRs and codewords), decodes those LLRs with the oracle and recomputes every
counter of every point: frames, frame errors, information-bit errors, the
reference BER_runner's codeword-bit errors over k (reference
lib/BER_runner.cc:148-160,198-199) and iterations."""
import numpy as np
import pytest

from wimax_ldpc_lib_b200 import waterfall

pytestmark = pytest.mark.gpu


def test_sweep_points_match_oracle_on_the_same_frames(wl, cuda, oracle):
    rate, z, batch = 0, 24, 2048
    per_point = 4096                      # sweep's first request: max(4096, ...) frames
    k = wl.code_info(rate, z).k
    points = waterfall.sweep(rate, z, wl.Decoder(rate, z, 10), start=1.5, step=0.5, min_errors=10 ** 9,
                             max_bits=per_point * k, batch=batch, max_points=2, log=lambda *a: None)
    assert [p["ebno_db"] for p in points] == [1.5, 2.0]

    src = waterfall.FrameSource(rate, z, batch)
    for p in points:
        frames = ferr = info_err = cw_err = iters = 0
        while frames < per_point:
            f = src.next(per_point - frames, p["ebno_db"])
            llr = src.llr[:f].cpu().numpy()
            cw = src.cw[:f].cpu().numpy()
            _, dec, _, it, _ = oracle.decode(rate, z, llr, 10)
            diff = dec.view(np.uint8) != cw
            frames += f
            ferr += int(diff[:, :k].any(axis=1).sum())
            info_err += int(diff[:, :k].sum())
            cw_err += int(diff.sum())
            iters += int(it.sum())
        assert p["frames"] == frames
        assert p["fer"] == ferr / frames
        assert p["bit_errors"] == info_err and p["ber"] == info_err / (frames * k)
        assert p["ber_reference_definition"] == cw_err / (frames * k)
        assert p["mean_iterations"] == iters / frames
    assert points[0]["fer"] > points[1]["fer"] > 0     # a waterfall: fewer errors at the higher Eb/N0
    assert points[0]["ebno_db"] < points[1]["ebno_db"]
