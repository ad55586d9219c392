"""The learned min-sum oracle: its analytic gradient against central finite
differences where a perturbation cannot cross a min / argmin / relu kink (the
loss is piecewise smooth), and its float forward against plain NMS when the
weights are the normalized min-sum constants."""
import numpy as np

import inputs


def random_weights(oracle, rate, z, T, seed):
    rs, cols, _ = oracle.code_blocks(rate, z)
    rng = np.random.default_rng(seed)
    w = np.zeros((2, T, 12, 24), np.float32)
    for t in range(T):
        for i in range(len(rs) - 1):
            for b in range(rs[i], rs[i + 1]):
                w[0, t, i, cols[b]] = 0.8 + 0.1 * rng.standard_normal()
                w[1, t, i, cols[b]] = 0.05 + 0.02 * rng.standard_normal()
    return w, rs, cols


def test_learned_gradient_matches_finite_differences(oracle):
    rate, z, T = 0, 24, 4
    _, cw, llr = inputs.frames(oracle, rate, z, 16, 1.5, seed=3)
    w, rs, cols = random_weights(oracle, rate, z, T, 0)
    loss, g = oracle.learned_loss_grad(rate, z, T, w, llr, cw)
    g = g.reshape(w.shape)
    assert 0.05 < loss < 1.0
    # weights of the last layers of the last iteration move no later decision
    for ix in [(0, T - 1, 11, cols[rs[11]]), (0, T - 1, 11, cols[rs[11] + 3]), (0, T - 1, 10, cols[rs[10] + 2])]:
        eps = 1e-3
        wp, wm = w.copy(), w.copy()
        wp[ix] += eps
        wm[ix] -= eps
        fd = (oracle.learned_loss_grad(rate, z, T, wp, llr, cw)[0] - oracle.learned_loss_grad(rate, z, T, wm, llr, cw)[0]) / (2 * eps)
        assert abs(fd - g[ix]) <= 1e-3 * abs(g[ix]) + 1e-9, (ix, fd, g[ix])


def test_learned_with_nms_weights_tracks_plain_decoder(oracle):
    rate, z, T = 0, 48, 8
    _, cw, llr = inputs.frames(oracle, rate, z, 200, 2.0, seed=11)
    w, rs, cols = random_weights(oracle, rate, z, T, 1)
    w[0][w[0] != 0] = 0.815
    w[1] = 0.0
    _, dl, itl, sfl = oracle.learned_decode(rate, z, T, w, llr)
    _, dp, rp, itp, sfp = oracle.decode(rate, z, llr, T)
    # float vs fp64 normalisation: decisions agree on almost every frame
    assert (sfl == sfp).mean() > 0.97
    assert abs(itl.mean() - itp.mean()) < 0.2
