"""BER_runner drop-in: the same BER sequence as the reference's own
BER_runner (LFSR info bits, mt19937(0) noise, error count over n bits)."""
import pytest

pytestmark = pytest.mark.gpu


def test_ber_runner_matches_reference(wl, cuda, golden_misc):
    for c in golden_misc["ber_runner"]:
        b = wl.BERRunner(c["rate"], c["z"], 1, 10)
        assert b.lengths() == (c["cw_len"], c["dw_len"])
        bers = [b.run_iteration(c["ebno"]) for _ in range(c["iters"])]
        assert bers == c["ber"], (c["rate"], c["z"])
        assert b.totals() == (c["bits"], c["errors"])
        b.reset_test()
        assert b.totals() == (0, 0)
