"""The oracle (C restatement in oracle/wldpc_oracle.c) against the reference's
own outputs: golden fixtures recorded from the compiled reference, and, where
the reference sources are present, the compiled reference live."""
import numpy as np
import pytest

import inputs
from cases import case_llr, expected_iters


def test_tables_match_reference(oracle, golden_tables):
    for c in golden_tables["cases"]:
        t = oracle.checknode_table(c["rate"], c["z"])
        info = oracle.code(c["rate"], c["z"])
        assert t.shape == (c["rows"], c["cols"])
        assert inputs.digest(t.astype("<i2")) == c["digest"], (c["rate"], c["z"])
        assert (info.D, info.X, info.n, info.m) == (c["D"], c["X"], c["N"], c["M"])


def test_decoder_matches_reference_golden(oracle, golden_decode):
    for c in golden_decode["cases"]:
        llr = case_llr(oracle, c)
        post, dec, ret, it, sf = oracle.decode(c["rate"], c["z"], llr, c["max_iter"], c["mode"])
        assert inputs.frame_digests(post, dec) == c["digests"], c["name"]
        assert ret.tolist() == c["ret"], c["name"]
        if "iters" in c:
            assert it.tolist() == expected_iters(c), c["name"]
            assert (sf == 1).tolist() == [i > c["max_iter"] for i in c["iters"]], c["name"]


def test_encoder_matches_reference_golden(oracle, golden_encode):
    for c in golden_encode["cases"]:
        n, m, k = inputs.code_dims(c["rate"], c["z"])
        u = inputs.info_bits(c["seed"], c["frames"], k)
        u[0, :4] = [2, 5, 255, 1]
        cw = oracle.encode(c["rate"], c["z"], u)
        assert [inputs.digest(cw[f]) for f in range(c["frames"])] == c["digests"], (c["rate"], c["z"])


def test_encoder_output_is_a_codeword(oracle):
    for rate in (0, 1, 2, 3, 5):
        for z in (24, 52, 96):
            n, m, k = inputs.code_dims(rate, z)
            u = inputs.info_bits(rate * 1000 + z, 8, k)
            cw = oracle.encode(rate, z, u)
            assert not oracle.syndrome(rate, z, cw.astype(np.int8)).any()


def test_bits_adapter_and_syndrome_golden(oracle, golden_misc):
    for c, s in zip(golden_misc["decode_bits"], golden_misc["syndrome"]):
        rate, z, seed = c["rate"], c["z"], c["seed"]
        n, m, k = inputs.code_dims(rate, z)
        u = inputs.info_bits(seed, 16, k)
        bits = oracle.encode(rate, z, u).astype(np.int8)
        flips = inputs.raw(seed + 1, 16 * 8).reshape(16, 8) % np.uint64(n)
        for f in range(16):
            for v in flips[f]:
                bits[f, int(v)] ^= 1
        bits[0, :3] = [3, -1, 2]
        d, ret, _ = oracle.decode_bits(rate, z, bits, 10)
        assert [inputs.digest(d[f]) for f in range(16)] == c["digests"]
        assert ret.tolist() == c["ret"]
        assert oracle.syndrome(rate, z, bits, False).tolist() == s["count"]
        assert oracle.syndrome(rate, z, bits, True).tolist() == s["early"]


def test_lfsr_period_restart(oracle):
    a, st, ix = oracle.lfsr(115200 + 50)
    b, _, _ = oracle.lfsr(50)
    assert (a[115200:] == b).all()        # restarted from the seed after reset_len bits
    assert 0.45 < a.mean() < 0.55


def test_philox_known_answer(oracle):
    # Random123 known-answer vectors for philox4x32-10
    assert oracle.philox([0, 0, 0, 0], [0, 0]).tolist() == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert oracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2).tolist() == [0x408F276D, 0x41C83B0E, 0xA20BC7C6,
                                                                        0x6D5451FD]
    assert oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]).tolist() == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_framegen_statistics(oracle):
    info, cw, llr, eb = oracle.framegen(0, 96, 42, 0, 64, 2.0)
    assert not oracle.syndrome(0, 96, cw.astype(np.int8)).any()
    assert (cw[:, :info.shape[1]] == info).all()
    sigma2 = 1.0 / (2 * 0.5 * 10 ** 0.2)
    y = llr * sigma2 / 2.0 - (cw * 2.0 - 1.0)
    assert abs(y.mean()) < 0.01 and abs(y.var() / sigma2 - 1.0) < 0.02


@pytest.mark.skipif(not __import__("oracle.oracle", fromlist=["x"]).reference_available(),
                    reason="reference not compiled here (oracle/_ref)")
def test_oracle_matches_live_reference(oracle):
    from oracle.oracle import Reference
    ref = Reference()
    for (rate, z, eb) in [(0, 96, 1.5), (5, 96, 4.0), (3, 40, 3.0)]:
        _, _, llr = inputs.frames(oracle, rate, z, 200, eb, seed=77 + z)
        po, do, ro, _, _ = oracle.decode(rate, z, llr, 10)
        pr, dr, rr = ref.decode(rate, z, llr, 10)
        assert (po.view(np.uint32) == pr.view(np.uint32)).all() and (do == dr).all() and (ro == rr).all()
