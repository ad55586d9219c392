"""The C++ facade (include/wimax_ldpc_lib/) used as reference code uses the
reference classes: compiled with g++ against the headers, linked to the
library, outputs compared with the oracle / the reference's golden values."""
import os
import subprocess

import numpy as np
import pytest

import inputs

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def facade_bin(wl, tmp_path_factory):
    out = str(tmp_path_factory.mktemp("facade") / "facade_check")
    libdir = os.path.dirname(wl.LIB_PATH)
    subprocess.check_call(["g++", "-std=c++11", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "facade_check.cc"), "-o", out, "-L", libdir,
                           "-lwimax_ldpc_b200", f"-Wl,-rpath,{libdir}"])
    return out


def test_facade_decode_matches_oracle(facade_bin, oracle, tmp_path):
    for rate, z in [(0, 24), (5, 96), (2, 56)]:
        frames = 40
        _, _, llr = inputs.frames(oracle, rate, z, frames, inputs.SWEEP_EBNO[rate], seed=123 + z)
        src, dst = tmp_path / "llr.f32", tmp_path / "out.bin"
        llr.tofile(src)
        subprocess.check_call([facade_bin, "decode", str(rate), str(z), str(frames), "10", str(src), str(dst)])
        n = 24 * z
        rec = np.fromfile(dst, dtype=np.uint8).reshape(frames, 4 * n + n + 4)
        post = rec[:, :4 * n].copy().view(np.float32)
        dec = rec[:, 4 * n:5 * n].copy().view(np.int8)
        ret = rec[:, 5 * n:].copy().view(np.uint32)[:, 0]
        po, do, ro, _, _ = oracle.decode(rate, z, llr, 10)
        assert (post.view(np.uint32) == po.view(np.uint32)).all()
        assert (dec == do).all() and (ret == ro).all()


def test_facade_encode_matches_oracle(facade_bin, oracle, tmp_path):
    rate, z, frames = 3, 84, 16
    n, m, k = inputs.code_dims(rate, z)
    u = inputs.info_bits(5, frames, k)
    u.tofile(tmp_path / "info.u8")
    subprocess.check_call([facade_bin, "encode", str(rate), str(z), str(frames), str(tmp_path / "info.u8"),
                           str(tmp_path / "cw.u8")])
    cw = np.fromfile(tmp_path / "cw.u8", dtype=np.uint8).reshape(frames, n)
    assert (cw == oracle.encode(rate, z, u)).all()


def test_facade_ber_runner_matches_reference(facade_bin, golden_misc):
    c = golden_misc["ber_runner"][0]
    out = subprocess.check_output([facade_bin, "ber", str(c["rate"]), str(c["z"]), str(c["iters"]),
                                   repr(c["ebno"])]).decode().split()
    assert int(out[0]) == c["bits"] and int(out[1]) == c["errors"]
    assert float(out[2]) == c["ber"][-1]
    assert (int(out[3]), int(out[4])) == (c["cw_len"], c["dw_len"])


def test_facade_throws_like_reference(facade_bin):
    assert subprocess.run([facade_bin, "invalid"], capture_output=True).returncode == 0
