"""GPU-backed command-line tools bin/test_encoder and bin/test_decoder: same
arguments, files and printed lines as the reference's tools (reference
lib/encode_example.cc, lib/decode_example.cc). Their files are checked
against the oracle: encoded frames are oracle codewords with at most
errors_to_add flips each, decoded datawords and the printed initial / final
error counts equal the oracle's decode(int8_t*, int8_t*) results."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "wimax_ldpc_lib_b200", "bin")


def _run(args, cwd):
    p = subprocess.run([os.path.join(BIN, args[0])] + [str(a) for a in args[1:]], cwd=cwd,
                       capture_output=True, text=True, timeout=120)
    return p.returncode, p.stdout


def test_cli_usage_without_gpu(wl):
    """Wrong argument counts print the reference's usage line and touch no device."""
    for tool in ("test_encoder", "test_decoder"):
        rc, out = _run([tool, "1"], ROOT)
        assert rc == 0
        assert "Incorrect number of arguments" in out and f"./{tool}" in out


@pytest.mark.gpu
@pytest.mark.parametrize("rate,z,flips", [(0, 96, 0), (0, 24, 12), (1, 48, 5), (3, 72, 3), (5, 96, 2)])
def test_encoder_cli(wl, cuda, oracle, tmp_path, rate, z, flips):
    n = 24 * z
    k = wl.code_info(rate, z).k
    rounds = 37
    rc, out = _run(["test_encoder", rate, z, rounds, flips, "data.bin", "enc.bin"], tmp_path)
    assert rc == 1 and "Average Rate (Mbits/Sec)" in out
    data = np.fromfile(tmp_path / "data.bin", np.uint8).reshape(rounds, k)
    enc = np.fromfile(tmp_path / "enc.bin", np.uint8).reshape(rounds, n)
    assert set(np.unique(data)) <= {0, 1}
    want = oracle.encode(rate, z, data)
    d = (enc != want).sum(axis=1)
    assert (d <= flips).all() and ((flips - d) % 2 == 0).all()
    if flips == 0:
        assert not oracle.syndrome(rate, z, enc.astype(np.int8)).any()


@pytest.mark.gpu
def test_encoder_cli_refuses_34b(wl, cuda, tmp_path):
    rc, out = _run(["test_encoder", 4, 96, 4, 0, "d.bin", "e.bin"], tmp_path)
    assert rc == 1 and "3/4B Not Implemented" in out


@pytest.mark.gpu
@pytest.mark.parametrize("rate,z,threads,frames,flips", [(0, 96, 4, 26, 20), (2, 24, 3, 10, 6), (5, 60, 1, 9, 4),
                                                         (4, 96, 8, 16, 30)])
def test_decoder_cli(wl, cuda, oracle, tmp_path, rate, z, threads, frames, flips):
    n = 24 * z
    k = wl.code_info(rate, z).k
    rng = np.random.default_rng(rate * 1000 + z)
    if rate == 4:   # no encoder: codewords from the device null-space generator
        torch = cuda
        cwd = torch.empty((frames, n), dtype=torch.uint8, device="cuda")
        llr = torch.empty((frames, n), dtype=torch.float32, device="cuda")
        wl.framegen_nullspace_device(rate, z, 11, 0, frames, 3.0, 3.0, codeword=cwd, llr=llr)
        torch.cuda.synchronize()
        cw = cwd.cpu().numpy()
    else:
        cw = oracle.encode(rate, z, rng.integers(0, 2, (frames, k), dtype=np.uint8))
    noisy = cw.copy()
    for f in range(frames):
        idx = rng.choice(n, flips, replace=False)
        noisy[f, idx] ^= 1
    noisy.astype(np.uint8).tofile(tmp_path / "enc.bin")
    rc, out = _run(["test_decoder", threads, rate, z, frames, "enc.bin", "dec.bin"], tmp_path)
    assert rc == 1, out
    used = frames // threads * threads
    dec_ref, ret_ref, _ = oracle.decode_bits(rate, z, noisy[:used].astype(np.int8), max_iter=10)
    got = np.fromfile(tmp_path / "dec.bin", np.int8)
    assert got.size == used * k
    assert np.array_equal(got.reshape(used, k), dec_ref[:, :k])
    init = [int(v) for v in re.findall(r"Initial Number of Errors \(\d+\): (\d+)", out)]
    final = [int(v) for v in re.findall(r"Final Number of Errors \(\d+\): (\d+)", out)]
    assert init == [int(v) for v in oracle.syndrome(rate, z, noisy[:used].astype(np.int8))]
    assert final == [int(v) for v in ret_ref]
    assert "Fastest Iteration (Mbits/Sec)" in out
