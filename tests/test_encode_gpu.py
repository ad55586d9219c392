"""GPU encoder and frame generator parity through the C ABI."""
import numpy as np
import pytest

import inputs

pytestmark = pytest.mark.gpu


def test_encoder_golden_device_batch(wl, cuda, golden_encode):
    torch = cuda
    for c in golden_encode["cases"]:
        n, m, k = inputs.code_dims(c["rate"], c["z"])
        u = inputs.info_bits(c["seed"], c["frames"], k)
        u[0, :4] = [2, 5, 255, 1]
        enc = wl.Encoder(c["rate"], c["z"])
        ud = torch.from_numpy(u).cuda()
        cw = torch.empty((c["frames"], n), dtype=torch.uint8, device="cuda")
        enc.encode_device(ud, cw)
        torch.cuda.synchronize()
        cw = cw.cpu().numpy()
        assert [inputs.digest(cw[f]) for f in range(c["frames"])] == c["digests"], (c["rate"], c["z"])
        assert inputs.digest(enc.encode(u[1])) == c["digests"][1]
        assert inputs.digest(enc.encode(u[0])) == c["digests"][0]   # non-0/1 bytes through the single-frame path


def test_encoder_large_batch_against_oracle(wl, cuda, oracle):
    torch = cuda
    for rate, z in [(0, 96), (5, 96), (2, 28), (3, 44)]:
        n, m, k = inputs.code_dims(rate, z)
        u = inputs.info_bits(rate + z, 4096, k)
        cw = torch.empty((4096, n), dtype=torch.uint8, device="cuda")
        wl.Encoder(rate, z).encode_device(torch.from_numpy(u).cuda(), cw)
        torch.cuda.synchronize()
        assert (cw.cpu().numpy() == oracle.encode(rate, z, u)).all()


@pytest.mark.parametrize("rate,z", [(0, 24), (1, 60), (3, 28), (3, 44), (5, 92), (2, 96)])
def test_encoder_partial_warps_odd_bytes_and_unaligned_buffers(wl, cuda, oracle, rate, z):
    """The (rate, z)-specialised encoder takes 32 frames per warp: 45 frames
    leave a partial warp; bytes other than 0/1 must count as 1 and pass
    through to the systematic part; rate 3/4 at z = 28, 44 moves 8-byte
    chunks; buffers that are only 4-byte aligned take the generic kernel."""
    torch = cuda
    n, m, k = inputs.code_dims(rate, z)
    frames = 45
    u = inputs.info_bits(7000 + rate * 100 + z, frames, k)
    r = inputs.raw(7001 + rate * 100 + z, frames * k).reshape(frames, k)
    u = np.where(r % np.uint64(7) == 0, (r >> np.uint64(8)) % np.uint64(256), u).astype(np.uint8)
    want = oracle.encode(rate, z, u)
    enc = wl.Encoder(rate, z)
    cw = torch.empty((frames, n), dtype=torch.uint8, device="cuda")
    enc.encode_device(torch.from_numpy(u).cuda(), cw)
    torch.cuda.synchronize()
    assert (cw.cpu().numpy() == want).all()
    ub = torch.zeros(frames * k + 16, dtype=torch.uint8, device="cuda")
    cb = torch.zeros(frames * n + 16, dtype=torch.uint8, device="cuda")
    ub[4:4 + frames * k] = torch.from_numpy(u.reshape(-1)).cuda()
    enc.encode_device(ub[4:4 + frames * k].view(frames, k), cb[4:4 + frames * n].view(frames, n))
    torch.cuda.synchronize()
    assert (cb[4:4 + frames * n].view(frames, n).cpu().numpy() == want).all()


@pytest.mark.parametrize("rate", [0, 1, 2, 3, 5])
def test_framegen_matches_oracle(wl, cuda, oracle, rate):
    torch = cuda
    for z in (24, 60, 96):
        n, m, k = inputs.code_dims(rate, z)
        frames = 64
        info = torch.empty((frames, k), dtype=torch.uint8, device="cuda")
        cw = torch.empty((frames, n), dtype=torch.uint8, device="cuda")
        llr = torch.empty((frames, n), dtype=torch.float32, device="cuda")
        eb = torch.empty(frames, dtype=torch.float32, device="cuda")
        wl.framegen_device(rate, z, 99, 1000, frames, 1.0, 4.0, info, cw, llr, eb)
        torch.cuda.synchronize()
        oi, oc, ol, oe = oracle.framegen(rate, z, 99, 1000, frames, 1.0, 4.0)
        assert (info.cpu().numpy() == oi).all() and (cw.cpu().numpy() == oc).all()
        assert np.array_equal(eb.cpu().numpy(), oe.astype(np.float32))
        # float transcendental functions on the GPU vs double on the host
        l = llr.cpu().numpy().astype(np.float64)
        tol = 2e-5 * np.maximum(1.0, np.abs(ol)) + 1e-4
        assert (np.abs(l - ol) <= tol).all()


def test_lfsr_stream_matches_reference_generator(wl, cuda, oracle):
    torch = cuda
    ref, _, _ = oracle.lfsr(3 * 115200 + 777)
    for first in (0, 1152 * 7, 115200 - 100, 2 * 115200 + 5):
        out = torch.empty(5000, dtype=torch.uint8, device="cuda")
        wl.lfsr_bits_device(first, out)
        torch.cuda.synchronize()
        assert (out.cpu().numpy() == ref[first:first + 5000]).all(), first
        buf = torch.zeros(5008, dtype=torch.uint8, device="cuda")   # output not 16-byte aligned
        wl.lfsr_bits_device(first, buf[3:3 + 4999])
        torch.cuda.synchronize()
        assert (buf[3:3 + 4999].cpu().numpy() == ref[first:first + 4999]).all(), first
        assert not buf[:3].cpu().numpy().any() and not buf[3 + 4999:].cpu().numpy().any()
