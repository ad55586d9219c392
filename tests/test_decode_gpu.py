"""GPU TDMP decoder parity through the C ABI: bit-exact posteriors, hard
decisions, return values and iteration counts against the reference's golden
outputs and the oracle, for every (rate, z), the three min-sum flavours and
the edge cases."""
import numpy as np
import pytest

import inputs
from cases import case_llr, expected_iters
from test_learned_oracle import random_weights

pytestmark = pytest.mark.gpu


def run_device(wl, torch, dec, llr_np, posterior=True):
    llr = torch.from_numpy(llr_np).cuda()
    hard = torch.empty(llr.shape, dtype=torch.int8, device="cuda")
    post = torch.empty_like(llr) if posterior else None
    status = torch.empty(llr.shape[0], dtype=torch.int32, device="cuda")
    dec.decode_device(llr, hard, post, status)
    torch.cuda.synchronize()
    dec.synchronize()
    return (post.cpu().numpy() if posterior else None), hard.cpu().numpy(), status.cpu().numpy()


def check_case(wl, c, post, hard, status):
    assert inputs.frame_digests(post, hard) == c["digests"], c["name"]
    assert wl.reference_return(status, c["max_iter"]).tolist() == c["ret"], c["name"]
    if "iters" in c:
        assert (status & 0xFFFF).tolist() == expected_iters(c), c["name"]
        assert ((status >> 16) & 1).tolist() == [int(i > c["max_iter"]) for i in c["iters"]], c["name"]


def test_golden_cases_device_batch(wl, cuda, oracle, golden_decode):
    decs = {}
    for c in golden_decode["cases"]:
        key = (c["rate"], c["z"], c["max_iter"], c["mode"])
        if key not in decs:
            decs[key] = wl.Decoder(c["rate"], c["z"], c["max_iter"], c["mode"])
        llr = case_llr(oracle, c)
        post, hard, status = run_device(wl, cuda, decs[key], llr)
        check_case(wl, c, post, hard, status)


def test_golden_cases_host_batch_in_place(wl, cuda, oracle, golden_decode):
    for c in golden_decode["cases"][:40]:
        dec = wl.Decoder(c["rate"], c["z"], c["max_iter"], c["mode"])
        llr = case_llr(oracle, c)
        post, hard, ne, status = dec.decode_host(llr)
        check_case(wl, c, post, hard, status)
        assert ne.tolist() == c["ret"]


def test_single_frame_reference_api(wl, cuda, oracle, golden_decode):
    c = golden_decode["cases"][0]
    dec = wl.Decoder(c["rate"], c["z"], c["max_iter"])
    llr = case_llr(oracle, c)
    for f in range(0, c["frames"], 97):
        post, hard, ne, it = dec.decode(llr[f])
        assert inputs.digest(post, hard) == c["digests"][f]
        assert ne == c["ret"][f]
        assert it == expected_iters(c)[f]


def test_in_place_posterior(wl, cuda, oracle):
    _, _, llr_np = inputs.frames(oracle, 5, 96, 256, 3.5, seed=31)
    po, do, ro, io, so = oracle.decode(5, 96, llr_np, 10)
    dec = wl.Decoder(5, 96, 10)
    llr = cuda.from_numpy(llr_np).cuda()
    hard = cuda.empty(llr.shape, dtype=cuda.int8, device="cuda")
    dec.decode_device(llr, hard, llr, None)      # posterior written over the input
    cuda.cuda.synchronize()
    assert (llr.cpu().numpy().view(np.uint32) == po.view(np.uint32)).all()
    assert (hard.cpu().numpy() == do).all()


@pytest.mark.parametrize("rate", range(6))
def test_all_z_against_oracle(wl, cuda, oracle, rate):
    for z in wl.Z_VALUES:
        _, _, llr = inputs.frames(oracle, rate, z, 48, inputs.SWEEP_EBNO[rate] - 0.25, seed=400 + rate * 100 + z)
        po, do, ro, io, so = oracle.decode(rate, z, llr, 10)
        post, hard, status = run_device(wl, cuda, wl.Decoder(rate, z, 10), llr)
        assert (post.view(np.uint32) == po.view(np.uint32)).all(), (rate, z)
        assert (hard == do).all(), (rate, z)
        assert ((status & 0xFFFF) == io).all() and (((status >> 16) & 1) == so).all(), (rate, z)


@pytest.mark.parametrize("rate", range(6))
def test_multi_frame_ctas_with_a_partial_last_cta(wl, cuda, oracle, rate):
    """z not a multiple of 32 puts several frames in one CTA (their stopping
    votes are per frame); 37 frames leave the last CTA partly empty, and every
    third frame is a clean codeword (0 iterations) next to noisy ones that stop
    at different iterations or run to the cap."""
    for z in (24, 28, 36, 44, 52, 68, 76, 84, 92):
        _, cw, llr = inputs.frames(oracle, rate, z, 37, inputs.SWEEP_EBNO[rate] - 0.5, seed=8100 + rate * 100 + z)
        llr[::3] = np.where(cw[::3] != 0, 4.0, -4.0).astype(np.float32)
        po, do, ro, io, so = oracle.decode(rate, z, llr, 10)
        assert (io[::3] == 0).all() and (io > 0).any()
        post, hard, status = run_device(wl, cuda, wl.Decoder(rate, z, 10), llr)
        assert (post.view(np.uint32) == po.view(np.uint32)).all(), (rate, z)
        assert (hard == do).all(), (rate, z)
        assert ((status & 0xFFFF) == io).all() and (((status >> 16) & 1) == so).all(), (rate, z)
        # the learned decoders' stopping votes on the same frames, against the oracle's restatements
        w, _, _ = random_weights(oracle, rate, z, 8, 8200 + rate * 100 + z)
        w[1] = np.abs(w[1])                      # in the binary16 decoder's range (b >= 0)
        for prec, ref in ((wl.LMS_F32, oracle.learned_decode), (wl.LMS_F16X2, oracle.learned16_decode)):
            po, do, io, so = ref(rate, z, 8, w, llr, cap=10)
            post, hard, _, st = wl.LearnedDecoder(rate, z, 8, weights=w, cap=10, precision=prec).decode_host(llr)
            assert (post.view(np.uint32) == po.view(np.uint32)).all(), (prec, rate, z)
            assert (hard == do).all() and ((st & 0xFFFF) == io).all() and (((st >> 16) & 1) == so).all(), (prec, rate, z)


@pytest.mark.parametrize("mode", [1, 2])
def test_oms_ms_all_rates_against_oracle(wl, cuda, oracle, mode):
    for rate in range(6):
        for z in (24, 36, 68, 96):
            _, _, llr = inputs.frames(oracle, rate, z, 32, inputs.SWEEP_EBNO[rate], seed=900 + rate * 100 + z)
            po, do, ro, io, so = oracle.decode(rate, z, llr, 10, mode)
            post, hard, status = run_device(wl, cuda, wl.Decoder(rate, z, 10, mode), llr)
            assert (post.view(np.uint32) == po.view(np.uint32)).all(), (mode, rate, z)
            assert (hard == do).all() and ((status & 0xFFFF) == io).all(), (mode, rate, z)


def test_bits_adapter_and_syndrome(wl, cuda, oracle, golden_misc):
    for c, s in zip(golden_misc["decode_bits"], golden_misc["syndrome"]):
        rate, z, seed = c["rate"], c["z"], c["seed"]
        n, m, k = inputs.code_dims(rate, z)
        bits = oracle.encode(rate, z, inputs.info_bits(seed, 16, k)).astype(np.int8)
        flips = inputs.raw(seed + 1, 16 * 8).reshape(16, 8) % np.uint64(n)
        for f in range(16):
            for v in flips[f]:
                bits[f, int(v)] ^= 1
        bits[0, :3] = [3, -1, 2]
        dec = wl.Decoder(rate, z, 10)
        for f in range(16):
            d, ne = dec.decode_bits(bits[f])
            assert inputs.digest(d) == c["digests"][f] and ne == c["ret"][f]
            assert dec.compute_syndrome(bits[f], False) == s["count"][f]
            assert dec.compute_syndrome(bits[f], True) == s["early"][f]


def test_decode_bits_batch_with_any_byte_values(wl, cuda, oracle):
    """decode(int8_t*) over a batch: bytes b become LLRs 2b - 1 (reference
    lib/ldpc_decoder.cc:108-118) for every int8 value, not only 0 and 1."""
    rate, z, frames = 0, 48, 37
    n, m, k = inputs.code_dims(rate, z)
    bits = oracle.encode(rate, z, inputs.info_bits(6300, frames, k)).astype(np.int8)
    r = inputs.raw(6301, frames * n).reshape(frames, n)
    bits[(r % np.uint64(97)) == 0] ^= 1
    odd = (r >> np.uint64(16)) % np.uint64(211) == 0
    bits[odd] = ((r[odd] >> np.uint64(32)) % np.uint64(256)).astype(np.uint8).view(np.int8)
    bits[0, :4] = [-128, 127, -1, 0]
    d_ref, ret_ref, _ = oracle.decode_bits(rate, z, bits, 10)
    d, ne = wl.Decoder(rate, z, 10).decode_bits_host(bits)
    assert (d == d_ref).all() and (ne == ret_ref).all()


@pytest.mark.parametrize("rate,z", [(0, 96), (4, 28), (5, 60), (1, 24), (3, 92), (2, 44)])
def test_syndrome_batch_against_oracle(wl, cuda, oracle, rate, z):
    """Batch compute_syndrome: 45 frames (a partial warp of the specialised
    kernel) of codewords with 0 to a few hundred flipped bits; a third of the
    frames carry bytes other than 0 and 1 (the reference XORs whole bytes, so
    the kernel checks bit planes 1..7 of those frames too)."""
    n, m, k = inputs.code_dims(rate, z)
    frames = 45
    cw = oracle.encode(rate, z, inputs.info_bits(6100 + z, frames, k)) if rate != 4 else np.zeros((frames, n), np.uint8)
    bits = cw.astype(np.int8)
    r = inputs.raw(6200 + rate * 100 + z, frames * n).reshape(frames, n)
    for f in range(frames):
        flips = (r[f] % np.uint64(max(1, 40 * f))) == 0 if f else np.zeros(n, bool)
        bits[f, flips] ^= 1
        if f % 3 == 1:
            odd = (r[f] >> np.uint64(20)) % np.uint64(9) == 0
            bits[f, odd] = ((r[f, odd] >> np.uint64(32)) % np.uint64(256)).astype(np.uint8).view(np.int8)
    dec = wl.Decoder(rate, z, 10)
    for early in (False, True):
        want = oracle.syndrome(rate, z, bits, early)
        assert (dec.syndrome_host(bits, early) == want).all(), (rate, z, early)
    assert (want == 0).any() and (want == 1).any()


def test_max_iter_zero_quirk(wl, cuda, oracle):
    llr = inputs.edge_llr("noise", 0, 48, 8, 5)
    dec = wl.Decoder(0, 48, 0)
    post, hard, ne, st = dec.decode_host(llr)
    assert (ne == 0).all()                       # the reference returns 0 with max_iter == 0
    assert ((st >> 16) & 1).all() and ((st & 0xFFFF) == 0).all()
    assert (post.view(np.uint32) == llr.view(np.uint32)).all()


def test_misaligned_pointers_rejected(wl, cuda):
    dec = wl.Decoder(0, 24, 10)
    buf = cuda.zeros(2 * 576 + 1, device="cuda")
    hard = cuda.empty(2 * 576, dtype=cuda.int8, device="cuda")
    L = wl.lib()
    import ctypes
    rc = L.wldpc_decode_batch_device(dec._h, ctypes.c_void_p(buf.data_ptr() + 4), ctypes.c_void_p(hard.data_ptr()),
                                     None, None, 2, None)
    assert rc == wl.ERR_ARG


def test_full_size_batch_properties(wl, cuda, oracle):
    """262144 frames of rate 5/6, z=96 (the throughput workload): a sample is
    compared bit for bit with the oracle; every frame reported valid satisfies
    all parity checks; two runs give identical outputs (checksum of checksums)."""
    torch = cuda
    rate, z, frames = 5, 96, 262144
    n = 24 * z
    llr = torch.empty((frames, n), dtype=torch.float32, device="cuda")
    info = torch.empty((frames, 20 * z), dtype=torch.uint8, device="cuda")
    wl.framegen_device(rate, z, 1234, 0, frames, 4.0, 4.0, info=info, llr=llr)
    dec = wl.Decoder(rate, z, 10)
    hard = torch.empty((frames, n), dtype=torch.int8, device="cuda")
    post = torch.empty_like(llr)
    status = torch.empty(frames, dtype=torch.int32, device="cuda")
    dec.decode_device(llr, hard, post, status)
    torch.cuda.synchronize()
    sample = np.random.default_rng(0).choice(frames, 1024, replace=False)
    sample.sort()
    llr_s = llr[torch.from_numpy(sample).cuda()].cpu().numpy()
    po, do, ro, io, so = oracle.decode(rate, z, llr_s, 10)
    idx = torch.from_numpy(sample).cuda()
    assert (post[idx].cpu().numpy().view(np.uint32) == po.view(np.uint32)).all()
    assert (hard[idx].cpu().numpy() == do).all()
    st = status.cpu().numpy()
    assert ((st[sample] & 0xFFFF) == io).all()
    valid = ((st >> 16) & 1) == 0
    h = hard.cpu().numpy()
    syn = oracle.syndrome(rate, z, h[valid][:20000], True)
    assert not syn.any()
    # info bits recovered on valid frames
    ok = (h[valid][:, :20 * z] == info.cpu().numpy()[valid]).all(axis=1)
    assert ok.mean() > 0.999
    d1 = torch.sum(post.view(torch.int32).to(torch.int64) * 1000003 % 998244353).item()
    hard2 = torch.empty_like(hard)
    post2 = torch.empty_like(post)
    dec.decode_device(llr, hard2, post2, None)
    torch.cuda.synchronize()
    assert torch.equal(post, post2) and torch.equal(hard, hard2)
    assert d1 == torch.sum(post2.view(torch.int32).to(torch.int64) * 1000003 % 998244353).item()
