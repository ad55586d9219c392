"""Mixed-code persistent decoder (config: all 114 codes in one batch, per-frame
Eb/N0 in [1, 4] dB, 3/4B frames from the null space of H): bit-exact against
the (rate, z)-specialised decoders and the oracle, stable across graph
replays and configurations; and the null-space generator's codewords."""
import numpy as np
import pytest

import inputs

pytestmark = pytest.mark.gpu


def test_nullspace_frames_are_codewords(wl, cuda, oracle):
    torch = cuda
    for rate, z in [(4, 96), (4, 24), (0, 48), (5, 60)]:
        n = 24 * z
        cw = torch.empty((64, n), dtype=torch.uint8, device="cuda")
        llr = torch.empty((64, n), dtype=torch.float32, device="cuda")
        wl.framegen_nullspace_device(rate, z, 5, 0, 64, 3.0, 3.0, codeword=cw, llr=llr)
        torch.cuda.synchronize()
        c = cw.cpu().numpy()
        assert not oracle.syndrome(rate, z, c.astype(np.int8)).any()
        assert 0.4 < c.mean() < 0.6 and len({bytes(r) for r in c}) == 64
        hard = (llr.cpu().numpy() >= 0).astype(np.uint8)
        assert (hard == c).mean() > 0.9


@pytest.fixture(scope="module")
def batch(wl, cuda):
    from wimax_ldpc_lib_b200.mixed_batch import build_batch
    return build_batch(12000, seed=77)


def test_mixed_matches_specialised_decoders(wl, cuda, batch):
    torch = cuda
    from wimax_ldpc_lib_b200.mixed_batch import decode_by_code
    variants, offsets, llr, cw, groups = batch
    assert len(groups) == 114
    frames = variants.numel()
    ref_hard = torch.empty(llr.numel(), dtype=torch.int8, device="cuda")
    ref_status = torch.empty(frames, dtype=torch.int32, device="cuda")
    decode_by_code(groups, llr, ref_hard, ref_status)
    mixed = wl.MixedDecoder(10)
    R, S = wl.MIXED_MSG_REGISTERS, wl.MIXED_MSG_SHARED
    # every CTA size, rows per thread and message layout; chunks from one
    # frame per item to the maximum
    C, Q = wl.MIXED_CONCURRENT, wl.MIXED_SERIAL
    for threads, layout, chunk, launch, rows in [(96, R, 32, C, 1), (96, S, 8, Q, 1), (192, R, 64, Q, 1),
                                                 (192, S, 16, C, 1), (96, R, 1, C, 1), (192, S, 3, Q, 1),
                                                 (96, R, 16, C, 2), (96, S, 64, Q, 2), (192, R, 8, Q, 2),
                                                 (192, S, 5, C, 2)]:
        mixed.set_tuning(threads, layout, chunk, launch)
        mixed.set_rows_per_thread(rows)
        assert mixed.tuning() == (threads, layout, chunk, launch) and mixed.rows_per_thread() == rows
        for _ in range(2):   # capture, then replay
            hard = torch.zeros(llr.numel(), dtype=torch.int8, device="cuda")
            status = torch.full((frames,), -1, dtype=torch.int32, device="cuda")
            post = torch.empty_like(llr)
            mixed.decode_device(variants, offsets, llr, hard, post, status)
            torch.cuda.synchronize()
            mixed.synchronize()
            assert torch.equal(hard, ref_hard), (threads, layout, chunk, rows)
            assert torch.equal(status, ref_status), (threads, layout, chunk, rows)


def test_mixed_matches_oracle_sample(wl, cuda, oracle, batch):
    torch = cuda
    variants, offsets, llr, cw, groups = batch
    mixed = wl.MixedDecoder(10)
    hard = torch.empty(llr.numel(), dtype=torch.int8, device="cuda")
    post = torch.empty_like(llr)
    status = torch.empty(variants.numel(), dtype=torch.int32, device="cuda")
    mixed.decode_device(variants, offsets, llr, hard, post, status)
    torch.cuda.synchronize()
    for (rate, z), (ids, start, c) in list(groups.items())[::9]:
        n = 24 * z
        k = min(c, 6)
        l = llr[start:start + k * n].view(k, n).cpu().numpy()
        po, do, ro, io, so = oracle.decode(rate, z, l, 10)
        assert (post[start:start + k * n].view(k, n).cpu().numpy().view(np.uint32) == po.view(np.uint32)).all()
        assert (hard[start:start + k * n].view(k, n).cpu().numpy() == do).all()
        st = status[torch.from_numpy(ids[:k]).cuda()].cpu().numpy()
        assert ((st & 0xFFFF) == io).all() and (((st >> 16) & 1) == so).all()


def test_mixed_autotune_and_bad_code(wl, cuda, batch):
    torch = cuda
    variants, offsets, llr, cw, groups = batch
    mixed = wl.MixedDecoder(10)
    hard = torch.empty(llr.numel(), dtype=torch.int8, device="cuda")
    ms = mixed.autotune(variants, offsets, llr, hard, repeats=1)
    threads, layout, chunk, launch = mixed.tuning()
    assert ms > 0 and threads in (96, 192) and layout in (0, 1) and chunk in (8, 16, 32, 64) and launch in (0, 1)
    assert mixed.rows_per_thread() in (1, 2)
    bad = variants.clone()
    bad[0] = 200
    mixed.decode_device(bad, offsets, llr, hard)
    torch.cuda.synchronize()
    with pytest.raises(wl.LdpcError):
        mixed.synchronize()
    # a frame that does not start on a 16-byte boundary is refused (and not decoded)
    odd = offsets.clone()
    odd[1] += 1
    mixed.decode_device(variants, odd, llr, hard)
    torch.cuda.synchronize()
    with pytest.raises(wl.LdpcError) as e:
        mixed.synchronize()
    assert e.value.code == wl.ERR_ARG
    mixed.decode_device(variants, offsets, llr, hard)   # and the handle still works
    mixed.synchronize()
    with pytest.raises(wl.LdpcError):
        mixed.set_tuning(96, 0, 65, 0)                     # at most 64 frames per work item
    with pytest.raises(wl.LdpcError):
        mixed.set_rows_per_thread(3)                       # one or two rows per thread
