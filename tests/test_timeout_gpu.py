"""A bounded device wait that runs out. The decode kernel stages each frame
with a bulk copy completed on an mbarrier and polls that barrier a bounded
number of times; on expiry it records a timeout in the handle's error word,
waits (with the full bound) for its copy to land and exits, and the host
reports WLDPC_ERR_TIMEOUT. The test hook wldpc_decoder_set_wait_limit(0)
makes every poll budget run out at once (nothing faults or hangs: the copy
itself completes normally); the next call with the default budget must be
clean and bit-exact."""
import numpy as np
import pytest

import inputs

pytestmark = pytest.mark.gpu


def test_staging_wait_timeout_is_reported_and_the_next_call_is_clean(wl, cuda, oracle):
    rate, z = 0, 96
    _, _, llr = inputs.frames(oracle, rate, z, 64, 2.0, seed=31)
    po, do, ro, io, so = oracle.decode(rate, z, llr, 10)
    dec = wl.Decoder(rate, z, 10)
    d_llr = cuda.from_numpy(llr).cuda()
    hard = cuda.empty(d_llr.shape, dtype=cuda.int8, device="cuda")
    status = cuda.empty(llr.shape[0], dtype=cuda.int32, device="cuda")

    dec.set_wait_limit(0)
    dec.decode_device(d_llr, hard, None, status)
    with pytest.raises(wl.LdpcError) as e:
        dec.synchronize()
    assert e.value.code == wl.ERR_TIMEOUT
    with pytest.raises(wl.LdpcError) as e:      # the synchronous host path reports it too
        dec.decode_host(llr)
    assert e.value.code == wl.ERR_TIMEOUT

    dec.set_wait_limit(wl.WAIT_LIMIT_DEFAULT)
    dec.decode_device(d_llr, hard, None, status)
    dec.synchronize()                           # the error word was cleared: no stale timeout
    cuda.cuda.synchronize()
    assert (hard.cpu().numpy() == do).all()
    assert ((status.cpu().numpy() & 0xFFFF) == io).all()
    post, h2, ne, st = dec.decode_host(llr)
    assert (post.view(np.uint32) == po.view(np.uint32)).all() and (h2 == do).all()


def test_wait_bound_is_under_a_second(wl, cuda):
    """The decoders' waits give up after WLDPC_WAIT_LIMIT_DEFAULT polls; on a
    barrier that never completes those polls must end well within a second
    (the documented bound), and scale with the poll count."""
    small = wl.wait_bound_ns(1 << 16)
    full = wl.wait_bound_ns(wl.WAIT_LIMIT_DEFAULT)
    print(f"wait bound: {small / 1e6:.3f} ms for 2^16 polls, {full / 1e6:.3f} ms for 2^22")
    assert 0 < small < full
    assert full < 1e9
