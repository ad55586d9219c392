"""A bounded device wait that runs out. The decode kernel stages each frame
with a bulk copy completed on an mbarrier and waits for that barrier at most
a bounded device time; on expiry it records a timeout in the handle's error
word, waits (with the full bound) for its copy to land and exits, and the
host reports WLDPC_ERR_TIMEOUT. The test hook wldpc_decoder_set_wait_limit(0)
makes every wait give up at once (nothing faults or hangs: the copy itself
completes normally); the next call with the default bound must be clean and
bit-exact. The bound itself is measured on a barrier that never completes."""
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
    with pytest.raises(wl.LdpcError) as e:      # and the single-frame path (pinned block)
        dec.decode(llr[0])
    assert e.value.code == wl.ERR_TIMEOUT

    dec.set_wait_limit(wl.WAIT_LIMIT_DEFAULT_US)
    p1, d1, ne1, it1 = dec.decode(llr[0])       # single frame after a timeout: clean and exact
    assert (p1.view(np.uint32) == po[0].view(np.uint32)).all() and (d1 == do[0]).all()
    assert it1 == io[0] and ne1 == ro[0]
    dec.decode_device(d_llr, hard, None, status)
    dec.synchronize()                           # the error word was cleared: no stale timeout
    cuda.cuda.synchronize()
    assert (hard.cpu().numpy() == do).all()
    assert ((status.cpu().numpy() & 0xFFFF) == io).all()
    post, h2, ne, st = dec.decode_host(llr)
    assert (post.view(np.uint32) == po.view(np.uint32)).all() and (h2 == do).all()


def test_wait_bound_is_a_time_bound(wl, cuda):
    """The kernels' waits give up after WLDPC_WAIT_LIMIT_DEFAULT_US of device
    time (one second), not after a poll count: a wait on a barrier that never
    completes must end close to its limit, for a short and the default limit."""
    short = wl.wait_bound_ns(20000)
    full = wl.wait_bound_ns(wl.WAIT_LIMIT_DEFAULT_US)
    print(f"wait bound: {short / 1e6:.3f} ms at a 20 ms limit, {full / 1e6:.3f} ms at the default")
    assert 20e6 <= short < 40e6
    assert 1e9 <= full < 1.1e9
