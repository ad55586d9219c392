"""The allocation-free decode entry point (wldpc_decode_host_noalloc).

It serves callers that cannot call cudaMalloc (device memory owned by another
allocator, real-time threads, calls that cannot keep a decoder handle). It
must give exactly what the allocating entry point (wldpc_decode_batch_host)
gives, on consecutive calls that reuse its static scratch. This file sorts
last so that a run stopping at the first failure has run every other test."""
import ctypes

import numpy as np
import pytest

import inputs

pytestmark = pytest.mark.gpu


def noalloc(wl, rate, z, max_iter, llr):
    L = wl.lib()
    f = L.wldpc_decode_host_noalloc
    f.argtypes = [ctypes.c_int, ctypes.c_uint, ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_size_t]
    rx = np.ascontiguousarray(llr, np.float32).copy()
    dec = np.empty(rx.shape, np.int8)
    ne = np.empty(rx.shape[0], np.uint32)
    rc = f(rate, z, max_iter, rx.ctypes.data, dec.ctypes.data, ne.ctypes.data, rx.shape[0])
    return rc, rx, dec, ne


@pytest.mark.parametrize("rate,z,frames,ebno", [(0, 96, 90, 2.0), (5, 24, 363, 3.5), (2, 60, 64, 2.5)])
def test_noalloc_matches_allocating_entry_point(wl, cuda, oracle, rate, z, frames, ebno):
    dec = wl.Decoder(rate, z, 10)
    for call in range(2):   # two calls in a row share (and reuse) the static scratch
        _, _, llr = inputs.frames(oracle, rate, z, frames, ebno + 0.25 * call, seed=4242 + 31 * call + z)
        rc, post, hard, ne = noalloc(wl, rate, z, 10, llr)
        assert rc == wl.OK
        post_ref, hard_ref, ne_ref, _ = dec.decode_host(llr)
        # bit-exact, the tolerance of every decoder test
        assert (post.view(np.uint32) == post_ref.view(np.uint32)).all()
        assert (hard == hard_ref).all()
        assert (ne == ne_ref).all()


def test_noalloc_rejects_requests_beyond_its_scratch(wl, cuda):
    llr = np.zeros((91, 2304), np.float32)    # 91 frames of z=96 do not fit in 1 MiB
    rc, _, _, _ = noalloc(wl, 0, 96, 10, llr)
    assert rc == -7
    assert b"scratch" in wl.lib().wldpc_strerror(rc)
    rc, _, _, _ = noalloc(wl, 0, 95, 10, llr[:1, :2280])
    assert rc == wl.ERR_CODE
