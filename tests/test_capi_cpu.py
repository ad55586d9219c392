"""C ABI checks that need no GPU: the library loads, exports every symbol
include/wimax_ldpc_b200.h declares and the facade classes, answers the host-
only table queries exactly as the reference, and maps the reference's
exceptions to error codes."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import inputs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "wimax_ldpc_b200.h")).read()
    return sorted(set(re.findall(r"WLDPC_API\s+[\w\s\*]*?\b(wldpc_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol(wl):
    names = declared_symbols()
    assert len(names) >= 20
    L = wl.lib()
    for n in names:
        assert hasattr(L, n), n
    out = subprocess.check_output(["nm", "-DC", "--defined-only", wl.LIB_PATH]).decode()
    for n in names:
        assert re.search(rf" T {n}$", out, re.M), n
    for sym in ["wimax_ldpc_lib::ldpc_decoder::decode(float*, signed char*)",
                "wimax_ldpc_lib::ldpc_decoder::decode(signed char*, signed char*)",
                "wimax_ldpc_lib::ldpc_decoder::compute_syndrome(signed char*, bool)",
                "wimax_ldpc_lib::ldpc_encoder::encode_data(unsigned char*, unsigned char*)",
                "wimax_ldpc_lib::BER_runner::run_iteration(double)",
                "wimax_ldpc_lib::ldpc::get_nanoseconds()"]:
        assert sym in out, sym


def test_library_is_sm100a_only(wl):
    out = subprocess.check_output(["cuobjdump", "--list-elf", wl.LIB_PATH]).decode()
    archs = set(re.findall(r"sm_(\d+a?)", out))
    assert archs == {"100a"}, archs


def test_code_info_and_tables_match_reference(wl, golden_tables):
    for c in golden_tables["cases"]:
        ci = wl.code_info(c["rate"], c["z"])
        assert (ci.n, ci.m, ci.rows, ci.cols, ci.D, ci.X) == (c["N"], c["M"], c["rows"], c["cols"], c["D"], c["X"])
        t = wl.checknode_table(c["rate"], c["z"])
        assert inputs.digest(t.astype("<i2")) == c["digest"]
        assert ci.edges == int((t >= 0).sum())


@pytest.mark.parametrize("rate,z", [(6, 96), (-1, 96), (0, 20), (0, 100), (0, 26), (3, 0)])
def test_invalid_code_is_rejected(wl, rate, z):
    # the reference prints and throws std::exception (reference lib/ldpc.cc:46-57,1198-1202)
    L = wl.lib()
    ci = wl.CodeInfo()
    assert L.wldpc_code_info_get(rate, z, ctypes.byref(ci)) == wl.ERR_CODE
    h = ctypes.c_void_p()
    assert L.wldpc_decoder_create(rate, z, 10, 1, 0, ctypes.byref(h)) == wl.ERR_CODE
    assert L.wldpc_encoder_create(rate, z, 1, ctypes.byref(h)) == wl.ERR_CODE
    assert L.wldpc_ber_runner_create(rate, z, 1, 10, ctypes.byref(h)) == wl.ERR_CODE


def test_argument_checks(wl):
    L = wl.lib()
    assert L.wldpc_code_info_get(0, 96, None) == wl.ERR_ARG
    assert L.wldpc_checknode_table(0, 96, None, 0) == wl.ERR_ARG
    small = np.empty(10, np.int16)
    assert L.wldpc_checknode_table(0, 96, ctypes.c_void_p(small.ctypes.data), small.size) == wl.ERR_ARG
    assert L.wldpc_decoder_destroy(None) == wl.ERR_ARG
    h = ctypes.c_void_p()
    assert L.wldpc_decoder_create(0, 96, 10, 1, 7, ctypes.byref(h)) == wl.ERR_ARG   # unknown mode
    # BER_runner refuses 3/4B like the reference (reference lib/BER_runner.cc:66-71)
    assert L.wldpc_ber_runner_create(4, 96, 1, 10, ctypes.byref(h)) == wl.ERR_UNSUPPORTED
    assert L.wldpc_framegen_device(4, 96, 1, 0, 1, 2.0, 2.0, None, None, None, None, None) == wl.ERR_UNSUPPORTED
    assert wl.lib().wldpc_strerror(wl.ERR_CODE) == b"invalid code rate or z factor"


def test_no_device_fails_loudly(wl):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert wl.lib().wldpc_decoder_create(0, 96, 10, 1, 0, ctypes.byref(h)) == wl.ERR_NO_DEVICE
    with pytest.raises(wl.LdpcError):
        wl.Decoder(0, 96)


def test_argument_checks_of_the_additions(wl):
    """Entry points with no reference counterpart (learned decoder and its
    data-parallel pieces, mixed batch, allocation-free decode) reject bad
    arguments before touching a device."""
    L = wl.lib()
    h = ctypes.c_void_p()
    nw = ctypes.c_size_t()
    # learned decoder: codes (all 114 are supported), iteration count
    assert L.wldpc_lms_create(6, 96, 8, ctypes.byref(h)) == wl.ERR_CODE
    assert L.wldpc_lms_create(0, 97, 8, ctypes.byref(h)) == wl.ERR_CODE
    assert L.wldpc_lms_create(0, 20, 8, ctypes.byref(h)) == wl.ERR_CODE
    assert L.wldpc_lms_create(0, 96, 0, ctypes.byref(h)) == wl.ERR_ARG
    assert L.wldpc_lms_create(0, 96, 9, ctypes.byref(h)) == wl.ERR_ARG
    # z = 36 has kernels now: without a device the call gets as far as the device check
    assert L.wldpc_lms_create(0, 36, 8, ctypes.byref(h)) == wl.ERR_NO_DEVICE
    assert L.wldpc_lms_create(0, 96, 8, None) == wl.ERR_ARG
    assert L.wldpc_lms_destroy(None) == wl.ERR_ARG
    assert L.wldpc_lms_grad_size(None, ctypes.byref(nw)) == wl.ERR_ARG
    assert L.wldpc_lms_step_grad(None, 16, 1.0, 2.0, 1, 0, None, None, None) == wl.ERR_ARG
    assert L.wldpc_lms_apply_grad(None, None, 1e-3, None) == wl.ERR_ARG
    assert L.wldpc_lms_set_precision(None, wl.LMS_F16X2) == wl.ERR_ARG
    # mixed batch: variant numbering rate * 19 + (z - 24) / 4, bad codes, bad caps
    assert L.wldpc_variant(0, 24) == 0 and L.wldpc_variant(0, 96) == 18 and L.wldpc_variant(5, 96) == 113
    assert L.wldpc_variant(6, 96) == wl.ERR_CODE and L.wldpc_variant(0, 26) == wl.ERR_CODE
    assert L.wldpc_mixed_create(0x10000, ctypes.byref(h)) == wl.ERR_ARG
    assert L.wldpc_mixed_create(10, None) == wl.ERR_ARG
    assert L.wldpc_mixed_destroy(None) == wl.ERR_ARG
    assert L.wldpc_mixed_set_config(None, 96, 32) == wl.ERR_ARG
    assert L.wldpc_mixed_set_rows_per_thread(None, 1) == wl.ERR_ARG
    assert L.wldpc_mixed_get_rows_per_thread(None, None) == wl.ERR_ARG
    # allocation-free decode: code, cap and the scratch limit come before any device call
    assert L.wldpc_decode_host_noalloc(0, 100, 10, None, None, None, 1) == wl.ERR_CODE
    assert L.wldpc_decode_host_noalloc(0, 96, 0x10000, None, None, None, 1) == wl.ERR_ARG
    assert L.wldpc_decode_host_noalloc(0, 96, 10, None, None, None, 0) == 0
    buf = np.zeros(2304, np.float32)
    out = np.zeros(2304, np.int8)
    assert L.wldpc_decode_host_noalloc(0, 96, 10, ctypes.c_void_p(buf.ctypes.data), ctypes.c_void_p(out.ctypes.data),
                                       None, 91) == -7   # WLDPC_ERR_SCRATCH: 90 frames of z=96 at most
