"""ctypes access to the test oracles.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py``, always as the checker (or, for the
baseline, as the thing timed on the host cores). The product package never
imports this module.

* ``Oracle`` wraps ``oracle/liboracle.so``, the C restatement
  (``wldpc_oracle.c``) of the reference's codec path.
* ``Reference`` wraps ``oracle/_ref/libwldpc_ref*.so``: the reference's own
  sources (reference lib/ldpc.cc, lib/ldpc_decoder.cc, lib/ldpc_encoder.cc,
  lib/BER_runner.cc, lib/matrices/) compiled unmodified by ``oracle/Makefile``
  behind a small C harness (``ref_harness.cc``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
REFERENCE_SRC = "/root/reference"

NMS, OMS, MS = 0, 1, 2
_REF_LIB = {NMS: "libwldpc_ref.so", OMS: "libwldpc_ref_oms.so", MS: "libwldpc_ref_ms.so"}

_p = ctypes.c_void_p
_i = ctypes.c_int
_l = ctypes.c_long


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def build(reference: bool = False) -> None:
    """Compile the restatement (and, with ``reference``, the reference oracle)."""
    subprocess.check_call(["make", "-s", "-C", HERE], stdout=subprocess.DEVNULL)
    if reference:
        subprocess.check_call(["make", "-s", "-C", HERE, "-j8", "ref", f"REF={REFERENCE_SRC}"],
                              stdout=subprocess.DEVNULL)


def reference_available(mode: int = NMS) -> bool:
    return os.path.exists(os.path.join(REF_DIR, _REF_LIB[mode]))


class CodeInfo:
    def __init__(self, rate, z, n, m, k, D, X, mb, nblk, max_deg):
        self.rate, self.z, self.n, self.m, self.k = rate, z, n, m, k
        self.D, self.X, self.mb, self.nblk, self.max_deg = D, X, mb, nblk, max_deg

    @property
    def edges(self):
        return self.nblk * self.z


class _WoCode(ctypes.Structure):
    _fields_ = [("rate", _i), ("z", _i), ("mb", _i), ("kb", _i), ("n", _i), ("m", _i),
                ("k", _i), ("D", _i), ("X", _i), ("nblk", _i), ("row_start", _i * 13),
                ("blk_col", _i * 96), ("blk_shift", _i * 96), ("max_deg", _i)]


class Oracle:
    """The C restatement (``wldpc_oracle.c``)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.wo_code.argtypes = [_i, _i, ctypes.POINTER(_WoCode)]
        L.wo_checknode_table.argtypes = [_i, _i, _p, _l, ctypes.POINTER(_i), ctypes.POINTER(_i)]
        L.wo_decode_batch.argtypes = [_i, _i, _i, _i, _l, _p, _p, _p, _p, _p, _i]
        L.wo_decode_bits_batch.argtypes = [_i, _i, _i, _l, _p, _p, _p, _p, _i]
        L.wo_syndrome_batch.argtypes = [_i, _i, _l, _p, _i, _p]
        L.wo_encode_batch.argtypes = [_i, _i, _l, _p, _p, _i]
        L.wo_lfsr_fill.argtypes = [_p, _p, ctypes.c_uint32, ctypes.c_uint32, _p, _l]
        L.wo_philox4x32_10.argtypes = [_p, _p, _p]
        L.wo_framegen.argtypes = [_i, _i, ctypes.c_uint64, ctypes.c_uint64, _l, ctypes.c_double,
                                  ctypes.c_double, _p, _p, _p, _p]
        L.wo_learned_decode_batch.argtypes = [_i, _i, _i, _i, _p, _l, _p, _p, _p, _p, _i]
        L.wo_learned16_decode_batch.argtypes = [_i, _i, _i, _i, _p, _l, _p, _p, _p, _p, _p, _i]
        L.wo_half_round.argtypes = [ctypes.c_double]
        L.wo_half_round.restype = ctypes.c_double
        L.wo_half_fma_relu.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.wo_half_fma_relu.restype = ctypes.c_double
        L.wo_learned_loss_grad.argtypes = [_i, _i, _i, _p, _l, _p, _p, _p]
        L.wo_learned_loss_grad.restype = ctypes.c_double
        self.threads = os.cpu_count() or 1

    def code(self, rate: int, z: int) -> CodeInfo:
        c = _WoCode()
        if self.lib.wo_code(rate, z, ctypes.byref(c)) != 0:
            raise ValueError(f"invalid rate/z {rate}/{z}")
        return CodeInfo(rate, z, c.n, c.m, c.k, c.D, c.X, c.mb, c.nblk, c.max_deg)

    def code_blocks(self, rate: int, z: int):
        """(row_start[mb+1], col[nblk], shift[nblk]) of the expanded code."""
        c = _WoCode()
        if self.lib.wo_code(rate, z, ctypes.byref(c)) != 0:
            raise ValueError(f"invalid rate/z {rate}/{z}")
        return (list(c.row_start)[:c.mb + 1], list(c.blk_col)[:c.nblk], list(c.blk_shift)[:c.nblk])

    def checknode_table(self, rate, z):
        buf = np.empty(96 * 12 * 24, np.int16)
        r, c = _i(), _i()
        if self.lib.wo_checknode_table(rate, z, _ptr(buf), buf.size, ctypes.byref(r), ctypes.byref(c)):
            raise ValueError("invalid code")
        return buf[: r.value * c.value].reshape(r.value, c.value).copy()

    def decode(self, rate, z, llr, max_iter=10, mode=NMS, threads=None):
        """Returns (posterior, decoded, ret, iters, synfail); llr is not modified."""
        llr = np.ascontiguousarray(llr, np.float32)
        frames = llr.shape[0]
        post = llr.copy()
        dec = np.empty(llr.shape, np.int8)
        ret = np.empty(frames, np.uint32)
        it = np.empty(frames, np.int32)
        sf = np.empty(frames, np.int32)
        rc = self.lib.wo_decode_batch(rate, z, max_iter, mode, frames, _ptr(post), _ptr(dec),
                                      _ptr(ret), _ptr(it), _ptr(sf), threads or self.threads)
        if rc:
            raise ValueError("wo_decode_batch failed")
        return post, dec, ret, it, sf

    def decode_bits(self, rate, z, bits, max_iter=10, threads=None):
        bits = np.ascontiguousarray(bits, np.int8)
        frames = bits.shape[0]
        dec = np.empty(bits.shape, np.int8)
        ret = np.empty(frames, np.uint32)
        it = np.empty(frames, np.int32)
        if self.lib.wo_decode_bits_batch(rate, z, max_iter, frames, _ptr(bits), _ptr(dec),
                                         _ptr(ret), _ptr(it), threads or self.threads):
            raise ValueError("wo_decode_bits_batch failed")
        return dec, ret, it

    def syndrome(self, rate, z, bits, early_exit=False):
        bits = np.ascontiguousarray(bits, np.int8)
        ret = np.empty(bits.shape[0], np.uint32)
        if self.lib.wo_syndrome_batch(rate, z, bits.shape[0], _ptr(bits), int(early_exit), _ptr(ret)):
            raise ValueError("wo_syndrome_batch failed")
        return ret

    def encode(self, rate, z, info, threads=None):
        info = np.ascontiguousarray(info, np.uint8)
        c = self.code(rate, z)
        cw = np.empty((info.shape[0], c.n), np.uint8)
        if self.lib.wo_encode_batch(rate, z, info.shape[0], _ptr(info), _ptr(cw), threads or self.threads):
            raise ValueError("wo_encode_batch failed")
        return cw

    def lfsr(self, nbits, state=0xDEADBEEF, index=0, start=0xDEADBEEF, reset_len=115200):
        st = np.array([state], np.uint32)
        ix = np.array([index], np.uint32)
        out = np.empty(nbits, np.uint8)
        self.lib.wo_lfsr_fill(_ptr(st), _ptr(ix), start, reset_len, _ptr(out), nbits)
        return out, int(st[0]), int(ix[0])

    def philox(self, ctr, key):
        c = np.asarray(ctr, np.uint32)
        k = np.asarray(key, np.uint32)
        o = np.empty(4, np.uint32)
        self.lib.wo_philox4x32_10(_ptr(c), _ptr(k), _ptr(o))
        return o

    def framegen(self, rate, z, seed, first_frame, frames, ebno_lo, ebno_hi=None):
        c = self.code(rate, z)
        ebno_hi = ebno_lo if ebno_hi is None else ebno_hi
        info = np.empty((frames, c.k), np.uint8)
        cw = np.empty((frames, c.n), np.uint8)
        llr = np.empty((frames, c.n), np.float64)
        eb = np.empty(frames, np.float64)
        if self.lib.wo_framegen(rate, z, seed, first_frame, frames, ebno_lo, ebno_hi,
                                _ptr(info), _ptr(cw), _ptr(llr), _ptr(eb)):
            raise ValueError("wo_framegen failed")
        return info, cw, llr, eb

    def learned_decode(self, rate, z, iterations, w, llr, threads=None, cap=None):
        llr = np.ascontiguousarray(llr, np.float32)
        w = np.ascontiguousarray(w, np.float32)
        post = llr.copy()
        dec = np.empty(llr.shape, np.int8)
        it = np.empty(llr.shape[0], np.int32)
        sf = np.empty(llr.shape[0], np.int32)
        if self.lib.wo_learned_decode_batch(rate, z, iterations, iterations if cap is None else cap, _ptr(w),
                                            llr.shape[0], _ptr(post),
                                            _ptr(dec), _ptr(it), _ptr(sf), threads or self.threads):
            raise ValueError("wo_learned_decode_batch failed")
        return post, dec, it, sf

    def learned16_decode(self, rate, z, iterations, w, llr, threads=None, cap=None):
        """The packed-half learned decoder restated per frame: (posterior, decoded,
        iterations, synfail); llr is not modified."""
        llr = np.ascontiguousarray(llr, np.float32)
        w = np.ascontiguousarray(w, np.float32)
        post = np.empty_like(llr)
        dec = np.empty(llr.shape, np.int8)
        it = np.empty(llr.shape[0], np.int32)
        sf = np.empty(llr.shape[0], np.int32)
        if self.lib.wo_learned16_decode_batch(rate, z, iterations, iterations if cap is None else cap, _ptr(w),
                                              llr.shape[0], _ptr(llr), _ptr(post), _ptr(dec), _ptr(it), _ptr(sf),
                                              threads or self.threads):
            raise ValueError("wo_learned16_decode_batch failed")
        return post, dec, it, sf

    def half_round(self, x: float) -> float:
        return self.lib.wo_half_round(float(x))

    def half_fma_relu(self, a: float, b: float, c: float) -> float:
        return self.lib.wo_half_fma_relu(float(a), float(b), float(c))

    def learned_loss_grad(self, rate, z, iterations, w, llr, cw):
        llr = np.ascontiguousarray(llr, np.float32)
        cw = np.ascontiguousarray(cw, np.uint8)
        w = np.ascontiguousarray(w, np.float32)
        g = np.empty(w.size, np.float64)
        loss = self.lib.wo_learned_loss_grad(rate, z, iterations, _ptr(w), llr.shape[0], _ptr(llr),
                                             _ptr(cw), _ptr(g))
        return loss, g


class Reference:
    """The reference's own sources compiled here (``oracle/_ref``)."""

    def __init__(self, mode: int = NMS):
        path = os.path.join(REF_DIR, _REF_LIB[mode])
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
        L = self.lib
        L.ref_code_info.argtypes = [_i, _i, _p]
        L.ref_checknode_table.argtypes = [_i, _i, _p, _l]
        L.ref_decode_batch.argtypes = [_i, _i, _i, _l, _p, _p, _p, _i]
        L.ref_decode_bits_batch.argtypes = [_i, _i, _i, _l, _p, _p, _p, _i]
        L.ref_syndrome_batch.argtypes = [_i, _i, _l, _p, _i, _p]
        L.ref_iterations.argtypes = [_i, _i, _i, _l, _p, _p, _i]
        L.ref_encode_batch.argtypes = [_i, _i, _l, _p, _p, _i]
        L.ref_ber_create.argtypes = [_i, _i, _i, _i]
        L.ref_ber_create.restype = _p
        L.ref_ber_run_iteration.argtypes = [_p, ctypes.c_double]
        L.ref_ber_run_iteration.restype = ctypes.c_double
        L.ref_ber_reset.argtypes = [_p]
        L.ref_ber_bits.argtypes = [_p]
        L.ref_ber_bits.restype = ctypes.c_uint64
        L.ref_ber_errors.argtypes = [_p]
        L.ref_ber_errors.restype = ctypes.c_uint64
        L.ref_ber_codeword_len.argtypes = [_p]
        L.ref_ber_dataword_len.argtypes = [_p]
        L.ref_ber_destroy.argtypes = [_p]
        self.threads = os.cpu_count() or 1

    def code_info(self, rate, z):
        o = np.zeros(7, np.int32)
        if self.lib.ref_code_info(rate, z, _ptr(o)) != 0:
            raise ValueError("reference rejected rate/z")
        return dict(zip(["N", "M", "z", "rows", "cols", "D", "X"], o.tolist()))

    def checknode_table(self, rate, z):
        info = self.code_info(rate, z)
        t = np.empty(info["rows"] * info["cols"], np.int16)
        self.lib.ref_checknode_table(rate, z, _ptr(t), t.size)
        return t.reshape(info["rows"], info["cols"])

    def decode(self, rate, z, llr, max_iter=10, threads=None):
        """Returns (posterior, decoded, ret); llr is not modified."""
        post = np.ascontiguousarray(llr, np.float32).copy()
        dec = np.empty(post.shape, np.int8)
        ret = np.empty(post.shape[0], np.uint32)
        if self.lib.ref_decode_batch(rate, z, max_iter, post.shape[0], _ptr(post), _ptr(dec),
                                     _ptr(ret), threads or self.threads):
            raise ValueError("reference decode failed")
        return post, dec, ret

    def decode_bits(self, rate, z, bits, max_iter=10, threads=None):
        bits = np.ascontiguousarray(bits, np.int8).copy()
        dec = np.empty(bits.shape, np.int8)
        ret = np.empty(bits.shape[0], np.uint32)
        if self.lib.ref_decode_bits_batch(rate, z, max_iter, bits.shape[0], _ptr(bits), _ptr(dec),
                                          _ptr(ret), threads or self.threads):
            raise ValueError("reference decode failed")
        return dec, ret

    def syndrome(self, rate, z, bits, early_exit=False):
        bits = np.ascontiguousarray(bits, np.int8).copy()
        ret = np.empty(bits.shape[0], np.uint32)
        self.lib.ref_syndrome_batch(rate, z, bits.shape[0], _ptr(bits), int(early_exit), _ptr(ret))
        return ret

    def iterations(self, rate, z, llr, cap=10, threads=None):
        llr = np.ascontiguousarray(llr, np.float32)
        it = np.empty(llr.shape[0], np.int32)
        self.lib.ref_iterations(rate, z, cap, llr.shape[0], _ptr(llr), _ptr(it), threads or self.threads)
        return it

    def encode(self, rate, z, info, threads=None):
        info = np.ascontiguousarray(info, np.uint8)
        n = self.code_info(rate, z)["N"]
        cw = np.empty((info.shape[0], n), np.uint8)
        if self.lib.ref_encode_batch(rate, z, info.shape[0], _ptr(info), _ptr(cw), threads or self.threads):
            raise ValueError("reference encode failed")
        return cw
