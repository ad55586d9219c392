"""wimax_ldpc_lib_b200 -- Python bindings of the B200-native WiMAX QC-LDPC codec.

The product is ``lib/libwimax_ldpc_b200.so``: sm_100a kernels behind the C ABI
declared in ``include/wimax_ldpc_b200.h`` plus the C++ facade of the
reference's classes (``include/wimax_ldpc_lib/``). This module binds the C ABI
with ctypes so that tests and ``bench.py`` can drive it; torch is used only to
hold device memory and streams. There is no CPU fallback: if the shared library
is missing, importing the bindings raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libwimax_ldpc_b200.so")
INCLUDE_DIR = os.path.join(os.path.dirname(HERE), "include")

HALFRATE, TWOTHIRDSA, TWOTHIRDSB, THREEQUARTERSA, THREEQUARTERSB, FIVESIXTHS = range(6)
RATE_NAMES = ["1/2", "2/3A", "2/3B", "3/4A", "3/4B", "5/6"]
Z_VALUES = tuple(range(24, 97, 4))
MODE_NMS, MODE_OMS, MODE_MS = 0, 1, 2
LMS_F32, LMS_F16X2 = 0, 1   # learned-decoder inference arithmetic (wldpc_lms_set_precision)
MIXED_MSG_REGISTERS, MIXED_MSG_SHARED = 0, 1   # mixed decoder message layout (wldpc_mixed_set_tuning)
MIXED_CONCURRENT, MIXED_SERIAL = 0, 1           # mixed decoder launch policy of its six per-rate grids

OK = 0
ERR_ARG, ERR_CODE, ERR_CUDA, ERR_NO_DEVICE, ERR_TIMEOUT, ERR_UNSUPPORTED, ERR_SCRATCH = -1, -2, -3, -4, -5, -6, -7
WAIT_LIMIT_DEFAULT_US = 1000000   # WLDPC_WAIT_LIMIT_DEFAULT_US: bound of the kernels' waits

_p = ctypes.c_void_p
_i = ctypes.c_int
_u = ctypes.c_uint
_sz = ctypes.c_size_t


class LdpcError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        msg = _lib().wldpc_strerror(code).decode() if _LIB is not None else str(code)
        super().__init__(f"{what}: {msg} ({code})" if what else f"{msg} ({code})")


class CodeInfo(ctypes.Structure):
    _fields_ = [("rate", _i), ("z", _i), ("n", _i), ("m", _i), ("k", _i), ("rows", _i), ("cols", _i),
                ("D", _i), ("X", _i), ("layers", _i), ("edges", _i)]


_LIB = None


def build(jobs: int = 8) -> None:
    """Compile lib/libwimax_ldpc_b200.so with nvcc (sm_100a); no GPU needed."""
    import subprocess
    subprocess.check_call(["make", "-s", "-C", HERE, f"-j{jobs}"])


def _lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run wimax_ldpc_lib_b200.build() (make -C wimax_ldpc_lib_b200)")
    L = ctypes.CDLL(LIB_PATH)
    L.wldpc_strerror.restype = ctypes.c_char_p
    L.wldpc_strerror.argtypes = [_i]
    L.wldpc_version.argtypes = []
    L.wldpc_code_info_get.argtypes = [_i, _u, ctypes.POINTER(CodeInfo)]
    L.wldpc_checknode_table.argtypes = [_i, _u, _p, _sz]
    L.wldpc_decoder_create.argtypes = [_i, _u, _u, _u, _i, ctypes.POINTER(_p)]
    L.wldpc_decoder_destroy.argtypes = [_p]
    L.wldpc_decoder_decode.argtypes = [_p, _p, _p, ctypes.POINTER(_u), ctypes.POINTER(_i)]
    L.wldpc_decoder_decode_bits.argtypes = [_p, _p, _p, ctypes.POINTER(_u)]
    L.wldpc_decoder_compute_syndrome.argtypes = [_p, _p, _i, ctypes.POINTER(_u)]
    L.wldpc_decode_batch_device.argtypes = [_p, _p, _p, _p, _p, _sz, _p]
    L.wldpc_decode_batch_host.argtypes = [_p, _p, _p, _p, _p, _sz]
    L.wldpc_decode_batch_host_hard.argtypes = [_p, _p, _p, _p, _p, _sz]
    L.wldpc_decoder_set_wait_limit.argtypes = [_p, _u]
    L.wldpc_wait_bound_ns.argtypes = [_u, ctypes.POINTER(ctypes.c_uint64)]
    L.wldpc_decode_bits_batch_host.argtypes = [_p, _p, _p, _p, _sz]
    L.wldpc_syndrome_batch_host.argtypes = [_p, _p, _i, _p, _sz]
    L.wldpc_encode_batch_host.argtypes = [_p, _p, _p, _sz]
    L.wldpc_decoder_synchronize.argtypes = [_p]
    L.wldpc_encoder_create.argtypes = [_i, _u, _u, ctypes.POINTER(_p)]
    L.wldpc_encoder_destroy.argtypes = [_p]
    L.wldpc_encoder_encode.argtypes = [_p, _p, _p]
    L.wldpc_encode_batch_device.argtypes = [_p, _p, _p, _sz, _p]
    L.wldpc_framegen_device.argtypes = [_i, _u, ctypes.c_uint64, ctypes.c_uint64, _sz, ctypes.c_float,
                                        ctypes.c_float, _p, _p, _p, _p, _p]
    L.wldpc_lms_create.argtypes = [_i, _u, _u, ctypes.POINTER(_p)]
    L.wldpc_lms_destroy.argtypes = [_p]
    L.wldpc_lms_set_weights.argtypes = [_p, _p]
    L.wldpc_lms_get_weights.argtypes = [_p, _p]
    L.wldpc_lms_decode_device.argtypes = [_p, _p, _p, _p, _p, _sz, _p]
    L.wldpc_lms_set_cap.argtypes = [_p, _u]
    L.wldpc_lms_set_precision.argtypes = [_p, _i]
    L.wldpc_lms_decode_host.argtypes = [_p, _p, _p, _p, _p, _sz]
    L.wldpc_lms_decode_host_hard.argtypes = [_p, _p, _p, _p, _p, _sz]
    L.wldpc_lms_loss_grad.argtypes = [_p, _p, _p, _sz, _p, ctypes.POINTER(ctypes.c_double)]
    L.wldpc_lms_train.argtypes = [_p, _u, _u, ctypes.c_float, ctypes.c_float, ctypes.c_uint64, ctypes.c_uint64,
                                  ctypes.c_float, _p]
    L.wldpc_lms_grad_size.argtypes = [_p, ctypes.POINTER(_sz)]
    L.wldpc_lms_step_grad.argtypes = [_p, _u, ctypes.c_float, ctypes.c_float, ctypes.c_uint64, ctypes.c_uint64, _p,
                                      _p, _p]
    L.wldpc_lms_apply_grad.argtypes = [_p, _p, ctypes.c_float, _p]
    L.wldpc_decode_host_noalloc.argtypes = [_i, _u, _u, _p, _p, _p, _sz]
    L.wldpc_lfsr_bits_device.argtypes = [ctypes.c_uint64, _sz, _p, _p]
    L.wldpc_framegen_nullspace_device.argtypes = [_i, _u, ctypes.c_uint64, ctypes.c_uint64, _sz, ctypes.c_float,
                                                  ctypes.c_float, _p, _p, _p, _p]
    L.wldpc_variant.argtypes = [_i, _u]
    L.wldpc_mixed_create.argtypes = [_u, ctypes.POINTER(_p)]
    L.wldpc_mixed_destroy.argtypes = [_p]
    L.wldpc_mixed_decode_device.argtypes = [_p, _p, _p, _p, _p, _p, _p, _sz, _p]
    L.wldpc_mixed_synchronize.argtypes = [_p]
    L.wldpc_mixed_set_config.argtypes = [_p, _i, _i]
    L.wldpc_mixed_get_config.argtypes = [_p, ctypes.POINTER(_i), ctypes.POINTER(_i)]
    L.wldpc_mixed_set_tuning.argtypes = [_p, _i, _i, _i, _i]
    L.wldpc_mixed_set_rows_per_thread.argtypes = [_p, _i]
    L.wldpc_mixed_get_rows_per_thread.argtypes = [_p, ctypes.POINTER(_i)]
    L.wldpc_mixed_get_tuning.argtypes = [_p, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i),
                                         ctypes.POINTER(_i)]
    L.wldpc_mixed_autotune.argtypes = [_p, _p, _p, _p, _p, _sz, _i, ctypes.POINTER(ctypes.c_float)]
    L.wldpc_ber_runner_create.argtypes = [_i, _u, _u, _u, ctypes.POINTER(_p)]
    L.wldpc_ber_runner_destroy.argtypes = [_p]
    L.wldpc_ber_runner_run_iteration.argtypes = [_p, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
    L.wldpc_ber_runner_reset.argtypes = [_p]
    L.wldpc_ber_runner_totals.argtypes = [_p, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    L.wldpc_ber_runner_lengths.argtypes = [_p, ctypes.POINTER(_u), ctypes.POINTER(_u)]
    _LIB = L
    return L


def lib():
    """The loaded ctypes library (raises ImportError if it is not built)."""
    return _lib()


def _check(rc: int, what: str = "") -> None:
    if rc != OK:
        raise LdpcError(rc, what)


def _np_ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _t_ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream_ptr(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def wait_bound_ns(limit_us: int = WAIT_LIMIT_DEFAULT_US) -> int:
    """Device nanoseconds the kernels' bounded wait with that limit takes on a
    barrier that never completes."""
    ns = ctypes.c_uint64()
    _check(_lib().wldpc_wait_bound_ns(limit_us, ctypes.byref(ns)), "wait_bound_ns")
    return ns.value


def code_info(rate: int, z: int) -> CodeInfo:
    ci = CodeInfo()
    _check(_lib().wldpc_code_info_get(rate, z, ctypes.byref(ci)), "code_info")
    return ci


def checknode_table(rate: int, z: int) -> np.ndarray:
    ci = code_info(rate, z)
    t = np.empty(ci.rows * ci.cols, np.int16)
    _check(_lib().wldpc_checknode_table(rate, z, _np_ptr(t), t.size), "checknode_table")
    return t.reshape(ci.rows, ci.cols)


def reference_return(status: np.ndarray, max_iter: int) -> np.ndarray:
    """ldpc_decoder::decode's return value from a status word array."""
    s = np.asarray(status)
    return np.zeros(s.shape, np.uint32) if max_iter == 0 else ((s >> 16) & 1).astype(np.uint32)


class Decoder:
    """wldpc_decoder handle: ldpc_decoder(rate, z, max_iter, threads) plus batch calls."""

    def __init__(self, rate: int, z: int, max_iter: int = 10, mode: int = MODE_NMS, num_threads: int = 1):
        self.rate, self.z, self.max_iter, self.mode = rate, z, max_iter, mode
        self.info = code_info(rate, z)
        self.n, self.k = self.info.n, self.info.k
        h = ctypes.c_void_p()
        _check(_lib().wldpc_decoder_create(rate, z, max_iter, num_threads, mode, ctypes.byref(h)), "decoder")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib().wldpc_decoder_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- reference methods (single frame, host memory) ---
    def decode(self, rx: np.ndarray):
        """decode(float*, int8_t*): returns (posterior, decoded, num_errors, iterations)."""
        post = np.ascontiguousarray(rx, np.float32).copy()
        dec = np.empty(self.n, np.int8)
        ne, it = _u(), _i()
        _check(_lib().wldpc_decoder_decode(self._h, _np_ptr(post), _np_ptr(dec), ctypes.byref(ne),
                                           ctypes.byref(it)), "decode")
        return post, dec, ne.value, it.value

    def decode_bits(self, bits: np.ndarray):
        b = np.ascontiguousarray(bits, np.int8)
        dec = np.empty(self.n, np.int8)
        ne = _u()
        _check(_lib().wldpc_decoder_decode_bits(self._h, _np_ptr(b), _np_ptr(dec), ctypes.byref(ne)), "decode_bits")
        return dec, ne.value

    def compute_syndrome(self, bits: np.ndarray, exit_early: bool = False) -> int:
        b = np.ascontiguousarray(bits, np.int8)
        ne = _u()
        _check(_lib().wldpc_decoder_compute_syndrome(self._h, _np_ptr(b), int(exit_early), ctypes.byref(ne)),
               "compute_syndrome")
        return ne.value

    # --- batch ---
    def decode_host(self, llr: np.ndarray):
        """frames x n host batch; returns (posterior, decoded, num_errors, status)."""
        post = np.ascontiguousarray(llr, np.float32).copy()
        frames = post.shape[0]
        dec = np.empty(post.shape, np.int8)
        ne = np.empty(frames, np.uint32)
        st = np.empty(frames, np.int32)
        _check(_lib().wldpc_decode_batch_host(self._h, _np_ptr(post), _np_ptr(dec), _np_ptr(ne), _np_ptr(st),
                                              frames), "decode_batch_host")
        return post, dec, ne, st

    def decode_host_into(self, rx, decoded, num_errors=None, status=None):
        """In-place host batch on caller buffers (numpy or pinned torch CPU tensors)."""
        ptr = _np_ptr if isinstance(rx, np.ndarray) else _t_ptr
        frames = rx.shape[0]
        _check(_lib().wldpc_decode_batch_host(self._h, ptr(rx), ptr(decoded), ptr(num_errors), ptr(status),
                                              frames), "decode_batch_host")

    def decode_bits_host(self, bits: np.ndarray):
        """Batch decode(int8_t*, int8_t*) of frames x n host bytes: (decoded, num_errors)."""
        b = np.ascontiguousarray(bits, np.int8)
        dec = np.empty(b.shape, np.int8)
        ne = np.empty(b.shape[0], np.uint32)
        _check(_lib().wldpc_decode_bits_batch_host(self._h, _np_ptr(b), _np_ptr(dec), _np_ptr(ne), b.shape[0]),
               "decode_bits_batch_host")
        return dec, ne

    def syndrome_host(self, bits: np.ndarray, exit_early: bool = False) -> np.ndarray:
        """Batch compute_syndrome over frames x n host bytes."""
        b = np.ascontiguousarray(bits, np.int8)
        out = np.empty(b.shape[0], np.uint32)
        _check(_lib().wldpc_syndrome_batch_host(self._h, _np_ptr(b), int(exit_early), _np_ptr(out), b.shape[0]),
               "syndrome_batch_host")
        return out

    def decode_host_hard_into(self, llr, decoded, num_errors=None, status=None):
        """Host batch without the posterior (llr is read only; numpy or pinned torch CPU tensors)."""
        ptr = _np_ptr if isinstance(llr, np.ndarray) else _t_ptr
        _check(_lib().wldpc_decode_batch_host_hard(self._h, ptr(llr), ptr(decoded), ptr(num_errors), ptr(status),
                                                   llr.shape[0]), "decode_batch_host_hard")

    def decode_device(self, llr, decoded, posterior=None, status=None, stream=None):
        """torch CUDA tensors, asynchronous on `stream` (default: torch's current stream)."""
        frames = llr.shape[0]
        _check(_lib().wldpc_decode_batch_device(self._h, _t_ptr(llr), _t_ptr(decoded), _t_ptr(posterior),
                                                _t_ptr(status), frames, _stream_ptr(stream)), "decode_batch_device")

    def set_wait_limit(self, limit_us: int) -> None:
        """Test hook: bound of the kernel's staging wait in microseconds (0 = time out at once)."""
        _check(_lib().wldpc_decoder_set_wait_limit(self._h, limit_us), "set_wait_limit")

    def synchronize(self):
        _check(_lib().wldpc_decoder_synchronize(self._h), "synchronize")


class Encoder:
    def __init__(self, rate: int, z: int, num_threads: int = 1):
        self.rate, self.z = rate, z
        self.info = code_info(rate, z)
        self.n, self.k = self.info.n, self.info.k
        h = ctypes.c_void_p()
        _check(_lib().wldpc_encoder_create(rate, z, num_threads, ctypes.byref(h)), "encoder")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib().wldpc_encoder_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def encode(self, info: np.ndarray) -> np.ndarray:
        u = np.ascontiguousarray(info, np.uint8)
        cw = np.empty(self.n, np.uint8)
        _check(_lib().wldpc_encoder_encode(self._h, _np_ptr(u), _np_ptr(cw)), "encode")
        return cw

    def encode_device(self, info, codeword, stream=None):
        _check(_lib().wldpc_encode_batch_device(self._h, _t_ptr(info), _t_ptr(codeword), info.shape[0],
                                                _stream_ptr(stream)), "encode_batch_device")


def framegen_device(rate, z, seed, first_frame, frames, ebno_lo, ebno_hi=None, info=None, codeword=None,
                    llr=None, ebno=None, stream=None):
    """Seeded synthetic frames into torch CUDA tensors (any may be None)."""
    ebno_hi = ebno_lo if ebno_hi is None else ebno_hi
    _check(_lib().wldpc_framegen_device(rate, z, seed, first_frame, frames, ebno_lo, ebno_hi, _t_ptr(info),
                                        _t_ptr(codeword), _t_ptr(llr), _t_ptr(ebno), _stream_ptr(stream)),
           "framegen")


def framegen_nullspace_device(rate, z, seed, first_frame, frames, ebno_lo, ebno_hi=None, codeword=None, llr=None,
                              ebno=None, stream=None):
    """Random codewords from the null space of H (any rate, 3/4B included) with AWGN LLRs."""
    ebno_hi = ebno_lo if ebno_hi is None else ebno_hi
    _check(_lib().wldpc_framegen_nullspace_device(rate, z, seed, first_frame, frames, ebno_lo, ebno_hi,
                                                  _t_ptr(codeword), _t_ptr(llr), _t_ptr(ebno), _stream_ptr(stream)),
           "framegen_nullspace")


def variant(rate: int, z: int) -> int:
    v = _lib().wldpc_variant(rate, z)
    _check(min(v, 0), "variant")
    return v


class MixedDecoder:
    """wldpc_mixed handle: one graph launch decodes frames of any mix of codes."""

    def __init__(self, max_iter: int = 10):
        h = ctypes.c_void_p()
        _check(_lib().wldpc_mixed_create(max_iter, ctypes.byref(h)), "mixed decoder")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib().wldpc_mixed_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def decode_device(self, variants, offsets, llr, decoded, posterior=None, status=None, stream=None):
        _check(_lib().wldpc_mixed_decode_device(self._h, _t_ptr(variants), _t_ptr(offsets), _t_ptr(llr),
                                                _t_ptr(decoded), _t_ptr(posterior), _t_ptr(status),
                                                variants.numel(), _stream_ptr(stream)), "mixed decode")

    def synchronize(self):
        _check(_lib().wldpc_mixed_synchronize(self._h), "mixed synchronize")

    def set_config(self, threads: int, chunk: int):
        _check(_lib().wldpc_mixed_set_config(self._h, threads, chunk), "mixed config")

    def config(self):
        t, c = _i(), _i()
        _check(_lib().wldpc_mixed_get_config(self._h, ctypes.byref(t), ctypes.byref(c)), "mixed config")
        return t.value, c.value

    def set_tuning(self, threads: int, layout: int, chunk: int, launch: int = MIXED_CONCURRENT):
        """CTA size (96 | 192), message layout (MIXED_MSG_*), frames per work
        item (1..64) and launch policy (MIXED_CONCURRENT | MIXED_SERIAL)."""
        _check(_lib().wldpc_mixed_set_tuning(self._h, threads, layout, chunk, launch), "mixed tuning")

    def tuning(self):
        """(threads, layout, chunk, launch)"""
        t, l, c, p = _i(), _i(), _i(), _i()
        _check(_lib().wldpc_mixed_get_tuning(self._h, ctypes.byref(t), ctypes.byref(l), ctypes.byref(c),
                                             ctypes.byref(p)), "mixed tuning")
        return t.value, l.value, c.value, p.value

    def set_rows_per_thread(self, rows: int):
        """1 or 2 expanded rows per thread: z or z/2 threads per frame."""
        _check(_lib().wldpc_mixed_set_rows_per_thread(self._h, rows), "mixed rows per thread")

    def rows_per_thread(self) -> int:
        r = _i()
        _check(_lib().wldpc_mixed_get_rows_per_thread(self._h, ctypes.byref(r)), "mixed rows per thread")
        return r.value

    def autotune(self, variants, offsets, llr, decoded, repeats: int = 3) -> float:
        ms = ctypes.c_float()
        _check(_lib().wldpc_mixed_autotune(self._h, _t_ptr(variants), _t_ptr(offsets), _t_ptr(llr), _t_ptr(decoded),
                                           variants.numel(), repeats, ctypes.byref(ms)), "mixed autotune")
        return ms.value


def lfsr_bits_device(first_bit: int, out, stream=None) -> None:
    """The reference BER_runner's info-bit stream from position first_bit into a uint8 CUDA tensor."""
    _check(_lib().wldpc_lfsr_bits_device(first_bit, out.numel(), _t_ptr(out), _stream_ptr(stream)), "lfsr")


class LearnedDecoder:
    """wldpc_lms handle: learned normalized/offset min-sum (weights per
    iteration, layer and base column), its training and inference."""

    def __init__(self, rate: int, z: int, iterations: int = 8, weights=None, cap: int | None = None,
                 precision: int = LMS_F32):
        self.rate, self.z, self.iterations = rate, z, iterations
        self.info = code_info(rate, z)
        self.n, self.k = self.info.n, self.info.k
        h = ctypes.c_void_p()
        _check(_lib().wldpc_lms_create(rate, z, iterations, ctypes.byref(h)), "learned decoder")
        self._h = h
        self.precision = LMS_F32
        if weights is not None:
            self.set_weights(weights)
        if cap is not None:
            self.set_cap(cap)
        if precision != LMS_F32:
            self.set_precision(precision)

    def set_precision(self, precision: int) -> None:
        """LMS_F32 (fp32 inference) or LMS_F16X2 (two frames per thread in
        packed binary16; needs |a| <= 2 and 0 <= b <= 1024)."""
        _check(_lib().wldpc_lms_set_precision(self._h, precision), "set_precision")
        self.precision = precision

    def set_cap(self, cap: int) -> None:
        """Iteration cap; iterations past the trained ones reuse the last iteration's weights."""
        _check(_lib().wldpc_lms_set_cap(self._h, cap), "set_cap")
        self.cap = cap

    def close(self):
        if getattr(self, "_h", None):
            _lib().wldpc_lms_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def table_shape(self):
        return (2, self.iterations, 12, 24)

    def get_weights(self) -> np.ndarray:
        t = np.zeros(self.table_shape, np.float32)
        _check(_lib().wldpc_lms_get_weights(self._h, _np_ptr(t)), "get_weights")
        return t

    def set_weights(self, table) -> None:
        t = np.ascontiguousarray(table, np.float32).reshape(self.table_shape)
        _check(_lib().wldpc_lms_set_weights(self._h, _np_ptr(t)), "set_weights")

    def decode_device(self, llr, decoded, posterior=None, status=None, stream=None):
        _check(_lib().wldpc_lms_decode_device(self._h, _t_ptr(llr), _t_ptr(decoded), _t_ptr(posterior),
                                              _t_ptr(status), llr.shape[0], _stream_ptr(stream)), "lms decode")

    def decode_host(self, llr: np.ndarray):
        post = np.ascontiguousarray(llr, np.float32).copy()
        frames = post.shape[0]
        dec = np.empty(post.shape, np.int8)
        ne = np.empty(frames, np.uint32)
        st = np.empty(frames, np.int32)
        _check(_lib().wldpc_lms_decode_host(self._h, _np_ptr(post), _np_ptr(dec), _np_ptr(ne), _np_ptr(st), frames),
               "lms decode_host")
        return post, dec, ne, st

    def decode_host_into(self, rx, decoded, num_errors=None, status=None):
        """In-place host batch (posterior written back into rx); numpy or pinned torch CPU tensors."""
        ptr = _np_ptr if isinstance(rx, np.ndarray) else _t_ptr
        _check(_lib().wldpc_lms_decode_host(self._h, ptr(rx), ptr(decoded), ptr(num_errors), ptr(status),
                                            rx.shape[0]), "lms decode_host")

    def decode_host_hard_into(self, llr, decoded, num_errors=None, status=None):
        """Host batch without the posterior (llr is read only)."""
        ptr = _np_ptr if isinstance(llr, np.ndarray) else _t_ptr
        _check(_lib().wldpc_lms_decode_host_hard(self._h, ptr(llr), ptr(decoded), ptr(num_errors), ptr(status),
                                                 llr.shape[0]), "lms decode_host_hard")

    def loss_grad(self, llr: np.ndarray, codeword: np.ndarray):
        l = np.ascontiguousarray(llr, np.float32)
        c = np.ascontiguousarray(codeword, np.uint8)
        g = np.zeros(self.table_shape, np.float32)
        loss = ctypes.c_double()
        _check(_lib().wldpc_lms_loss_grad(self._h, _np_ptr(l), _np_ptr(c), l.shape[0], _np_ptr(g),
                                          ctypes.byref(loss)), "lms loss_grad")
        return loss.value, g

    def train(self, steps: int, batch: int, ebno_lo: float, ebno_hi: float, seed: int, first_frame: int = 0,
              lr: float = 1e-3) -> np.ndarray:
        hist = np.zeros(max(steps, 1), np.float32)
        _check(_lib().wldpc_lms_train(self._h, steps, batch, ebno_lo, ebno_hi, seed, first_frame, lr,
                                      _np_ptr(hist)), "lms train")
        return hist[:steps]

    def grad_size(self) -> int:
        nw = ctypes.c_size_t()
        _check(_lib().wldpc_lms_grad_size(self._h, ctypes.byref(nw)), "grad_size")
        return nw.value

    def step_grad(self, batch: int, ebno_lo: float, ebno_hi: float, seed: int, first_frame: int, grad, loss=None,
                  stream=None):
        """Gradient of one generated batch into `grad` (float32 CUDA tensor of
        grad_size() values) and its loss into `loss` (one float32, optional);
        the weights do not change."""
        _check(_lib().wldpc_lms_step_grad(self._h, batch, ebno_lo, ebno_hi, seed, first_frame, _t_ptr(grad),
                                          _t_ptr(loss), _stream_ptr(stream)), "lms step_grad")

    def apply_grad(self, grad, lr: float = 1e-3, stream=None):
        """One Adam step with the gradient in `grad` (float32 CUDA tensor)."""
        _check(_lib().wldpc_lms_apply_grad(self._h, _t_ptr(grad), lr, _stream_ptr(stream)), "lms apply_grad")


WEIGHTS_DIR = os.path.join(HERE, "weights")


def learned_weights(rate: int, z: int, evaluated_only: bool = True):
    """Shipped learned min-sum weights for (rate, z): the table trained at
    that z, else the one trained at the nearest z of the same rate (the
    weights are per iteration, layer and base column, so a table applies to
    every z of its rate). Returns (meta, weights float32 [2][T][12][24],
    source z), or (None, None, None) when the rate has no trained table or,
    with evaluated_only, when a transferred table was never evaluated at that
    z (weights/lms_transfer.json). meta["evaluation"] holds the held-out
    evaluation at (rate, z) when there is one."""
    import json
    trained = []
    for name in os.listdir(WEIGHTS_DIR) if os.path.isdir(WEIGHTS_DIR) else []:
        parts = name[:-5].split("_") if name.startswith("lms_r") and name.endswith(".json") else []
        if len(parts) == 4 and parts[1] == f"r{rate}" and parts[2].startswith("z"):
            trained.append((int(parts[2][1:]), name))
    if not trained:
        return None, None, None
    src_z, name = min(trained, key=lambda t: (abs(t[0] - z), -t[0]))
    with open(os.path.join(WEIGHTS_DIR, name)) as f:
        meta = json.load(f)
    if src_z != z:
        ev = None
        tpath = os.path.join(WEIGHTS_DIR, "lms_transfer.json")
        if os.path.exists(tpath):
            with open(tpath) as f:
                for c in json.load(f)["codes"]:
                    if c["rate"] == rate and c["z"] == z and c["source_z"] == src_z:
                        ev = {"points": c["points"], "source": c["source"]}
        if ev is None and evaluated_only:
            return None, None, None
        meta = dict(meta, z=z, source_z=src_z, evaluation=ev)
    return meta, np.array(meta["weights"], np.float32), src_z


class BERRunner:
    def __init__(self, rate: int, z: int, num_threads: int = 1, max_iter: int = 10):
        h = ctypes.c_void_p()
        _check(_lib().wldpc_ber_runner_create(rate, z, num_threads, max_iter, ctypes.byref(h)), "BER_runner")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib().wldpc_ber_runner_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run_iteration(self, ebno_db: float) -> float:
        b = ctypes.c_double()
        _check(_lib().wldpc_ber_runner_run_iteration(self._h, ebno_db, ctypes.byref(b)), "run_iteration")
        return b.value

    def reset_test(self):
        _lib().wldpc_ber_runner_reset(self._h)

    def totals(self):
        b, e = ctypes.c_uint64(), ctypes.c_uint64()
        _lib().wldpc_ber_runner_totals(self._h, ctypes.byref(b), ctypes.byref(e))
        return b.value, e.value

    def lengths(self):
        c, d = _u(), _u()
        _lib().wldpc_ber_runner_lengths(self._h, ctypes.byref(c), ctypes.byref(d))
        return c.value, d.value
