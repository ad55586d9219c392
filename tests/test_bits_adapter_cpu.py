"""The decode(int8_t*) adapter's arithmetic (bits_to_llr_kernel): the
reference computes bit*2.0-1.0 in double and stores a float (reference
lib/ldpc_decoder.cc:108-118); the kernel adds 2b - 1 to the mantissa of
1.5 * 2^23 (bit pattern 0x4B3FFFFF + 2b) and subtracts 1.5 * 2^23 in float.
Both give the same float, sign included, for every int8 value."""
import numpy as np


def test_mantissa_conversion_equals_the_reference_double_arithmetic():
    b = np.arange(-128, 128, dtype=np.int64)
    pattern = ((0x4B3FFFFF + 2 * b) & 0xFFFFFFFF).astype(np.uint32)
    got = pattern.view(np.float32) - np.float32(12582912.0)
    want = (b.astype(np.float64) * 2.0 - 1.0).astype(np.float32)
    assert got.dtype == np.float32
    assert (got.view(np.uint32) == want.view(np.uint32)).all()
