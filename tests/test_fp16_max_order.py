"""The property the fp16x2 running maximum of sw_qpair4_kernel<..., HMAX>
rests on, checked exhaustively on the CPU: for every 16-bit pattern from the
bias 1024 (0x0400, the smallest positive normal fp16) up to 0x7c00 (+inf), the
fp16 value order equals the integer order, so a half-precision max of H's bit
patterns is their integer max; NaN patterns (0x7c01-0x7fff) lose to any number
(IEEE maxNum), and patterns with the sign bit set count as negative."""
import numpy as np


def test_positive_fp16_patterns_order_like_integers():
    pats = np.arange(0x0400, 0x7C01, dtype=np.uint16)
    vals = pats.view(np.float16).astype(np.float64)
    assert np.all(np.diff(vals) > 0)


def test_nan_and_negative_patterns_never_win():
    nan = np.arange(0x7C01, 0x8000, dtype=np.uint16).view(np.float16)
    assert np.all(np.isnan(nan))
    # maxNum semantics: fmax ignores NaN
    a = np.full(nan.shape, np.float16(1024 * 2.0 ** -24 * 1024), dtype=np.float16)
    assert np.all(np.fmax(a, nan) == a)
    neg = np.arange(0x8000, 0x10000, dtype=np.uint32).astype(np.uint16).view(np.float16)
    finite = neg[np.isfinite(neg)]
    assert np.all(finite <= 0)
