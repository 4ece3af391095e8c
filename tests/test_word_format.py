"""The tensor engine's short-term word format, restated in numpy on the CPU.

Accumulating calls of the tcgen05 engine reduce-add one int64 word per
visibility, w = im * 2^32 + re, into a short-term buffer (64-bit two's
complement, wrapping like the L2's .add.u64), which is folded into the int64
(re, im) integration buffer before it holds more than kWordSamples samples:
re is the word's low 32 bits read as a signed int32, im = (w - re) >> 32.
One sample adds at most 2^15 in magnitude to re or im (both products at
-128 x -128), so the decoding is exact up to 65535 samples; these tests check
the restated arithmetic at that bound, with extreme and random partial sums.
"""
import re as regex
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def word_samples_limit():
    text = open(os.path.join(ROOT, "xgpu_b200", "csrc", "tc_job.h")).read()
    return int(regex.search(r"kWordSamples\s*=\s*(\d+)", text).group(1))


def encode(re_part, im_part):
    with np.errstate(over="ignore"):
        return (np.asarray(im_part, np.int64) * np.int64(1 << 32) + np.asarray(re_part, np.int64))


def wrap_sum(words):
    """Sum in 64-bit two's complement, as reduce-adds of u64 in L2 do."""
    return np.asarray(words, np.int64).view(np.uint64).sum(dtype=np.uint64).view(np.int64)


def decode(w):
    w = np.asarray(w, np.int64)
    re_part = (w.view(np.uint64) & np.uint64(0xFFFFFFFF)).astype(np.uint32).view(np.int32)
    re_part = re_part.astype(np.int64)
    return re_part, (w - re_part) >> 32


def test_limit_keeps_sums_inside_int32():
    limit = word_samples_limit()
    assert limit % 16 == 0
    assert limit * (1 << 15) < (1 << 31)      # |sum| < 2^31 for re and im
    assert limit >= 32768                     # one full launch segment fits


def test_extreme_sums_decode_exactly():
    limit = word_samples_limit()
    full = 1 << 15            # one sample's largest contribution
    for s_re, s_im in [(full, full), (-full, -full), (full, -full), (-full, full), (0, -full),
                       (-full, 0), (1, -1), (-1, 1)]:
        # the sum of `limit` samples, added one call (one word) at a time
        per_call = 1024
        words = [encode(s_re * per_call, s_im * per_call)] * (limit // per_call)
        rest = limit % per_call
        if rest:
            words.append(encode(s_re * rest, s_im * rest))
        total = wrap_sum(np.array(words))
        got_re, got_im = decode(total)
        assert got_re == s_re * limit and got_im == s_im * limit


def test_random_partial_sums_decode_exactly():
    rng = np.random.default_rng(7)
    limit = word_samples_limit()
    full = 1 << 15
    for _ in range(200):
        ncalls = int(rng.integers(1, 65))
        samples = rng.multinomial(limit, np.ones(ncalls) / ncalls)
        re_parts = [int(rng.integers(-full * s, full * s + 1)) for s in samples]
        im_parts = [int(rng.integers(-full * s, full * s + 1)) for s in samples]
        total = wrap_sum(encode(re_parts, im_parts))
        got_re, got_im = decode(total)
        assert got_re == sum(re_parts) and got_im == sum(im_parts)
