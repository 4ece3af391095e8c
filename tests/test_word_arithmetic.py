"""The word buffer's arithmetic, restated on the CPU.

Adding launches of the CTA-pair kernel keep each visibility's sums of a call
as one 64-bit word, im * 2^32 + re (modulo 2^64), and add words with 64-bit
reduce-adds; the fold splits a word back into its parts as
re = (int32) low 32 bits, im = (word - re) >> 32 (arithmetic shift).  The
split is exact while both parts' sums stay inside the int32 range, which
bounds the samples the words may hold between folds: one sample adds at most
2 * 128^2 = 32768 to a part (int8 re*re + im*im at -128), so 65535 samples
stay below 2^31 and 65536 do not.  These checks restate that arithmetic with
numpy's wrapping uint64 operations."""
import numpy as np

MAX_PER_SAMPLE = 2 * 128 * 128
WORDS_MAX_SAMPLES = 65535


def pack(re, im):
    """im * 2^32 + re modulo 2^64, as the epilogue forms each call's word."""
    return (im.astype(np.int64).astype(np.uint64) << np.uint64(32)) + \
        re.astype(np.int64).astype(np.uint64)


def split(words):
    """The fold's split of a summed word into its two signed parts."""
    re = (words & np.uint64(0xFFFFFFFF)).astype(np.uint32).view(np.int32).astype(np.int64)
    im = (words - re.astype(np.uint64)).view(np.int64) >> np.int64(32)
    return re, im


def test_bound_of_samples_between_folds():
    assert MAX_PER_SAMPLE * WORDS_MAX_SAMPLES < 2**31
    assert MAX_PER_SAMPLE * (WORDS_MAX_SAMPLES + 1) >= 2**31


def test_sums_of_words_split_into_the_sums_of_their_parts():
    """Random per-call parts of both signs whose running sums stay inside
    int32, summed as words in any order, split exactly."""
    rng = np.random.default_rng(3)
    calls, nvis = 64, 4096
    limit = (2**31 - 1) // calls
    re = rng.integers(-limit, limit + 1, size=(calls, nvis), dtype=np.int64)
    im = rng.integers(-limit, limit + 1, size=(calls, nvis), dtype=np.int64)
    acc = np.zeros(nvis, dtype=np.uint64)
    for k in rng.permutation(calls):
        acc += pack(re[k], im[k])
    got_re, got_im = split(acc)
    assert np.array_equal(got_re, re.sum(axis=0))
    assert np.array_equal(got_im, im.sum(axis=0))


def test_extreme_sums_at_the_bound():
    """65535 samples of the largest contribution of either sign in either
    part: the sums reach +-2,147,450,880 and still split exactly."""
    per_call = 1008          # samples per call, as in the GPU test at the bound
    calls = WORDS_MAX_SAMPLES // per_call   # 65 calls, 65520 samples
    top = MAX_PER_SAMPLE * per_call
    corners = np.array([[top, top], [top, -top], [-top, top], [-top, -top]], dtype=np.int64)
    acc = np.zeros(4, dtype=np.uint64)
    for _ in range(calls):
        acc += pack(corners[:, 0], corners[:, 1])
    re, im = split(acc)
    assert np.array_equal(re, calls * corners[:, 0])
    assert np.array_equal(im, calls * corners[:, 1])
    assert int(np.abs(re).max()) == calls * top < 2**31
    # one sample short of the bound in a single part, both signs
    for v in (MAX_PER_SAMPLE * WORDS_MAX_SAMPLES, -MAX_PER_SAMPLE * WORDS_MAX_SAMPLES):
        w = pack(np.array([v]), np.array([-v]))
        r, i = split(w)
        assert int(r[0]) == v and int(i[0]) == -v


def test_split_fails_past_the_bound():
    """Past 2^31 the low part wraps: the reason the words are folded before
    they would hold more than 65535 samples."""
    v = MAX_PER_SAMPLE * (WORDS_MAX_SAMPLES + 1)      # 2^31
    r, i = split(pack(np.array([v]), np.array([0])))
    assert (int(r[0]), int(i[0])) != (v, 0)
