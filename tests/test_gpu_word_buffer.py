"""The CTA-pair kernel's short-term word buffer.

Launches of the CTA-pair kernel whose work items drain with the split
epilogue (at most 8 stages of 128 samples) put each visibility's sums of the
call into one 64-bit word, im * 2^32 + re -- storing them when the words hold
nothing and the launch has one item per tile, adding them otherwise -- and
the context moves the words into its int64 integration buffer (storing when
that holds nothing yet) before every read, on xgpuFlushIntegrationBuffer, and
before the words would hold more than 65535 samples (while each part's sum
stays below 2^31 in magnitude, the two parts separate exactly).  These tests
drive sums to within 0.03% of that bound, with both signs in both parts, over
several 32-station blocks (diagonal and off-diagonal), and check every read
path, a clear with words pending, launches with time splits, a change of
kernel in the middle of an integration and calls whose time segments go to
different buffers.  The oracle's sums are exact int64, as xGPU's integer
engine would hold them without wrapping (cpu_xengine.c:16-60 restated in
oracle/).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, F, T = 256, 3, 1008        # 8 stages of 128 samples (the last one partial): word mode
WORD_CALLS = 65               # 65 x 1008 = 65520 samples, the most below 65536 in steps of 1008


def extreme_input():
    """Every sample the same: each station/polarisation is one of the four
    corners (+-128 / 127 in re and im), so that re and im sums of both signs
    come within 0.03% of 2^31 after 65520 samples."""
    corners = np.array([[-128, -128], [127, -128], [-128, 127], [127, 127]], dtype=np.int8)
    rng = np.random.default_rng(5)
    pick = rng.integers(0, 4, size=(F, N, 2))
    one = corners[pick]                                    # [f][s][p][re,im]
    return np.ascontiguousarray(np.broadcast_to(one, (T, F, N, 2, 2))).reshape(-1)


@pytest.fixture(scope="module")
def case(oracle_mod):
    x = extreme_input()
    one = oracle_mod.xengine_i64(x, N, F, T)
    return x, one


def make(xg):
    c = xg.Correlator(N, F, T, ntimepipe=16, engine="tensor", output="int32", order="tri")
    c.tune(1, 0, 1)                     # CTA pairs, one time split, full grid
    return c


def test_sums_at_the_word_bound(xg, case):
    """65 calls, all in the words (65520 samples: the largest re sum is
    2^31 - 524288), read by the int64 dump (the fold stores them into the
    empty int64 buffer); then 140 more calls, which fold twice on the way
    (adding), read again."""
    import torch
    x, one = case
    assert int(np.abs(one).max()) * WORD_CALLS > 2**31 - 2**20
    d = torch.from_numpy(x).cuda()
    torch.cuda.synchronize()
    with make(xg) as c:
        for _ in range(WORD_CALLS):
            c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump_int64(), WORD_CALLS * one)
        for _ in range(140):
            c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump_int64(), (WORD_CALLS + 140) * one)
        c.clear()
        for _ in range(WORD_CALLS + 1):   # the last call folds the first 65 (stored) first
            c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump_int64(), (WORD_CALLS + 1) * one)


def test_flush_then_more_calls(xg, case):
    """xgpuFlushIntegrationBuffer in the middle of an integration changes no
    sum: the calls after it start new words."""
    import torch
    x, one = case
    d = torch.from_numpy(x).cuda()
    torch.cuda.synchronize()
    with make(xg) as c:
        for k in range(40):
            c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
            if k in (3, 4, 17):
                c.flush()
        c.flush()
        c.flush()                       # nothing pending: a no-op
        torch.cuda.synchronize()
        assert np.array_equal(c.dump_int64(), 40 * one)


def test_clear_discards_pending_words(xg, case, oracle_mod):
    """A clear with words pending discards them with the rest of the
    integration; the next integration (other input) starts from zero."""
    import torch
    x, one = case
    y = oracle_mod.gaussian_input(N, F, T, seed=41, sigma=40.0)
    dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    torch.cuda.synchronize()
    want_y = oracle_mod.xengine_i64(y, N, F, T)
    with make(xg) as c:
        for _ in range(30):
            c.run_device(dx.data_ptr(), xg.SYNCOP_NONE)
        c.clear()
        for _ in range(3):
            c.run_device(dy.data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump_int64(), 3 * want_y)


def test_every_read_path_sees_the_words(xg, case, oracle_mod):
    """Words pending at a dump reach every reader: the int32 dump of
    xgpuDumpDeviceIntegrationBuffer (wrapping like xGPU's int32 buffer), the
    dumping call over device input, and the dumping call over host input
    (whose own launches add straight into the int64 buffer while the dump's
    channel groups are formatted)."""
    import torch
    x, one = case
    d = torch.from_numpy(x).cuda()
    torch.cuda.synchronize()
    with make(xg) as c:
        for _ in range(12):
            c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump(), (12 * one).astype(np.int32))
        c.run_device(d.data_ptr(), xg.SYNCOP_DUMP)
        assert np.array_equal(c.output_view()[: c.info.matLength * 2], (13 * one).astype(np.int32))
        for _ in range(5):
            c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        c.set_input(x)
        c.run(xg.SYNCOP_DUMP)
        assert np.array_equal(c.output_view()[: c.info.matLength * 2], (19 * one).astype(np.int32))
        assert np.array_equal(c.dump_int64(), 19 * one)


def test_time_splits_and_a_change_of_kernel(xg, oracle_mod):
    """Word launches with two time splits (items of 8 stages, T = 2048) add
    into words cleared first once they hold stale sums (after a fold or a
    clear); switching to single CTAs and back in the middle of an
    integration leaves sums in both buffers, which every dump joins."""
    import torch
    n, f, t = 256, 2, 2048
    xs = [oracle_mod.gaussian_input(n, f, t, seed=60 + q, sigma=40.0) for q in range(3)]
    ds = [torch.from_numpy(x).cuda() for x in xs]
    torch.cuda.synchronize()
    w = [oracle_mod.xengine_i64(x, n, f, t) for x in xs]
    with xg.Correlator(n, f, t, engine="tensor", output="int32", order="tri") as c:
        c.tune(2, 0, 1)
        for d in ds:
            c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump_int64(), w[0] + w[1] + w[2])
        c.run_device(ds[0].data_ptr(), xg.SYNCOP_NONE)          # stale words: cleared first
        assert np.array_equal(c.dump_int64(), 2 * w[0] + w[1] + w[2])
        c.clear()
        c.run_device(ds[1].data_ptr(), xg.SYNCOP_NONE)          # words only
        c.tune(1, 0, 0)                                         # single CTAs: the int64 buffer
        c.run_device(ds[2].data_ptr(), xg.SYNCOP_NONE)
        c.tune(1, 0, 1)                                         # pairs, one item per tile
        c.run_device(ds[0].data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump_int64(), w[0] + w[1] + w[2])
        c.clear()
        c.tune(1, 0, 0)
        c.run_device(ds[2].data_ptr(), xg.SYNCOP_NONE)          # the int64 buffer first
        c.tune(2, 0, 1)
        c.run_device(ds[1].data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump_int64(), w[1] + w[2])


def test_segments_in_both_buffers(xg, oracle_mod):
    """A call of 65536 + 512 samples runs as three launches of at most 32768
    samples: the two long segments go to the int64 buffer (joint epilogue),
    the short third one to the words; over calls, clears and dumps the sums
    stay exact."""
    import torch
    n, f, t = 64, 2, 65536 + 512
    xs = [oracle_mod.gaussian_input(n, f, t, seed=80 + q, sigma=20.0) for q in range(2)]
    ds = [torch.from_numpy(x).cuda() for x in xs]
    torch.cuda.synchronize()
    w = [oracle_mod.xengine_i64(x, n, f, t) for x in xs]
    with xg.Correlator(n, f, t, ntimepipe=128, engine="tensor", output="int32", order="tri") as c:
        c.tune(1, 0, 1)
        for d in ds + ds:
            c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump_int64(), 2 * (w[0] + w[1]))
        c.clear()
        c.run_device(ds[1].data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump_int64(), w[1])


@pytest.mark.parametrize("n", [32, 96, 160, 224])
def test_odd_block_counts(xg, oracle_mod, n):
    """With an odd number of 32-station blocks the last pair tile's second CTA
    holds a block past the last station; it writes no words (its offset would
    be the next channel's block, or past the buffer for the last channel), so
    storing calls leave every channel's words intact."""
    import torch
    f, t = 3, 1024
    xs = [oracle_mod.gaussian_input(n, f, t, seed=n + q, sigma=30.0) for q in range(2)]
    ds = [torch.from_numpy(x).cuda() for x in xs]
    torch.cuda.synchronize()
    w = [oracle_mod.xengine_i64(x, n, f, t) for x in xs]
    with xg.Correlator(n, f, t, engine="tensor", output="int32", order="tri") as c:
        c.tune(1, 0, 1)
        for d in ds + ds + ds:
            c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump_int64(), 3 * (w[0] + w[1]))
        c.run_device(ds[1].data_ptr(), xg.SYNCOP_NONE)          # stored into stale words
        c.run_device(ds[0].data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump_int64(), 4 * (w[0] + w[1]))
