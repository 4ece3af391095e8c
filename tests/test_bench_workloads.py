"""The bench's synthetic workloads, checked on the CPU: the 96-subarray batch
and the served request stream are seeded draws with the stated ranges, and
the same seed gives the same workload (so every run measures the same work)."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_uneven_subarrays_are_seeded_and_in_range():
    shapes = bench.uneven_subarray_shapes()
    assert shapes == bench.uneven_subarray_shapes()
    assert len(shapes) == 96
    for n, f, t, sigma in shapes:
        assert 32 <= n <= 1024 and n % 16 == 0
        assert 1 <= f <= 64
        assert 256 <= t <= 8192 and t % 256 == 0
        assert 4.0 <= sigma <= 32.0
    # log-uniform stations: both small and large arrays occur
    ns = np.array([s[0] for s in shapes])
    assert ns.min() < 64 and ns.max() > 512


def test_served_requests_are_a_seeded_poisson_stream():
    seconds, rate = 10.0, 200.0
    reqs = bench.served_requests(seconds, rate_jobs=rate)
    assert reqs == bench.served_requests(seconds, rate_jobs=rate)
    arrivals = np.array([r["arrival_s"] for r in reqs])
    assert (np.diff(arrivals) > 0).all() and arrivals[-1] <= seconds
    # Poisson count: mean rate * seconds = 2000, standard deviation ~45
    assert abs(len(reqs) - rate * seconds) < 5 * np.sqrt(rate * seconds)
    for r in reqs:
        assert 32 <= r["nstation"] <= 1024 and r["nstation"] % 16 == 0
        assert 1 <= r["nfrequency"] <= 64
        assert r["ntime"] % 256 == 0 and 256 <= r["ntime"] <= 8192
        assert 4 <= r["nblocks"] <= 32
    assert len({r["seed"] for r in reqs}) == len(reqs)


def test_ops_formula_is_the_reference_flop_count():
    # 16 F T N(N+1): 8 operations per complex multiply-add over N(N+1)/2
    # baselines and 4 polarisation products (kernel.cuh:419)
    assert bench.ops(256, 10, 1024) == 16 * 10 * 1024 * 256 * 257


def test_served_check_sample_is_seeded_and_covers_a_large_array():
    reqs = bench.served_requests(60.0)
    pick = bench.served_check_sample(reqs)
    assert pick == bench.served_check_sample(reqs)
    assert len(pick) >= 12
    assert any(reqs[q]["nstation"] > 512 for q in pick)
    small = [q for q in pick if reqs[q]["nstation"] <= 512]
    assert all(bench.request_ops(reqs[q]) <= 3e11 for q in small)


def test_channel_input_is_the_channel_of_the_generated_block(oracle_mod):
    """The large-array leg regenerates one channel of a device-generated block
    on the host; it must be that channel's slice of the whole block."""
    n, f_total, t = 32, 5, 64
    for kind, width in ((0, 4), (1, 2)):
        full = oracle_mod.generate(t * f_total * n * width, kind, 9000, 40.0)
        for f in (0, f_total - 1):
            want = np.ascontiguousarray(full.reshape(t, f_total, n * width)[:, f, :]).reshape(-1)
            if kind == 1:
                want = oracle_mod.unpack4(want)
            got = bench.channel_input(oracle_mod, kind, 9000, 40.0, n, f_total, t, f)
            assert np.array_equal(got, want)


def test_fold_launches_counted_in_the_timed_region():
    """gpu_launches counts the word buffer's folds: the words take every call
    from the first one, a fold comes before they would pass 65535 samples
    (calls 63, 126, 189 at T=1024) and one closes the timed region."""
    pair = {"pair": 1, "ksplit": 1}
    assert bench.word_folds(pair, 1024, 5, 20) == 1
    assert bench.word_folds(pair, 1024, 10, 200) == 4
    assert bench.word_folds(pair, 1024, 70, 3) == 1      # the fold at call 63 is in warm-up
    assert bench.word_folds(pair, 1024, 63, 3) == 2      # call 63 is timed
    assert bench.word_folds(pair, 8192, 3, 20) == 0      # 64-stage items: int64 buffer
    assert bench.word_folds({"pair": 1, "ksplit": 8}, 8192, 3, 20) == 4   # calls 7, 14, 21 + 1
    assert bench.word_folds({"pair": 0, "ksplit": 1}, 1024, 3, 20) == 0
    assert bench.word_folds(None, 1024, 3, 20) == 0
