"""The continuous-batching server: every request's result is the same in the
mix as alone (and equal to the oracle), under admission pressure, with
periodic dumps, and in the one-request-at-a-time plain baseline."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MB = 1 << 20


def requests(n_req=12, seed=4, rate=2e6, span=0.05):
    rng = np.random.default_rng(seed)
    arrivals = np.sort(rng.uniform(0, span, n_req))
    out = []
    for q in range(n_req):
        out.append({"nstation": int(rng.choice([16, 32, 48, 64, 96, 128])),
                    "nfrequency": int(rng.integers(1, 5)),
                    "ntime": int(256 * rng.integers(1, 5)),
                    "nblocks": int(rng.integers(2, 6)),
                    "seed": 1000 + q, "sigma": float(rng.uniform(4, 32)),
                    "arrival_s": float(arrivals[q])})
    return out


def expected(oracle_mod, r):
    n, f, t = r["nstation"], r["nfrequency"], r["ntime"]
    acc = np.zeros(f * n * (n + 1) // 2 * 8, dtype=np.int64)
    for b in range(r["nblocks"]):
        x = oracle_mod.serve_block_input(n, f, t, r["seed"], r["sigma"], b)
        oracle_mod.xengine_i64(x, n, f, t, acc=acc)
    return acc.astype(np.int32)


def test_mix_equals_alone_and_oracle(xg, oracle_mod):
    reqs = requests()
    stats, res = xg.serve(reqs, 2e6, 512 * MB, host_budget_bytes=256 * MB, collect=True)
    assert stats["jobs"] == len(reqs) and stats["dumps"] == len(reqs)
    assert stats["admitted_peak"] >= 2          # requests really overlapped
    for r, got in zip(reqs, res):
        assert np.array_equal(got, expected(oracle_mod, r)), r
    # the first request alone
    alone = dict(reqs[3], arrival_s=0.0)
    _, res1 = xg.serve([alone], 2e6, 512 * MB, host_budget_bytes=256 * MB, collect=True)
    assert np.array_equal(res1[0], res[3])


def test_admission_under_a_small_budget(xg, oracle_mod):
    reqs = requests(8, seed=5)
    # room for roughly one or two requests at a time
    biggest = max(r["nfrequency"] * r["nstation"] * (r["nstation"] + 1) // 2 * 96 for r in reqs)
    stats, res = xg.serve(reqs, 2e6, max(2 * MB, int(1.5 * biggest)), host_budget_bytes=256 * MB,
                          collect=True)
    assert stats["jobs"] == len(reqs)
    assert stats["admitted_peak"] < len(reqs)
    for r, got in zip(reqs, res):
        assert np.array_equal(got, expected(oracle_mod, r))


def test_periodic_dumps_and_plain_baseline(xg, oracle_mod):
    reqs = requests(6, seed=6)
    for r in reqs:
        r["dump_every"] = 1
    stats, res = xg.serve(reqs, 2e6, 512 * MB, host_budget_bytes=256 * MB, collect=True)
    assert stats["dumps"] == sum(r["nblocks"] for r in reqs)
    stats_p, res_p = xg.serve(reqs, 2e6, 512 * MB, mode=xg.XGPU_SERVE_PLAIN_SERIAL,
                              host_budget_bytes=256 * MB, collect=True)
    assert stats_p["admitted_peak"] == 1
    for r, a, b in zip(reqs, res, res_p):
        assert np.array_equal(a, b)
        assert np.array_equal(a, expected(oracle_mod, r))


def test_rejects_bad_streams(xg):
    reqs = requests(3)
    reqs[1]["arrival_s"], reqs[2]["arrival_s"] = 0.5, 0.1   # unsorted
    with pytest.raises(xg.XGPUError):
        xg.serve(reqs, 2e6, 64 * MB, host_budget_bytes=64 * MB)
    with pytest.raises(xg.XGPUError):
        xg.serve(requests(2), 0.0, 64 * MB, host_budget_bytes=64 * MB)
