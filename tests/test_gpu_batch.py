"""Time splits, autotuning and batches of uneven subarrays (tensor-core engine).

Each batch job is compared with the plain CUDA-core engine run job by job on
the same input (and with the oracle), bit for bit, as the batched-subarray
configuration requires: all jobs go into one persistent launch whose CTAs
take work items from a global queue, optionally replayed from a CUDA graph.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def plain_job_by_job(xg, x_dev, n, f, t):
    with xg.Correlator(n, f, t, ntimepipe=16, engine="plain") as c:
        c.run_device(x_dev.data_ptr(), xg.SYNCOP_SYNC_COMPUTE)
        return c.dump_int64()


@pytest.mark.parametrize("pair", [0, 1])
@pytest.mark.parametrize("ksplit", [2, 3, 8])
def test_time_splits_are_exact(xg, oracle_mod, ksplit, pair):
    n, f, t = 64, 3, 1024 + 384
    x = oracle_mod.gaussian_input(n, f, t, seed=ksplit, sigma=30.0)
    with xg.Correlator(n, f, t, ntimepipe=128, engine="tensor") as c:
        c.tune(ksplit, 0, pair)
        c.set_input(x)
        c.run(xg.SYNCOP_SYNC_COMPUTE)        # first call after init stores (buffer zero)
        c.set_input(x)
        c.run(xg.SYNCOP_DUMP)                # second call adds
        got = c.dump_int64()
    assert np.array_equal(got, 2 * oracle_mod.xengine_i64(x, n, f, t))


def test_context_autotune_keeps_results(xg, oracle_mod):
    n, f, t = 128, 4, 2048
    x = oracle_mod.gaussian_input(n, f, t, seed=9)
    with xg.Correlator(n, f, t, engine="tensor") as c:
        c.set_input(x)
        c.run(xg.SYNCOP_SYNC_COMPUTE)
        c.tune(0)                             # autotune must not touch the integration
        c.set_input(x)
        c.run(xg.SYNCOP_DUMP)
        got = c.dump_int64()
    assert np.array_equal(got, 2 * oracle_mod.xengine_i64(x, n, f, t))


@pytest.mark.parametrize("n,f,t", [(16, 2, 64), (32, 3, 256), (48, 2, 128), (64, 5, 1024),
                                   (80, 1, 512), (112, 2, 384), (128, 4, 2048), (256, 10, 1024),
                                   (320, 2, 768), (512, 3, 8192)])
def test_pair_kernel_parity(xg, oracle_mod, n, f, t):
    """CTA-pair kernel (256x256 tiles): bit-exact, store and accumulate paths."""
    x = oracle_mod.gaussian_input(n, f, t, seed=n * 7 + t, sigma=24.0)
    exact = oracle_mod.xengine_i64(x, n, f, t)
    with xg.Correlator(n, f, t, ntimepipe=16, engine="tensor") as c:
        c.tune(1, 0, 1)
        c.set_input(x)
        c.run(xg.SYNCOP_SYNC_COMPUTE)    # stores into the cleared buffer
        assert np.array_equal(c.dump_int64(), exact)
        c.set_input(x)
        c.run(xg.SYNCOP_DUMP)            # adds (bulk reduce-add)
        assert np.array_equal(c.dump_int64(), 2 * exact)
        got = c.output_view()[: c.info.matLength * 2]
        assert np.array_equal(got, (2 * exact).astype(np.int32))


@pytest.mark.parametrize("n,f,t,grid", [(256, 10, 1024, 0), (64, 3, 1024 + 384, 7), (48, 2, 128, 5),
                                        (128, 5, 2048, 148), (16, 1, 64, 0)])
def test_stream_k_shares_are_exact(xg, oracle_mod, n, f, t, grid):
    """Stream-K: CTAs take equal shares of all (tile, step) pairs; tiles cut
    between CTAs add up exactly.  The first call after a clear stores (plain
    tiles), the following ones add with stream-K shares."""
    x = oracle_mod.gaussian_input(n, f, t, seed=3 * n + t, sigma=28.0)
    exact = oracle_mod.xengine_i64(x, n, f, t)
    with xg.Correlator(n, f, t, ntimepipe=16, engine="tensor") as c:
        c.tune(1, grid, 2)
        c.set_input(x)
        for _ in range(3):
            c.run(xg.SYNCOP_SYNC_COMPUTE)
        assert np.array_equal(c.dump_int64(), 3 * exact)


def test_pair_kernel_small_grid_and_autotune(xg, oracle_mod):
    n, f, t = 256, 6, 2048
    x = oracle_mod.gaussian_input(n, f, t, seed=77)
    exact = oracle_mod.xengine_i64(x, n, f, t)
    with xg.Correlator(n, f, t, engine="tensor") as c:
        c.tune(3, 10, 1)                  # 5 clusters walk all items
        assert c.tuning() == {"ksplit": 3, "grid": 10, "pair": 1}
        c.set_input(x)
        c.run(xg.SYNCOP_SYNC_COMPUTE)
        assert np.array_equal(c.dump_int64(), exact)
        c.tune(0)                         # autotune over both kernels
        got = c.tuning()
        assert got["ksplit"] >= 1 and got["pair"] in (0, 1, 2) and got["grid"] >= 0
        c.tune(got["ksplit"], got["grid"], got["pair"])   # a kept choice round-trips
        assert c.tuning() == got
        c.clear()
        c.set_input(x)
        c.run(xg.SYNCOP_SYNC_COMPUTE)
        assert np.array_equal(c.dump_int64(), exact)


def make_jobs(torch, oracle_mod, shapes, seed0=100):
    jobs, keep = [], []
    for q, (n, f, t) in enumerate(shapes):
        x = oracle_mod.gaussian_input(n, f, t, seed=seed0 + q, sigma=4.0 + 4 * (q % 8))
        xd = torch.from_numpy(x).cuda()
        st = torch.full((f * n * (n + 1) // 2 * 8,), 7, dtype=torch.int64, device="cuda")
        jobs.append({"input": xd.data_ptr(), "state": st.data_ptr(), "nstation": n,
                     "nfrequency": f, "ntime": t})
        keep.append((x, xd, st, n, f, t))
    return jobs, keep


UNEVEN = [(32, 5, 256), (48, 1, 512), (64, 7, 2304), (96, 2, 768), (128, 3, 256), (160, 1, 1280),
          (16, 9, 4096), (256, 2, 1024), (80, 4, 8192), (32, 64, 256)]


@pytest.mark.parametrize("autotune,graph,pair", [(False, False, False), (False, False, True),
                                                 (False, True, True), (True, False, False),
                                                 (True, True, False)])
def test_batch_matches_plain_job_by_job(xg, oracle_mod, autotune, graph, pair):
    import torch
    jobs, keep = make_jobs(torch, oracle_mod, UNEVEN)
    with xg.Batch(jobs, autotune=autotune, graph=graph, pair=pair) as b:
        b.run()
        b.sync()
        info = b.info()
        assert info["work_items"] > 0 and info["grid"] > 0
        for x, xd, st, n, f, t in keep:
            got = st.cpu().numpy()
            assert np.array_equal(got, plain_job_by_job(xg, xd, n, f, t)), (n, f, t)
            assert np.array_equal(got, oracle_mod.xengine_i64(x, n, f, t)), (n, f, t)
        # a second run replaces (accumulate = 0) rather than adds
        b.run()
        b.sync()
        for x, xd, st, n, f, t in keep[:3]:
            assert np.array_equal(st.cpu().numpy(), oracle_mod.xengine_i64(x, n, f, t))


def test_batch_accumulates(xg, oracle_mod):
    import torch
    shapes = [(64, 2, 512), (32, 3, 1024), (112, 1, 256)]
    jobs, keep = make_jobs(torch, oracle_mod, shapes, seed0=300)
    for j, (x, xd, st, n, f, t) in zip(jobs, keep):
        st.zero_()
        j["accumulate"] = 1
    with xg.Batch(jobs, graph=True, pair=True) as b:
        for _ in range(3):
            b.run()
        b.sync()
    for x, xd, st, n, f, t in keep:
        assert np.array_equal(st.cpu().numpy(), 3 * oracle_mod.xengine_i64(x, n, f, t))


def test_batch_rejects_bad_jobs(xg):
    import torch
    x = torch.zeros(1024, dtype=torch.int8, device="cuda")
    st = torch.zeros(1024, dtype=torch.int64, device="cuda")
    bad = [{"input": x.data_ptr(), "state": st.data_ptr(), "nstation": 24, "nfrequency": 1,
            "ntime": 16},
           {"input": x.data_ptr() + 1, "state": st.data_ptr(), "nstation": 16, "nfrequency": 1,
            "ntime": 16}]
    for j in bad:
        with pytest.raises(xg.XGPUError):
            xg.Batch([j])
