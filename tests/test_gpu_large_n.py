"""Station counts from 513 to 1024, as the batched and served configurations
draw them (N log-uniform in [32, 1024]): every tensor-core kernel, the plain
dp4a engine, packed input, batches that mix N=1024 with N=32, and a served
stream with large requests among small ones -- each bit-exact with the
oracle's int64 sums (xGPU omp_xengine.c:41-89, which puts no limit on N).

At N=1024 a channel has 4096 Gram rows: 32 single-CTA row tiles (528 tile
pairs per channel) or 16 CTA-pair row tiles (136 tile pairs), and the int64
offsets of a channel's rows pass 2^22 words; the partial last tiles of
N = 528, 784 and 928 leave rows past N that must not be written.

Also here: the plain FP32 engine on sums far past 2^24, where float sums
round.  xGPU's float engine adds each sample's two exact products with one
rounding (omp_xengine.c:24-28); the FP32 engine does the same in time order,
so it equals the oracle's restatement of that engine bit for bit (tolerance
0, inside the 1e-6 relative the X-engine's FP32 path is held to), and its
distance from the exact int64 sums is the reference's own.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LARGE_N = [528, 640, 784, 928, 1024]


def shape_for(n):
    """(channels, samples) small enough for the oracle, with partial stages."""
    return (2, 640) if n <= 784 else (1, 896)


@pytest.mark.parametrize("n", LARGE_N)
@pytest.mark.parametrize("tune", [(1, 0, 1), (1, 0, 0), (3, 0, 1), (2, 37, 0)],
                         ids=["pair", "single", "pair-split3", "single-split2-grid37"])
def test_tensor_kernels_at_large_n(xg, oracle_mod, n, tune):
    f, t = shape_for(n)
    x = oracle_mod.gaussian_input(n, f, t, seed=n + 13 * tune[0] + tune[2], sigma=30.0)
    exact = oracle_mod.xengine_i64(x, n, f, t)
    with xg.Correlator(n, f, t, ntimepipe=16, engine="tensor") as c:
        c.tune(*tune)
        c.set_input(x)
        c.run(xg.SYNCOP_SYNC_COMPUTE)     # stores into the cleared buffer
        assert np.array_equal(c.dump_int64(), exact)
        c.set_input(x)
        c.run(xg.SYNCOP_DUMP)             # adds (bulk reduce-add)
        assert np.array_equal(c.dump_int64(), 2 * exact)
        got = c.output_view()[: c.info.matLength * 2]
        assert np.array_equal(got, (2 * exact).astype(np.int32))


@pytest.mark.parametrize("n", [528, 1024])
def test_plain_dp4a_at_large_n(xg, oracle_mod, n):
    t = 512
    x = oracle_mod.gaussian_input(n, 1, t, seed=n, sigma=40.0)
    with xg.Correlator(n, 1, t, engine="plain") as c:
        c.set_input(x)
        c.run(xg.SYNCOP_DUMP)
        assert np.array_equal(c.dump_int64(), oracle_mod.xengine_i64(x, n, 1, t))


@pytest.mark.parametrize("n,tune", [(1024, (1, 0, 1)), (928, (1, 0, 1)), (1024, (1, 0, 0))])
def test_packed4_at_large_n(xg, oracle_mod, n, tune):
    """Packed 4+4-bit input: expanded inside the CTA-pair kernel, or by the
    pre-pass for single CTAs."""
    f, t = 1, 512
    packed = oracle_mod.generate(t * f * n * 2, 1, n + 7)
    with xg.Correlator(n, f, t, ntimepipe=16, engine="tensor", input_format="packed4") as c:
        c.tune(*tune)
        c.set_input(packed)
        c.run(xg.SYNCOP_DUMP)
        got = c.dump_int64()
    assert np.array_equal(got, oracle_mod.xengine_i64(oracle_mod.unpack4(packed), n, f, t))


def test_register_tile_order_at_n1024(xg, oracle_mod):
    n, f, t = 1024, 1, 256
    x = oracle_mod.gaussian_input(n, f, t, seed=99, sigma=20.0)
    with xg.Correlator(n, f, t, engine="tensor", order="rt", output="float32") as c:
        c.set_input(x)
        c.run(xg.SYNCOP_DUMP)
        got = c.output_view()[: c.info.matLength * 2].copy()   # the view dies with the context
    exact = oracle_mod.xengine_i64(x, n, f, t).astype(np.float32)
    assert np.array_equal(got, oracle_mod.tri_to_order(exact, n, f, 3000))


MIXED = [(1024, 2, 512), (32, 5, 256), (928, 1, 768), (48, 3, 1024), (528, 2, 256),
         (32, 64, 256), (784, 1, 1280)]


@pytest.mark.parametrize("autotune,graph,pair", [(False, False, False), (False, False, True),
                                                 (True, True, False), (False, True, True)])
def test_batch_mixing_n1024_and_n32(xg, oracle_mod, autotune, graph, pair):
    """One persistent launch over jobs from N=32 to N=1024; each job equals
    the plain engine run on its own and the oracle."""
    import torch
    jobs, keep = [], []
    for q, (n, f, t) in enumerate(MIXED):
        x = oracle_mod.gaussian_input(n, f, t, seed=700 + q, sigma=4.0 + 4 * q)
        xd = torch.from_numpy(x).cuda()
        st = torch.full((xg.state_elems(n, f),), 7, dtype=torch.int64, device="cuda")
        jobs.append({"input": xd.data_ptr(), "state": st.data_ptr(), "nstation": n,
                     "nfrequency": f, "ntime": t})
        keep.append((x, xd, st, n, f, t))
    with xg.Batch(jobs, autotune=autotune, graph=graph, pair=pair) as b:
        b.run()
        b.sync()
        for x, xd, st, n, f, t in keep:
            got = st.cpu().numpy()
            assert np.array_equal(got, oracle_mod.xengine_i64(x, n, f, t)), (n, f, t)
            if n >= 512:
                with xg.Correlator(n, f, t, ntimepipe=16, engine="plain") as c:
                    c.run_device(xd.data_ptr(), xg.SYNCOP_SYNC_COMPUTE)
                    assert np.array_equal(got, c.dump_int64()), (n, f, t)


def test_served_mix_with_large_requests(xg, oracle_mod):
    """Continuous batching with N=1024 and N=640 requests among small ones:
    each result equals the oracle and the same request served alone."""
    MB = 1 << 20
    rng = np.random.default_rng(11)
    arrivals = np.sort(rng.uniform(0, 0.05, 8))
    reqs = [{"nstation": int(rng.choice([16, 32, 64, 128])), "nfrequency": int(rng.integers(1, 4)),
             "ntime": int(256 * rng.integers(1, 4)), "nblocks": int(rng.integers(2, 5)),
             "seed": 2000 + q, "sigma": float(rng.uniform(4, 32)), "arrival_s": float(arrivals[q])}
            for q in range(8)]
    reqs[2].update(nstation=1024, nfrequency=1, ntime=256, nblocks=3)
    reqs[5].update(nstation=640, nfrequency=2, ntime=512, nblocks=2)

    def expected(r):
        n, f, t = r["nstation"], r["nfrequency"], r["ntime"]
        acc = np.zeros(xg.state_elems(n, f), dtype=np.int64)
        for b in range(r["nblocks"]):
            x = oracle_mod.serve_block_input(n, f, t, r["seed"], r["sigma"], b)
            oracle_mod.xengine_i64(x, n, f, t, acc=acc)
        return acc.astype(np.int32)

    stats, res = xg.serve(reqs, 2e6, 2048 * MB, host_budget_bytes=512 * MB, collect=True)
    assert stats["jobs"] == len(reqs) and stats["dumps"] == len(reqs)
    assert stats["admitted_peak"] >= 2
    for r, got in zip(reqs, res):
        assert np.array_equal(got, expected(r)), r
    alone = dict(reqs[2], arrival_s=0.0)
    _, res1 = xg.serve([alone], 2e6, 2048 * MB, host_budget_bytes=512 * MB, collect=True)
    assert np.array_equal(res1[0], res[2])


@pytest.mark.parametrize("calls", [1, 4])
def test_fp32_engine_past_2_24_equals_reference_float_engine(xg, oracle_mod, calls):
    """N=32, F=2, 32768 samples at sigma 40: auto-correlation sums reach 1e8,
    where float sums round.  One call of 32768 samples, or four of 8192 (the
    integration continues the buffer's sums), equals the reference's float
    arithmetic bit for bit; both sit the same distance from the exact sums."""
    n, f, t = 32, 2, 32768
    x = oracle_mod.gaussian_input(n, f, t, seed=5, sigma=40.0)
    tc = t // calls
    with xg.Correlator(n, f, tc, engine="plain", compute="fp32", output="float32") as c:
        for q in range(calls):
            c.set_input(x[q * tc * f * n * 4:(q + 1) * tc * f * n * 4])
            c.run(xg.SYNCOP_DUMP if q == calls - 1 else xg.SYNCOP_SYNC_TRANSFER)
        got = c.output_view()[: c.info.matLength * 2].copy()
    ref = oracle_mod.xengine_f32(x, n, f, t)
    exact = oracle_mod.xengine_i64(x, n, f, t).astype(np.float64)
    assert np.abs(exact).max() > 2 ** 26          # far past exact float integers
    assert not np.array_equal(ref.astype(np.float64), exact)   # the reference rounds here
    assert np.array_equal(got, ref)                # max relative error 0 (tolerance 1e-6)


# The largest station counts xgpuInitEx accepts (up to 8192): at N=8192 a
# channel has 32768 Gram rows, 8256 CTA-pair tile pairs (32896 single-CTA
# ones, and as many 32x32-station blocks for the plain engine), and its
# int64 buffer holds 268 million words, so row offsets pass 2^28.  One
# channel and a few stages keep the oracle in seconds.
@pytest.mark.parametrize("n", [2048, 4096, 8192])
@pytest.mark.parametrize("tune", [(1, 0, 1), (1, 0, 0)], ids=["pair", "single"])
def test_tensor_kernels_at_the_largest_n(xg, oracle_mod, n, tune):
    f, t = 1, 144    # a partial second stage
    x = oracle_mod.gaussian_input(n, f, t, seed=n + tune[2], sigma=30.0)
    exact = oracle_mod.xengine_i64(x, n, f, t)
    with xg.Correlator(n, f, t, ntimepipe=16, engine="tensor") as c:
        c.tune(*tune)
        c.set_input(x)
        c.run(xg.SYNCOP_SYNC_COMPUTE)     # stores into the cleared buffer
        c.set_input(x)
        c.run(xg.SYNCOP_DUMP)             # adds
        assert np.array_equal(c.dump_int64(), 2 * exact)
        got = c.output_view()[: c.info.matLength * 2]
        assert np.array_equal(got, (2 * exact).astype(np.int32))


@pytest.mark.parametrize("n,compute", [(8192, "int8"), (2048, "fp32")])
def test_plain_engines_at_the_largest_n(xg, oracle_mod, n, compute):
    t = 64
    x = oracle_mod.gaussian_input(n, 1, t, seed=n + 1, sigma=20.0)
    exact = oracle_mod.xengine_i64(x, n, 1, t)
    output = "int32" if compute == "int8" else "float32"
    with xg.Correlator(n, 1, t, ntimepipe=16, engine="plain", compute=compute,
                       output=output) as c:
        c.set_input(x)
        c.run(xg.SYNCOP_DUMP)
        got = c.output_view()[: c.info.matLength * 2]
        # int8 sums are exact; FP32 sums of 64 samples stay below 2^24, so exact too
        assert np.array_equal(got, exact.astype(got.dtype))


# The largest channel count xgpuInitEx accepts, 65535: the plain engines
# launch one grid row per channel (gridDim.y at its limit), the tensor-core
# kernels count 65535 channels' tiles as work items.
@pytest.mark.parametrize("engine,compute,tune", [
    ("tensor", "int8", (1, 0, 1)), ("tensor", "int8", (1, 0, 0)),
    ("plain", "int8", None), ("plain", "fp32", None)],
    ids=["pair", "single", "dp4a", "fp32"])
def test_the_largest_channel_count(xg, oracle_mod, engine, compute, tune):
    n, f, t = 16, 65535, 32
    x = oracle_mod.gaussian_input(n, f, t, seed=5, sigma=20.0)
    exact = oracle_mod.xengine_i64(x, n, f, t)
    output = "int32" if compute == "int8" else "float32"
    with xg.Correlator(n, f, t, ntimepipe=16, engine=engine, compute=compute,
                       output=output) as c:
        if tune:
            c.tune(*tune)
        c.set_input(x)
        c.run(xg.SYNCOP_DUMP)
        got = c.output_view()[: c.info.matLength * 2]
        assert np.array_equal(got, exact.astype(got.dtype))
