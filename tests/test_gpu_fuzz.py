"""Seeded random configurations through the C ABI, each compared bit for bit
with the oracle: station counts that leave partial 32-station blocks,
channel and sample counts that leave partial tiles and pipeline stages,
every engine and tensor-core kernel choice, time splits, grids, input
formats, accumulating call sequences with each syncOp, and device-resident
input.  The draw is fixed (seed below), so a failure reproduces by its case
number.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEED = 20261203
NCASES = 40


def draw_cases():
    rng = np.random.default_rng(SEED)
    cases = []
    for q in range(NCASES):
        n = int(rng.choice([16, 32, 48, 64, 80, 112, 144, 176, 208, 256]))
        f = int(rng.integers(1, 7))
        t = int(16 * rng.integers(1, 160))                  # up to 2544 samples
        engine = str(rng.choice(["tensor", "tensor", "tensor", "plain", "fp32"]))
        fmt = str(rng.choice(["int8", "int8", "packed4", "dp4a_swizzled", "block32"]))
        calls = int(rng.integers(1, 4))
        device = bool(rng.integers(0, 2)) and fmt == "int8"
        tune = None
        if engine == "tensor":
            tune = (int(rng.choice([1, 1, 2, 3, 5])), int(rng.choice([0, 0, 7, 24, 37, 148])),
                    int(rng.choice([0, 1, 2])))
        cases.append((q, n, f, t, engine, fmt, calls, device, tune))
    return cases


def make_input(oracle_mod, n, f, t, fmt, seed, sigma):
    """(bytes to feed, int8 samples they stand for)."""
    if fmt == "packed4":
        packed = oracle_mod.generate(t * f * n * 2, 1, seed)
        return packed, oracle_mod.unpack4(packed)
    x = oracle_mod.gaussian_input(n, f, t, seed=seed, sigma=sigma)
    if fmt == "dp4a_swizzled":
        return oracle_mod.swizzle(x, n, f, t), x
    if fmt == "block32":
        return oracle_mod.block32(x), x
    return x, x


@pytest.mark.parametrize("case", draw_cases(), ids=lambda c: f"case{c[0]}")
def test_random_configuration(xg, oracle_mod, case):
    import torch
    q, n, f, t, engine, fmt, calls, device, tune = case
    compute = "fp32" if engine == "fp32" else "int8"
    eng = "plain" if engine in ("plain", "fp32") else "tensor"
    output = "float32" if compute == "fp32" else "int32"
    # FP32 sums stay integers below 2^24 (exact) at sigma 8; the integer
    # engines get wider inputs, full range at times
    sigma = 8.0 if compute == "fp32" else float(8 + (37 * q) % 100)
    feeds = [make_input(oracle_mod, n, f, t, fmt, 1000 * q + k, sigma) for k in range(calls)]
    exact = sum(oracle_mod.xengine_i64(x, n, f, t) for _, x in feeds)
    syncs = [xg.SYNCOP_SYNC_TRANSFER, xg.SYNCOP_SYNC_COMPUTE, xg.SYNCOP_NONE]
    with xg.Correlator(n, f, t, ntimepipe=16, engine=eng, compute=compute, output=output,
                       order="tri", input_format=fmt) as c:
        if tune is not None:
            c.tune(*tune)
        keep = []
        for k, (feed, _) in enumerate(feeds):
            if device:
                d = torch.from_numpy(np.ascontiguousarray(feed)).cuda()
                torch.cuda.synchronize()
                keep.append(d)
                c.run_device(d.data_ptr(), syncs[k % 3])
            else:
                c.set_input(feed)
                # the host buffer is rewritten by the next set_input: wait for its copy
                c.run(xg.SYNCOP_SYNC_TRANSFER if k < calls - 1 else xg.SYNCOP_DUMP)
        got = c.dump()
        if compute == "int8":
            assert np.array_equal(c.dump_int64(), exact), case
            assert np.array_equal(got, exact.astype(np.int32)), case
        else:
            # float sums of integers are exact below 2^24
            assert np.abs(exact).max() < 2**24
            assert np.array_equal(got, exact.astype(np.float32)), case


def draw_batches():
    rng = np.random.default_rng(SEED + 1)
    out = []
    for q in range(6):
        njobs = int(rng.integers(3, 16))
        jobs = []
        for k in range(njobs):
            n = int(rng.choice([16, 32, 48, 80, 128, 176, 256, 384]))
            f = int(rng.integers(1, 9))
            t = int(256 * rng.integers(1, 9)) if rng.integers(0, 2) else int(16 * rng.integers(1, 40))
            jobs.append((n, f, t, int(rng.integers(0, 2))))
        flags = (bool(rng.integers(0, 2)), bool(rng.integers(0, 2)), bool(rng.integers(0, 2)))
        runs = int(rng.integers(1, 4))
        out.append((q, jobs, flags, runs))
    return out


@pytest.mark.parametrize("batch", draw_batches(), ids=lambda b: f"batch{b[0]}")
def test_random_batch(xg, oracle_mod, batch):
    """A random batch of uneven subarrays (some accumulating, some replacing
    their buffer each run), with random autotune / graph / CTA-pair flags, run
    one to three times: every job's int64 buffer equals the oracle."""
    import torch
    q, shapes, (autotune, graph, pair), runs = batch
    jobs, keep = [], []
    for k, (n, f, t, acc) in enumerate(shapes):
        x = oracle_mod.gaussian_input(n, f, t, seed=7000 + 100 * q + k, sigma=float(4 + 7 * k % 40))
        xd = torch.from_numpy(x).cuda()
        st = torch.zeros(f * n * (n + 1) // 2 * 8, dtype=torch.int64, device="cuda")
        jobs.append({"input": xd.data_ptr(), "state": st.data_ptr(), "nstation": n,
                     "nfrequency": f, "ntime": t, "accumulate": acc})
        keep.append((x, xd, st, n, f, t, acc))
    torch.cuda.synchronize()
    with xg.Batch(jobs, autotune=autotune, graph=graph, pair=pair) as b:
        for _ in range(runs):
            b.run()
        b.sync()
    for x, xd, st, n, f, t, acc in keep:
        want = (runs if acc else 1) * oracle_mod.xengine_i64(x, n, f, t)
        assert np.array_equal(st.cpu().numpy(), want), (n, f, t, acc)
