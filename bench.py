#!/usr/bin/env python
"""X-engine benchmark: libxgpu.so on B200 vs the reference's CPU engine.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one GPU; with --gpus N every rank runs it on its own channels, so
per-GPU work is fixed: weak scaling, no collective): xGPU's default build
shape, NSTATION=256, NPOL=2, NFREQUENCY=10, NTIME=1024, Gaussian int8 samples
(sigma 16, seeded).  A step is one xgpuCudaXengine call's worth of samples
correlated by the tcgen05 int8 engine into the int64 integration buffer.

* value      -- X-engine TOPS (16*F*T*N(N+1) ops per step, the flop count of
                xGPU kernel.cuh:419) with the input resident in HBM, K steps
                timed with CUDA events on the engine's stream, the input
                rotating over buffers larger than L2 in total.
* e2e        -- the same metric through the reference-facing call sequence
                with host buffers: xgpuClearDeviceIntegrationBuffer +
                xgpuCudaXengine(SYNCOP_DUMP), i.e. pinned host -> device copy,
                correlation, device-side formatting and the device -> host
                dump inside every step (one integration of one dump).
* detail     -- the plain CUDA-core dp4a and FP32 engines on the same
                workload, and the tensor engine at NSTATION=512, NFREQUENCY=256,
                NTIME=8192 (one block of the large-array configuration).
* cpu_baseline / --impl reference -- the reference's own xgpuOmpXengine
                (src/omp_xengine.c built with -fopenmp under oracle/_ref, DP4A
                variant) on all host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "X-engine TOPS: int8-TC vs plain @N=256/512, bit-exact; served p50/p99 dump ms"
N, F, T = 256, 10, 1024
N3, F3, T3 = 512, 256, 8192
SIGMA = 16.0
L2_BYTES = 126 * 1024 * 1024


def ops(n, f, t):
    return 16.0 * f * t * n * (n + 1)


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh), "MEASURED_PEAKS.json"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback (no MEASURED_PEAKS.json)"


def read_profile_traffic(pair):
    """Per-launch DRAM bytes of the headline kernel from its committed ncu summary."""
    name = "xengine_tc2_kernel_n256.md" if pair == 1 else "xengine_tc_kernel_n256.md"
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a run."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.fh = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.fh.seek(0)
        rows = [r.split(",") for r in self.fh.read().splitlines() if r.strip()]
        os.unlink(self.fh.name)
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                clk, mx, pw = float(r[1]), float(r[2]), float(r[3])
            except (ValueError, IndexError):
                continue
            smax = max(smax, mx)
            if pw > 200.0:  # under load
                sm.append(clk)
            for nm, v in zip(names, r[5:9]):
                if "Active" in v and "Not" not in v:
                    reasons.add(nm)
        if not sm:
            sm = [float(r[1]) for r in rows if len(r) > 1 and r[1].strip().replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=180),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


TUNING = {}   # (engine, n, f, t) -> the tensor engine's autotuned setting
FOLDS = {}    # (engine, n, f, t) -> word-buffer folds inside the timed region
WORD_MAX_SAMPLES = 65535


def word_folds(tuning, t, warmup, steps):
    """Launches of the library's fold kernel inside a timed run of `steps`
    calls after `warmup`: CTA-pair launches whose items take at most 8 stages
    of 128 samples put their sums into a word buffer (the first call of the
    integration stores its words, the others add), folded before it would
    pass 65535 samples and once at the closing flush."""
    if not tuning or not tuning["pair"]:
        return 0
    stages = -(-t // 128)
    ksplit = max(1, min(tuning["ksplit"], stages))
    if -(-stages // ksplit) > 8:
        return 0
    samples, folds = 0, 0
    for k in range(warmup + steps):
        if samples + t > WORD_MAX_SAMPLES:
            folds += k >= warmup
            samples = 0
        samples += t
    return folds + (samples > 0)


def device_engine_ms(xg, torch, engine, compute, n, f, t, steps, warmup, world, seed=1,
                     sigma=SIGMA, min_rotate_bytes=2 * L2_BYTES, max_bufs=16, tune=None):
    """Average ms per xgpuCudaXengineDevice call (input resident in HBM).  The
    tensor engine's time splits and grid come from the library's autotuner, or
    from `tune` = (ksplit, grid, pair)."""
    c = xg.Correlator(n, f, t, engine=engine, compute=compute, output="int32", order="tri",
                      device=torch.cuda.current_device())
    if engine == "tensor":
        c.tune(*tune) if tune else c.tune(0)   # kernel, time splits and grid chosen by timing
    # The timing events go on the context's own stream, where consecutive
    # accumulating calls may overlap (programmatic dependent launch).
    stream = torch.cuda.ExternalStream(c.stream)
    nbytes = int(c.info.vecLength) * 2
    nbuf = max(1, min(max_bufs, -(-min_rotate_bytes // nbytes)))
    bufs = []
    for q in range(nbuf):
        b = torch.empty(nbytes, dtype=torch.int8, device="cuda")
        xg.generate_device(b.data_ptr(), nbytes, 0, seed + q, sigma, torch.cuda.current_device())
        bufs.append(b)
    for k in range(warmup):
        c.run_device(bufs[k % nbuf].data_ptr(), xg.SYNCOP_NONE)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(steps):
        c.run_device(bufs[k % nbuf].data_ptr(), xg.SYNCOP_NONE)
    # The integration is complete on the device when the region ends: sums
    # that the CTA-pair kernel keeps in its short-term word buffer are added
    # into the int64 buffer inside the timed region.
    c.flush()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms = e0.elapsed_time(e1) / steps
    TUNING[(engine, n, f, t)] = c.tuning() if engine == "tensor" else None
    FOLDS[(engine, n, f, t)] = word_folds(TUNING[(engine, n, f, t)], t, warmup, steps)
    c.close()
    del bufs
    torch.cuda.empty_cache()
    return ms, nbuf * nbytes


def e2e_ms(xg, oracle, n, f, t, steps, warmup, device):
    """Wall ms per integration through xgpuCudaXengine with pinned host buffers."""
    c = xg.Correlator(n, f, t, engine="tensor", output="int32", order="tri", device=device)
    x = oracle.gaussian_input(n, f, t, seed=1, sigma=SIGMA)
    c.set_input(x)
    for _ in range(warmup):
        c.clear()
        c.run(xg.SYNCOP_DUMP)
    t0 = time.perf_counter()
    for _ in range(steps):
        c.clear()
        c.run(xg.SYNCOP_DUMP)
    ms = (time.perf_counter() - t0) * 1e3 / steps
    h2d = int(c.info.vecLength) * 2
    d2h = int(c.info.matLength) * 8
    # the last dump must equal the oracle
    got = c.output_view()[: c.info.matLength * 2]
    ok = bool((got == oracle.xengine_i64(x, n, f, t).astype("int32")).all())
    c.close()
    return ms, h2d, d2h, ok


def e2e_streaming(xg, oracle, n, f, t, calls, reps, device):
    """The reference driver's own call pattern (cuda_correlator.c:196-230,
    defaults :46-47): an integration of `calls` xgpuCudaXengine calls over host
    buffers, SYNCOP_SYNC_TRANSFER on all but the last, SYNCOP_DUMP on the last
    (copy of each call's input under the previous call's correlation, one dump
    per integration).  Host wall clock over `reps` integrations."""
    c = xg.Correlator(n, f, t, engine="tensor", output="int32", order="tri", device=device)
    x = oracle.gaussian_input(n, f, t, seed=1, sigma=SIGMA)
    c.set_input(x)

    def integration():
        c.clear()
        for q in range(calls):
            c.run(xg.SYNCOP_DUMP if q == calls - 1 else xg.SYNCOP_SYNC_TRANSFER)
    for _ in range(2):
        integration()
    t0 = time.perf_counter()
    for _ in range(reps):
        integration()
    ms = (time.perf_counter() - t0) * 1e3 / reps
    got = c.output_view()[: c.info.matLength * 2]
    ok = bool((got == (calls * oracle.xengine_i64(x, n, f, t)).astype("int32")).all())
    h2d = calls * int(c.info.vecLength) * 2
    d2h = int(c.info.matLength) * 8
    c.close()
    return {"calls_per_integration": calls, "integrations": reps,
            "ms_per_call": ms / calls, "tops": calls * ops(n, f, t) / (ms * 1e-3) / 1e12,
            "h2d_bytes_per_integration": h2d, "d2h_bytes_per_integration": d2h,
            "host_link_gbs": (h2d + d2h) / (ms * 1e-3) / 1e9, "bit_exact_vs_oracle": ok,
            "syncops": "SYNCOP_SYNC_TRANSFER x (calls-1), SYNCOP_DUMP"}


def fp32_engine_long(xg, oracle, device, n=32, f=2, t=32768, sigma=40.0):
    """The plain FP32 engine where float sums round (autos ~1e8 > 2^24): its
    relative error against the reference's float arithmetic (the oracle's
    restatement of omp_xengine.c:24-28; the stated tolerance is 1e-6) and, for
    context, both against the exact int64 sums."""
    import numpy as np
    x = oracle.gaussian_input(n, f, t, seed=5, sigma=sigma)
    with xg.Correlator(n, f, t, engine="plain", compute="fp32", output="float32",
                       device=device) as c:
        c.set_input(x)
        c.run(xg.SYNCOP_DUMP)
        got = c.output_view()[: c.info.matLength * 2].astype(np.float64)
    ref = oracle.xengine_f32(x, n, f, t).astype(np.float64)
    exact = oracle.xengine_i64(x, n, f, t).astype(np.float64)
    nz = ref != 0
    nze = exact != 0
    return {"nstation": n, "nfrequency": f, "ntime": t, "sigma": sigma,
            "max_abs_sum": float(np.abs(exact).max()),
            "max_rel_err_vs_reference_float": float((np.abs(got - ref)[nz] / np.abs(ref[nz])).max()),
            "tolerance": 1e-6,
            "max_rel_err_vs_exact": float((np.abs(got - exact)[nze] / np.abs(exact[nze])).max()),
            "reference_float_max_rel_err_vs_exact":
                float((np.abs(ref - exact)[nze] / np.abs(exact[nze])).max())}


def float_output_error(xg, oracle, n, f, t, sigma, device):
    """Float32-output mode against the FP64 host oracle: one call, dumped as
    float32 (the exact int64 sums are rounded once, at dump).  Returns the max
    relative error over non-zero elements (bound 2^-24) and the largest |sum|
    (beyond 2^24 the rounding shows)."""
    import numpy as np
    x = oracle.gaussian_input(n, f, t, seed=1, sigma=sigma)
    c = xg.Correlator(n, f, t, ntimepipe=128, engine="tensor", output="float32", order="tri",
                      device=device)
    c.set_input(x)
    c.run(xg.SYNCOP_DUMP)
    got = c.output_view()[: c.info.matLength * 2].astype(np.float64)
    c.close()
    exact = oracle.xengine_i64(x, n, f, t).astype(np.float64)
    nz = exact != 0
    rel = np.abs(got[nz] - exact[nz]) / np.abs(exact[nz])
    return {"nstation": n, "nfrequency": f, "ntime": t, "sigma": sigma,
            "max_abs_sum": float(np.abs(exact).max()),
            "max_rel_err_vs_fp64": float(rel.max()), "bound": 2.0 ** -24,
            "zeros_exact": bool(not got[~nz].any())}


def uneven_subarray_shapes(seed=3, k=96):
    """96 subarrays: N log-uniform in [32,1024] rounded to 16, F uniform in
    [1,64], T a uniform multiple of 256 in [256,8192], sigma uniform in [4,32]."""
    import numpy as np
    rng = np.random.default_rng(seed)
    n = np.clip(np.round(np.exp(rng.uniform(np.log(32), np.log(1024), k)) / 16).astype(int) * 16,
                32, 1024)
    f = rng.integers(1, 65, k)
    t = 256 * rng.integers(1, 33, k)
    sig = rng.uniform(4, 32, k)
    return [(int(a), int(b_), int(c), float(d)) for a, b_, c, d in zip(n, f, t, sig)]


def bench_uneven_batch(xg, torch, steps):
    """One persistent launch over 96 uneven subarrays (autotuned, CUDA graph)
    vs the same jobs run one by one on the tensor-core and plain engines; every
    job's batched sums are compared with the plain engine's."""
    import numpy as np
    shapes = uneven_subarray_shapes()
    dev = torch.cuda.current_device()
    stream = torch.cuda.Stream()
    inputs, states, jobs = [], [], []
    for q, (n, f, t, sig) in enumerate(shapes):
        x = torch.empty(4 * n * f * t, dtype=torch.int8, device="cuda")
        xg.generate_device(x.data_ptr(), x.numel(), 0, 3000 + q, sig, dev)
        s = torch.empty(xg.state_elems(n, f), dtype=torch.int64, device="cuda")
        inputs.append(x)
        states.append(s)
        jobs.append({"input": x.data_ptr(), "state": s.data_ptr(), "nstation": n,
                     "nfrequency": f, "ntime": t})
    total_ops = sum(ops(n, f, t) for n, f, t, _ in shapes)
    out = {"jobs": len(shapes), "total_ops": total_ops}
    with xg.Batch(jobs, device=dev, stream=stream.cuda_stream, autotune=True, graph=True) as b:
        b.run()
        b.sync()
        out["tuning"] = b.info()
        k = max(2, min(steps, 10))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            b.run()
        e1.record(stream)
        b.sync()
        ms = e0.elapsed_time(e1) / k
    out["batched_ms"] = ms
    out["batched_tops"] = total_ops / (ms * 1e-3) / 1e12
    # The batch's buffers now hold its last run; the job-by-job contexts below
    # have buffers of their own, so every job's batched result is compared
    # with the plain engine's, bit for bit.
    out["jobs_compared_vs_plain"] = 0
    out["bit_exact_vs_plain"] = True
    out["max_nstation_compared"] = 0
    # job by job on each engine (per-call device time summed)
    for engine in ("tensor", "plain"):
        tot = 0.0
        for q, (n, f, t, _) in enumerate(shapes):
            with xg.Correlator(n, f, t, ntimepipe=256, engine=engine, device=dev) as c:
                st = torch.cuda.Stream()
                c.set_stream(st.cuda_stream)
                c.run_device(inputs[q].data_ptr(), xg.SYNCOP_SYNC_COMPUTE)   # warm
                c.clear()
                a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a0.record(st)
                c.run_device(inputs[q].data_ptr(), xg.SYNCOP_NONE)
                a1.record(st)
                a1.synchronize()
                tot += a0.elapsed_time(a1)
                if engine == "plain":
                    same = bool(np.array_equal(c.dump_int64(), states[q].cpu().numpy()))
                    out["bit_exact_vs_plain"] &= same
                    out["jobs_compared_vs_plain"] += 1
                    out["max_nstation_compared"] = max(out["max_nstation_compared"], n)
        out[f"{engine}_job_by_job_ms"] = tot
        out[f"{engine}_job_by_job_tops"] = total_ops / (tot * 1e-3) / 1e12
    out["batched_over_plain_job_by_job"] = out["plain_job_by_job_ms"] / out["batched_ms"]
    del inputs, states
    torch.cuda.empty_cache()
    return out


def served_requests(seconds, seed=4, rate_jobs=200.0):
    """Poisson arrivals of subarrays drawn like the 96-subarray batch, each
    integrating 4-32 blocks."""
    import numpy as np
    rng = np.random.default_rng(seed)
    t, reqs = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate_jobs)
        if t > seconds:
            break
        n = int(min(1024, max(32, round(np.exp(rng.uniform(np.log(32), np.log(1024))) / 16) * 16)))
        reqs.append({"nstation": n, "nfrequency": int(rng.integers(1, 65)),
                     "ntime": int(256 * rng.integers(1, 33)), "nblocks": int(rng.integers(4, 33)),
                     "seed": 5000 + len(reqs), "sigma": float(rng.uniform(4, 32)),
                     "arrival_s": float(t)})
    return reqs


SAMPLE_RATE = 1.0e5   # per-channel complex samples/s of the served stream


def request_ops(r):
    return ops(r["nstation"], r["nfrequency"], r["ntime"]) * r["nblocks"]


def served_check_sample(reqs, k=12, max_ops=3e11, seed=5):
    """Indices of served requests whose dumps the bench checks against the
    oracle: a seeded draw of k requests among those the oracle integrates in
    a few seconds on the host (at most max_ops), plus the cheapest request
    with N > 512."""
    import numpy as np
    cheap = [q for q, r in enumerate(reqs) if request_ops(r) <= max_ops]
    rng = np.random.default_rng(seed)
    pick = set(int(q) for q in rng.choice(cheap, size=min(k, len(cheap)), replace=False))
    big = [q for q, r in enumerate(reqs) if r["nstation"] > 512]
    if big:
        pick.add(min(big, key=lambda q: request_ops(reqs[q])))
    return sorted(pick)


def served_expected(oracle, r):
    """Final int32 triangular dump of a served request, from the oracle."""
    import numpy as np
    n, f, t = r["nstation"], r["nfrequency"], r["ntime"]
    acc = np.zeros(f * n * (n + 1) // 2 * 8, dtype=np.int64)
    for b in range(r["nblocks"]):
        x = oracle.serve_block_input(n, f, t, r["seed"], r["sigma"], b)
        oracle.xengine_i64(x, n, f, t, acc=acc)
    return acc.astype(np.int32)


def bench_served_stream(xg, seconds, plain_seconds, device):
    import numpy as np
    import oracle
    reqs = served_requests(seconds)
    check = served_check_sample(reqs)
    st, res = xg.serve(reqs, SAMPLE_RATE, 120 << 30, host_budget_bytes=24 << 30, device=device,
                       collect=check)
    exact = [bool(np.array_equal(res[q], served_expected(oracle, reqs[q]))) for q in check]
    out = {"arrival_rate_per_s": 200.0, "seconds": seconds, "sample_rate_hz": SAMPLE_RATE,
           "requests": len(reqs), "served": st,
           "served_bit_exact_sampled": all(exact), "sampled_requests": len(check),
           "sampled_max_nstation": max(reqs[q]["nstation"] for q in check),
           "sampled_ops": sum(request_ops(reqs[q]) for q in check)}
    if plain_seconds > 0:
        reqs_p = served_requests(plain_seconds)
        sp, _ = xg.serve(reqs_p, SAMPLE_RATE, 120 << 30, mode=xg.XGPU_SERVE_PLAIN_SERIAL,
                         host_budget_bytes=8 << 30, device=device)
        out["plain_serial"] = sp
        out["plain_serial_seconds_of_arrivals"] = plain_seconds
    return out


def channel_input(oracle, kind, seed, sigma, n, f_total, t, f):
    """Channel f's samples ([t][s][p][c] int8) of a seeded device-generated
    block [t][f_total][s][p] (kind 0: int8 {re,im}; kind 1: packed 4+4-bit),
    regenerated on the host: the generator's byte k depends only on (seed, k)."""
    import numpy as np
    width = n * (4 if kind == 0 else 2)
    rows = [oracle.generate(width, kind, seed, sigma, offset=(q * f_total + f) * width)
            for q in range(t)]
    x = np.concatenate(rows)
    return x if kind == 0 else oracle.unpack4(x)


def bench_large_array(xg, torch, device, blocks=64, check_channels=(0, F3 - 1)):
    """The large-array configuration: N=512, F=256, T=8192 per block, 64 blocks
    integrated before one dump, with packed 4+4-bit input expanded on the device
    (uniform [-7,7]) and an int8 variant (sigma 40).  Two distinct input blocks
    alternate (4.3 / 2.1 GB each, far above L2).  Exactness: the first block's
    sums on two channels equal the oracle's (int64, omp_xengine.c:45-89), and
    64 blocks alternating A, B equal 32 x (A + B) (linearity, every channel)."""
    import numpy as np
    import oracle
    out = {"nstation": N3, "nfrequency": F3, "ntime": T3, "blocks": blocks}
    for fmt, kind, sig in (("packed4", 1, 0.0), ("int8", 0, 40.0)):
        # The context's own streams (packed input is expanded on a side stream
        # before each block's correlation); timed by the host around a
        # synchronised 64-block run (hundreds of ms).
        c = xg.Correlator(N3, F3, T3, ntimepipe=128, engine="tensor", input_format=fmt,
                          device=device)
        c.tune(1, 0, 1)
        nbytes = int(c.info.vecLength) * (1 if fmt == "packed4" else 2)
        bufs = []
        for q in range(2):
            x = torch.empty(nbytes, dtype=torch.int8, device="cuda")
            xg.generate_device(x.data_ptr(), nbytes, kind, 9000 + q, sig or 16.0, device)
            bufs.append(x)
        # A alone: sampled channels against the oracle; then A + B, for the
        # linearity check
        c.clear()
        c.run_device(bufs[0].data_ptr(), xg.SYNCOP_SYNC_COMPUTE)
        a_sums = c.dump_int64()
        nb8 = N3 * (N3 + 1) // 2 * 8
        channels_exact = True
        for f in check_channels:
            x = channel_input(oracle, kind, 9000, sig or 16.0, N3, F3, T3, f)
            want = oracle.xengine_i64(x, N3, 1, T3)
            channels_exact &= bool(np.array_equal(a_sums[f * nb8:(f + 1) * nb8], want))
        del a_sums
        c.run_device(bufs[1].data_ptr(), xg.SYNCOP_SYNC_COMPUTE)
        ab = torch.from_numpy(c.dump_int64())
        c.clear()
        torch.cuda.synchronize()
        h0 = time.perf_counter()
        for q in range(blocks - 1):
            c.run_device(bufs[q & 1].data_ptr(), xg.SYNCOP_NONE)
        c.run_device(bufs[(blocks - 1) & 1].data_ptr(), xg.SYNCOP_SYNC_COMPUTE)
        ms = (time.perf_counter() - h0) * 1e3
        full = torch.from_numpy(c.dump_int64())
        o = ops(N3, F3, T3) * blocks
        out[fmt] = {"ms_total": ms, "ms_per_block": ms / blocks, "tops": o / (ms * 1e-3) / 1e12,
                    "max_abs_visibility": int(full.abs().max()),
                    "exceeds_int32": bool(full.abs().max() > 2**31 - 1),
                    "linearity_exact": bool(torch.equal(full, (blocks // 2) * ab)),
                    "oracle_channels_exact": channels_exact,
                    "oracle_channels": list(check_channels)}
        c.close()
        del bufs
        torch.cuda.empty_cache()
    return out


def int8_peak_tops(torch):
    """Dense int8 tensor throughput of cuBLASLt (torch._int_mm) at 8192^3."""
    try:
        m = 8192
        a = torch.randint(-128, 127, (m, m), dtype=torch.int8, device="cuda")
        b = torch.randint(-128, 127, (m, m), dtype=torch.int8, device="cuda").t()
        for _ in range(3):
            torch._int_mm(a, b)
        torch.cuda.synchronize()
        best = 1e9
        for _ in range(5):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(5):
                torch._int_mm(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1) / 5)
        return 2.0 * m ** 3 / (best * 1e-3) / 1e12
    except Exception:
        return None


def cpu_model():
    """The host CPU's model name (for the CPU baseline's record), or None."""
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_baseline(steps_cap=None, budget_s=12.0):
    """The reference's xgpuOmpXengine on the host, DP4A build, this workload."""
    import oracle
    if not oracle.ref_available("c2", "dp4a_rt"):
        return None
    R = oracle.RefLib("c2", "dp4a_rt")
    x = oracle.gaussian_input(N, F, T, seed=1, sigma=SIGMA)
    R.omp_xengine(x)  # warm
    times = []
    t_start = time.perf_counter()
    while True:
        t0 = time.perf_counter()
        R.omp_xengine(x)
        times.append(time.perf_counter() - t0)
        if steps_cap and len(times) >= steps_cap:
            break
        if time.perf_counter() - t_start > budget_s and len(times) >= 3:
            break
    med = statistics.median(times)
    return {"value": ops(N, F, T) / med / 1e12, "unit": "TOPS", "cores": os.cpu_count(),
            "kind": "reference", "cpu_model": cpu_model(),
            "sample": f"{len(times)} full calls of xgpuOmpXengine (src/omp_xengine.c, -O3 -fopenmp, "
                      f"DP4A build) at N={N} F={F} T={T}; median {med * 1e3:.1f} ms per call",
            "ms_per_call": med * 1e3}


def run_reference(args, world, rank):
    if rank != 0:
        return
    import oracle
    base = {"metric": METRIC, "unit": "TOPS", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True}
    if not oracle.ref_available("c2", "dp4a_rt"):
        base["unavailable"] = "reference CPU engine not built (oracle/_ref missing)"
        print(json.dumps(base))
        return
    R = oracle.RefLib("c2", "dp4a_rt")
    x = oracle.gaussian_input(N, F, T, seed=1, sigma=SIGMA)
    for _ in range(args.warmup):
        R.omp_xengine(x)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        R.omp_xengine(x)
    ms = (time.perf_counter() - t0) * 1e3 / args.steps
    v = ops(N, F, T) / (ms * 1e-3) / 1e12
    base.update({
        "value": v, "ms_per_step": ms, "scaling": "weak", "vs_baseline": None, "dtype": "int8",
        "data": "synthetic: seeded Gaussian int8, sigma 16",
        "config": {"workload": f"xgpuOmpXengine NSTATION={N} NPOL=2 NFREQUENCY={F} NTIME={T}, "
                               "one call per step", "nstation": N, "npol": 2, "nfrequency": F,
                   "ntime": T, "parallelism": "host cores of rank 0 (OpenMP)"},
        "cpu_baseline": {"value": v, "unit": "TOPS", "cores": os.cpu_count(), "kind": "reference",
                         "cpu_model": cpu_model(),
                         "sample": f"{args.steps} calls of the reference xgpuOmpXengine (DP4A "
                                   "build, OpenMP on all host cores)"},
        "e2e": {"value": v, "unit": "TOPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    })
    print(json.dumps(base))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--tune", type=lambda v: tuple(int(x) for x in v.split(",")), default=None,
                    help="ksplit,grid,pair for the headline leg instead of the autotuner (a "
                         "profiler's serialised launches mislead the autotuner)")
    ap.add_argument("--no-detail", action="store_true",
                    help="skip the plain, N=512, batched and served legs")
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="seconds of Poisson arrivals for the served stream")
    ap.add_argument("--plain-serve-seconds", type=float, default=2.0,
                    help="seconds of arrivals for the one-at-a-time plain baseline (it falls "
                         "behind the arrivals, so its latency grows with this)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        # CPU only: rank 0 times the reference, the other ranks exit at once;
        # no process group is needed
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")),
                      int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_setup(args)

    import torch
    import oracle
    import xgpu_b200 as xg
    torch.cuda.set_device(local)
    clocks = Clocks(local)

    # headline: tensor engine, xGPU's default shape, input resident in HBM
    ms, rot_bytes = device_engine_ms(xg, torch, "tensor", "int8", N, F, T, args.steps,
                                     args.warmup, world, tune=args.tune)
    ms = max_over_ranks(world, ms)
    value = world * ops(N, F, T) / (ms * 1e-3) / 1e12

    detail = {}
    # The detail legs characterise one GPU; with several ranks (weak-scaling
    # replicas) only the headline and end-to-end legs run.
    if not args.no_detail and world == 1:
        k2 = max(3, min(args.steps, 50))
        ms_p, _ = device_engine_ms(xg, torch, "plain", "int8", N, F, T, k2, 3, world)
        ms_f, _ = device_engine_ms(xg, torch, "plain", "fp32", N, F, T, k2, 3, world)
        detail["plain_dp4a_n256_tops"] = ops(N, F, T) / (ms_p * 1e-3) / 1e12
        detail["plain_fp32_n256_tops"] = ops(N, F, T) / (ms_f * 1e-3) / 1e12
        detail["tc_over_plain_dp4a_n256"] = value / world / detail["plain_dp4a_n256_tops"]
        # the plain engines' own rooflines: measured CUDA-core dp4a and FP32
        # FMA rates (X-engine operations per second)
        for kind in ("dp4a", "fp32"):
            pk = xg.core_peak(kind, local) / 1e12
            detail[f"core_{kind}_peak_tops_measured"] = pk
            detail[f"plain_{kind}_n256_frac_of_core_peak"] = detail[f"plain_{kind}_n256_tops"] / pk
        # The FP32 engine adds each sample's exact product pair with one
        # rounding, as xGPU's float engine does: 6 FP32 instructions (FMUL,
        # FFMA, FADD per component) per complex MAC of 8 operations, where the
        # measured rate counts 4 FMAs.  Its instruction ceiling is 4/6 of it.
        detail["plain_fp32_n256_frac_of_instruction_ceiling"] = (
            detail["plain_fp32_n256_tops"] / (detail["core_fp32_peak_tops_measured"] * 4 / 6))
        if rank == 0:
            # the default shape itself (every sum below 2^24: exact) and a long
            # integration whose sums pass 2^24
            detail["float32_output_n256_f10_t1024"] = float_output_error(xg, oracle, N, F, T, SIGMA, local)
            detail["float32_output_long"] = float_output_error(xg, oracle, 64, 10, 32768, 40.0,
                                                               local)
            detail["fp32_engine_vs_reference_float"] = fp32_engine_long(xg, oracle, local)
        k3 = max(3, min(args.steps, 10))
        ms3, _ = device_engine_ms(xg, torch, "tensor", "int8", N3, F3, T3, k3, 2, world,
                                  sigma=40.0, min_rotate_bytes=0, max_bufs=1)
        detail["tc_n512_tops"] = ops(N3, F3, T3) / (ms3 * 1e-3) / 1e12
        detail["tc_n512_ms_per_block"] = ms3
        detail["tc_n512_tuning"] = TUNING.get(("tensor", N3, F3, T3))
        if rank == 0:
            detail["large_array_n512_f256_t8192"] = bench_large_array(xg, torch, local)
            detail["uneven_batch_96_subarrays"] = bench_uneven_batch(xg, torch, args.steps)
            c5 = bench_served_stream(xg, args.serve_seconds, args.plain_serve_seconds, local)
            detail["served_stream"] = c5
            detail["served_p50_dump_ms"] = c5["served"]["dump_p50_ms"]
            detail["served_p99_dump_ms"] = c5["served"]["dump_p99_ms"]
            detail["served_tops"] = c5["served"]["tops"]

    e2e_v = None
    if rank == 0:
        k_e = max(3, min(args.steps, 50))
        ms_e, h2d, d2h, ok = e2e_ms(xg, oracle, N, F, T, k_e, 3, local)
        e2e_v = {"value": ops(N, F, T) / (ms_e * 1e-3) / 1e12, "unit": "TOPS",
                 "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": ms_e,
                 "steps": k_e, "bit_exact_vs_oracle": ok,
                 # each step copies its input in and its dump out, channel
                 # group by channel group (the two directions overlap): the
                 # host link sets the pace
                 "host_link_gbs": (h2d + d2h) / (ms_e * 1e-3) / 1e9}
        if not args.no_detail and world == 1:
            detail["e2e_streaming"] = e2e_streaming(xg, oracle, N, F, T, 8, max(3, min(args.steps, 20)),
                                                    local)
    clk = clocks.stop()
    peak8 = int8_peak_tops(torch) if rank == 0 else None
    if rank != 0:
        barrier(world)
        import torch.distributed as dist
        dist.destroy_process_group()
        return

    peaks, peak_src = load_peaks()
    # Roofline of the tensor kernel at this workload.  Algorithmic bytes per
    # launch: input 4*F*T*N + int64 integration buffer read and written
    # (2 * 16 * F * N(N+1)/2 * 4 ... = 2 * F * N(N+1)/2 * 4 pol * 2 * 8 B).
    in_bytes = 4.0 * F * T * N
    state_bytes = F * N * (N + 1) / 2 * 4 * 2 * 8
    alg_bytes = in_bytes + 2 * state_bytes
    t_s = ms * 1e-3
    hbm_ach = alg_bytes / t_s / 1e9
    tops_ach = ops(N, F, T) / t_s / 1e12
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    t_hbm = alg_bytes / (hbm_peak * 1e9)
    t_tc = ops(N, F, T) / ((peak8 or 2 * float(peaks.get("bf16_tflops", 1590.0))) * 1e12)
    tuning = TUNING.get(("tensor", N, F, T)) or {}
    traffic = read_profile_traffic(tuning.get("pair", 0))
    kernel = "xengine_tc2_kernel" if tuning.get("pair", 0) == 1 else "xengine_tc_kernel"
    if t_hbm >= t_tc:
        roof = {"bound": "hbm", "kernel": kernel, "achieved": hbm_ach, "peak": hbm_peak, "unit": "GB/s",
                "frac": hbm_ach / hbm_peak, "traffic": traffic,
                "peak_source": f"hbm_gbs of {peak_src} (of measured)",
                "algorithmic_bytes_per_launch": alg_bytes,
                "note": "algorithmic bytes = input + int64 buffer read and written; adding "
                        "launches keep the call's sums in a word buffer of half those bytes, "
                        "which stays in L2 between calls, so DRAM sees less (traffic: ncu, "
                        "cold stand-alone launch: input + words)"}
    else:
        roof = {"bound": "tensor", "kernel": kernel, "achieved": tops_ach, "peak": peak8, "unit": "TOPS",
                "frac": tops_ach / peak8, "traffic": traffic,
                "peak_source": "dense int8 cuBLASLt GEMM 8192^3 measured in this run (of measured)"}
    detail["int8_tensor_peak_tops_measured"] = peak8
    detail["tc_n256_frac_of_int8_peak"] = tops_ach / peak8 if peak8 else None
    detail["tc_n256_hbm_gbs"] = hbm_ach
    if "tc_n512_tops" in detail and peak8:
        detail["tc_n512_frac_of_int8_peak"] = detail["tc_n512_tops"] / peak8

    line = {
        "metric": METRIC, "value": value, "unit": "TOPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int8",
        "data": "synthetic: seeded Gaussian int8 samples, sigma 16 (counter-based generator)",
        "config": {"workload": f"xGPU default shape NSTATION={N} NPOL=2 NFREQUENCY={F} NTIME={T}: "
                               "one xgpuCudaXengineDevice call per step on input resident in "
                               "HBM (SYNCOP_NONE, accumulating), tcgen05 int8 engine, int64 "
                               "integration buffer; host buffers and copies: see e2e",
                   "nstation": N, "npol": 2, "nfrequency": F, "ntime": T,
                   "parallelism": f"channel-sharded replicas x{world} (no collective)",
                   "l2": f"input rotates over {rot_bytes / 2**20:.0f} MiB of buffers (> 126 MiB L2)",
                   "tuning": TUNING.get(("tensor", N, F, T)),
                   "launches": "programmatic (PDL): each accumulating call may start while the "
                               "previous call's launch finishes; ms_per_step is the spacing",
                   "timing": "CUDA events on the context's stream around the K calls and "
                             "the closing xgpuFlushIntegrationBuffer (the word buffer's "
                             "fold into the int64 buffer); the time includes filling and "
                             "draining the chain of overlapping launches (about 35 us per "
                             "run), so short runs read lower"},
        "e2e": e2e_v, "gpu_launches": args.steps + FOLDS.get(("tensor", N, F, T), 0),
        "roofline": roof,
        # the host-core baseline is timed at N=1 only
        "cpu_baseline": cpu_baseline() if world == 1 else None, "clocks": clk, "detail": detail,
    }
    print(json.dumps(line))
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
