"""Parity of libxgpu.so on a B200 against the oracle, through the C ABI.

Integer engines (tcgen05 tensor cores, CUDA-core dp4a) must be bit-exact with
the oracle's int64 sums, which tests/test_oracle_golden.py pins to the
reference's xgpuOmpXengine.  The FP32 engine must equal the reference's float
engine exactly where every partial sum is an integer below 2^24 (the
configurations below), and stay within 1e-6 relative of the exact sums
otherwise.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ENGINES = [("tensor", "int8"), ("plain", "int8"), ("plain", "fp32")]


def correlate(xg, chunks, n, f, t, engine, compute, output="int32", order="tri", **kw):
    """Run one integration of len(chunks) calls through xgpuCudaXengine."""
    with xg.Correlator(n, f, t, engine=engine, compute=compute, output=output, order=order,
                       **kw) as c:
        for q, x in enumerate(chunks):
            c.set_input(x)
            c.run(xg.SYNCOP_DUMP if q == len(chunks) - 1 else xg.SYNCOP_NONE)
        out = c.output_view()[: c.info.matLength * 2].copy()
        exact = c.dump_int64() if compute == "int8" else None
    return out, exact


def expected_words(oracle_mod, exact, n, f, order, output):
    words = exact.astype(np.int32) if output == "int32" else exact.astype(np.float32)
    if order == "tri":
        return words
    code = {"ri": 2000, "rt": 3000}[order]
    return oracle_mod.tri_to_order(words, n, f, code)


@pytest.mark.parametrize("engine,compute", ENGINES)
@pytest.mark.parametrize("n,f,t", [(16, 2, 64), (32, 3, 256), (48, 2, 128), (64, 10, 1024),
                                   (80, 1, 512), (256, 10, 1024)])
def test_single_call_triangular(xg, oracle_mod, engine, compute, n, f, t):
    x = oracle_mod.gaussian_input(n, f, t, seed=n + f + t, sigma=16.0)
    exact = oracle_mod.xengine_i64(x, n, f, t)
    output = "int32" if compute == "int8" else "float32"
    out, ex64 = correlate(xg, [x], n, f, t, engine, compute, output=output)
    if compute == "int8":
        assert np.array_equal(ex64, exact)
        assert np.array_equal(out, exact.astype(np.int32))
    else:
        assert np.array_equal(out, oracle_mod.xengine_f32(x, n, f, t))


@pytest.mark.parametrize("engine,compute", ENGINES)
@pytest.mark.parametrize("order", ["tri", "ri", "rt"])
@pytest.mark.parametrize("output", ["int32", "float32"])
def test_orders_and_output_types(xg, oracle_mod, engine, compute, order, output):
    n, f, t = 32, 3, 256
    x = oracle_mod.gaussian_input(n, f, t, seed=77, sigma=20.0)
    exact = oracle_mod.xengine_i64(x, n, f, t)
    out, _ = correlate(xg, [x], n, f, t, engine, compute, output=output, order=order)
    assert np.array_equal(out, expected_words(oracle_mod, exact, n, f, order, output))


@pytest.mark.parametrize("engine", ["tensor", "plain"])
def test_reference_shapes_against_reference_digests(xg, oracle_mod, golden, engine):
    """Configs 1-2 (N=64/256, F=10, T=1024): the dumped int32 triangular matrix
    hashes to the reference xgpuOmpXengine DP4A output's digest."""
    import hashlib
    meta, _ = golden
    for shape in ("c1", "c2"):
        e = meta["shapes"][shape]
        x = oracle_mod.gaussian_input(e["n"], e["f"], e["t"], seed=e["seed"], sigma=e["sigma"])
        out, _ = correlate(xg, [x], e["n"], e["f"], e["t"], engine, "int8")
        assert hashlib.sha256(out.tobytes()).hexdigest() == e["omp_dp4a_sha"], shape


def test_fp32_reference_digest(xg, oracle_mod, golden):
    import hashlib
    meta, _ = golden
    for shape in ("c1", "c2"):
        e = meta["shapes"][shape]
        x = oracle_mod.gaussian_input(e["n"], e["f"], e["t"], seed=e["seed"], sigma=e["sigma"])
        out, _ = correlate(xg, [x], e["n"], e["f"], e["t"], "plain", "fp32", output="float32")
        assert hashlib.sha256(out.tobytes()).hexdigest() == e["omp_fp32_sha"], shape


@pytest.mark.parametrize("engine,compute", ENGINES)
def test_multi_call_integration_and_clear(xg, oracle_mod, engine, compute):
    n, f, t = 48, 4, 256
    xs = [oracle_mod.gaussian_input(n, f, t, seed=s) for s in (1, 2, 3)]
    output = "int32" if compute == "int8" else "float32"
    with xg.Correlator(n, f, t, engine=engine, compute=compute, output=output) as c:
        # Each syncOp once; the host buffer is rewritten only after a call that
        # waited for its transfer (SYNC_TRANSFER / SYNC_COMPUTE), and the last
        # call (SYNCOP_NONE) is completed by xgpuDumpDeviceIntegrationBuffer.
        for x, sync in zip(xs, (xg.SYNCOP_SYNC_TRANSFER, xg.SYNCOP_SYNC_COMPUTE, xg.SYNCOP_NONE)):
            c.set_input(x)
            c.run(sync)
        got = c.dump()
        exact = oracle_mod.xengine_i64(np.concatenate(xs), n, f, 3 * t)
        assert np.array_equal(got, exact.astype(got.dtype))
        # clear starts a new integration
        c.clear()
        assert not c.dump().any()
        c.set_input(xs[0])
        c.run(xg.SYNCOP_DUMP)
        got = c.output_view()[: c.info.matLength * 2]
        assert np.array_equal(got, oracle_mod.xengine_i64(xs[0], n, f, t).astype(got.dtype))


@pytest.mark.parametrize("engine", ["tensor", "plain"])
def test_exact_past_int32(xg, oracle_mod, engine):
    """Full-scale -128 input for 3 x 32768 samples: every auto-correlation real
    part is 3 * 32768 * 32768 = 3.2e9 > 2^31.  The int64 dump is exact; the
    int32 dump wraps exactly as xGPU's int32 buffer would."""
    n, f, t = 16, 1, 32768
    x = np.full(t * f * n * 4, -128, dtype=np.int8)
    x[1::4] = 127   # make the imaginary parts non-trivial
    with xg.Correlator(n, f, t, ntimepipe=128, engine=engine) as c:
        c.set_input(x)
        for _ in range(2):
            c.run(xg.SYNCOP_SYNC_COMPUTE)
        c.run(xg.SYNCOP_DUMP)
        ex = c.dump_int64()
        out = c.output_view()[: c.info.matLength * 2].copy()
    one = oracle_mod.xengine_i64(x, n, f, t)
    want = 3 * one
    assert np.abs(want).max() > 2**31
    assert np.array_equal(ex, want)
    assert np.array_equal(out, want.astype(np.int32))


@pytest.mark.parametrize("engine", ["tensor", "plain"])
def test_float_output_relative_error_vs_fp64(xg, oracle_mod, engine):
    """Float32 output of the integer engines: the exact int64 sums are rounded
    to float once, at dump (round to nearest), so against the FP64 host oracle
    the relative error of every non-zero element is at most 2^-24 (6e-8, well
    inside 1e-6), here with sums far beyond 2^24 where float accumulation
    would drift; zero sums stay zero.  (The other orders place the same
    rounded words: test_orders_and_output_types.)"""
    n, f, t = 32, 2, 32768
    x = oracle_mod.gaussian_input(n, f, t, seed=17, sigma=40.0)
    with xg.Correlator(n, f, t, ntimepipe=128, engine=engine, output="float32") as c:
        c.set_input(x)
        c.run(xg.SYNCOP_SYNC_COMPUTE)
        c.run(xg.SYNCOP_DUMP)
        out = c.output_view()[: c.info.matLength * 2].astype(np.float64)
    exact = (2 * oracle_mod.xengine_i64(x, n, f, t)).astype(np.float64)   # FP64 oracle
    assert np.abs(exact).max() > 4 * 2**24
    nz = exact != 0
    rel = np.abs(out[nz] - exact[nz]) / np.abs(exact[nz])
    assert rel.max() <= 2.0**-24
    assert rel.max() > 0            # the sums are large enough to round
    assert not out[~nz].any()


@pytest.mark.parametrize("engine,compute", ENGINES)
def test_full_range_and_known_answers(xg, oracle_mod, golden, engine, compute):
    _, arr = golden
    n, f, t = 16, 2, 64
    x = arr["s16_fullrange_input"]
    out, _ = correlate(xg, [x], n, f, t, engine, compute,
                       output="int32" if compute == "int8" else "float32")
    want = arr["s16_fullrange_omp_dp4a"]
    assert np.array_equal(out.astype(np.int64), want.astype(np.int64))
    # known answer: only station 5 pol X non-zero, value (3 + 4j) at every sample
    x = np.zeros(t * f * n * 4, dtype=np.int8).reshape(t, f, n, 2, 2)
    x[:, :, 5, 0, 0] = 3
    x[:, :, 5, 0, 1] = 4
    out, _ = correlate(xg, [x.ravel()], n, f, t, engine, compute,
                       output="int32" if compute == "int8" else "float32")
    v = out.reshape(f, n * (n + 1) // 2, 2, 2, 2).astype(np.int64)
    k55 = 5 * 6 // 2 + 5
    assert (v[:, k55, 0, 0, 0] == 25 * t).all() and (v[:, k55, 0, 0, 1] == 0).all()
    v[:, k55, 0, 0, 0] = 0
    assert not v.any()


@pytest.mark.parametrize("engine", ["tensor", "plain"])
def test_packed4_input(xg, oracle_mod, engine):
    """4+4-bit packed input (one byte per complex sample) expands exactly."""
    n, f, t = 64, 3, 512
    packed = oracle_mod.generate(t * f * n * 2, 1, 2)
    x = oracle_mod.unpack4(packed)
    with xg.Correlator(n, f, t, engine=engine, input_format="packed4") as c:
        c.set_input(packed)
        c.run(xg.SYNCOP_DUMP)
        ex = c.dump_int64()
    assert np.array_equal(ex, oracle_mod.xengine_i64(x, n, f, t))


@pytest.mark.parametrize("engine", ["tensor", "plain"])
def test_dp4a_swizzled_input(xg, oracle_mod, engine):
    n, f, t = 32, 2, 256
    x = oracle_mod.gaussian_input(n, f, t, seed=8)
    with xg.Correlator(n, f, t, engine=engine, input_format="dp4a_swizzled") as c:
        c.set_input(oracle_mod.swizzle(x, n, f, t))
        c.run(xg.SYNCOP_DUMP)
        ex = c.dump_int64()
    assert np.array_equal(ex, oracle_mod.xengine_i64(x, n, f, t))


@pytest.mark.parametrize("engine,compute", [("tensor", "int8"), ("plain", "int8"),
                                            ("plain", "fp32")])
def test_block32_input(xg, oracle_mod, engine, compute):
    """xGPU's COMPLEX_BLOCK_SIZE=32 input layout, unblocked on the device."""
    n, f, t = 48, 3, 512
    x = oracle_mod.gaussian_input(n, f, t, seed=21, sigma=40.0)
    out = "int32" if compute == "int8" else "float32"
    with xg.Correlator(n, f, t, engine=engine, compute=compute, output=out,
                       input_format="block32") as c:
        assert c.info.complex_block_size == 32
        c.set_input(oracle_mod.block32(x))
        c.run(xg.SYNCOP_DUMP)
        got = c.output_view()[: c.info.matLength * 2]
        exact = oracle_mod.xengine_i64(x, n, f, t)
        if compute == "int8":
            assert np.array_equal(c.dump_int64(), exact)
            assert np.array_equal(got, exact.astype(np.int32))
        else:
            assert np.array_equal(got, oracle_mod.xengine_f32(x, n, f, t))


def test_core_peaks(xg):
    """The measured CUDA-core rates are positive, repeatable within 10%, and
    in the range 148 SMs allow (dp4a: 8 operations each; FMA: 2)."""
    for kind, lo, hi in (("dp4a", 30e12, 1.2e15), ("fp32", 20e12, 3e14)):
        a, b = xg.core_peak(kind), xg.core_peak(kind)
        assert lo < a < hi and lo < b < hi, (kind, a, b)
        assert abs(a - b) < 0.1 * max(a, b), (kind, a, b)


def test_device_generator_matches_host(xg, oracle_mod):
    import torch
    for kind, sigma in [(0, 16.0), (0, 40.0), (1, 0.0), (2, 0.0)]:
        nbytes = 1 << 20 | 3
        d = torch.empty(nbytes, dtype=torch.int8, device="cuda")
        xg.generate_device(d.data_ptr(), nbytes, kind, 1234, sigma)
        assert np.array_equal(d.cpu().numpy(), oracle_mod.generate(nbytes, kind, 1234, sigma))


@pytest.mark.parametrize("engine", ["tensor", "plain"])
def test_device_input_and_offsets(xg, oracle_mod, engine):
    import torch
    n, f, t = 64, 2, 256
    x = oracle_mod.gaussian_input(n, f, t, seed=5)
    d = torch.from_numpy(x).cuda()
    with xg.Correlator(n, f, t, engine=engine) as c:
        c.run_device(d.data_ptr(), xg.SYNCOP_SYNC_COMPUTE)
        got = c.dump()
        assert np.array_equal(got, oracle_mod.xengine_i64(x, n, f, t).astype(np.int32))


def page_aligned(count, dtype, page=4096):
    itemsize = np.dtype(dtype).itemsize
    nbytes = -(-count * itemsize // page) * page
    raw = np.zeros(nbytes + page, dtype=np.uint8)
    start = (-raw.ctypes.data) % page
    return raw[start: start + nbytes].view(dtype)[:count]


def test_caller_buffers_registered_and_offsets(xg, oracle_mod):
    """Caller-allocated host buffers (registered page-rounded, or not at all)
    and input/output offsets, as xgpu.h:103-109 describes."""
    n, f, t = 32, 2, 128
    x = oracle_mod.gaussian_input(n, f, t, seed=6)
    exact = oracle_mod.xengine_i64(x, n, f, t).astype(np.int32)
    for flags in (0, xg.XGPU_DONT_REGISTER):
        cfg = xg.default_config()
        cfg.nstation, cfg.nfrequency, cfg.ntime, cfg.ntimepipe = n, f, t, 128
        cfg.output_type, cfg.matrix_order = xg.XGPU_INT32, xg.TRIANGULAR_ORDER
        off_in, off_out = 100, 7
        # Page-aligned, page-sized buffers: registration is page-rounded, so
        # two buffers must not share a page (as with xGPU).
        inbuf = page_aligned(x.size + 2 * off_in + 64, np.int8)
        inbuf[2 * off_in: 2 * off_in + x.size] = x
        outbuf = page_aligned(2 * (exact.size // 2 + off_out) + 16, np.int32)
        ctx = xg.XGPUContext()
        ctx.array_h = inbuf.ctypes.data
        ctx.array_len = inbuf.size // 2
        ctx.matrix_h = outbuf.ctypes.data
        ctx.matrix_len = outbuf.size // 2
        L = xg.lib()
        assert L.xgpuInitEx(ctypes.byref(ctx), flags, ctypes.byref(cfg)) == 0
        if flags:
            assert L.xgpuCudaXengine(ctypes.byref(ctx), 1) == xg.XGPU_HOST_BUFFER_NOT_SET
            assert L.xgpuSetHostInputBuffer(ctypes.byref(ctx)) == 0
            assert L.xgpuSetHostOutputBuffer(ctypes.byref(ctx)) == 0
        ctx.input_offset, ctx.output_offset = off_in, off_out
        assert L.xgpuCudaXengine(ctypes.byref(ctx), xg.SYNCOP_DUMP) == 0
        assert np.array_equal(outbuf[2 * off_out: 2 * off_out + exact.size], exact)
        # an offset that runs past the caller's buffer is refused
        ctx.input_offset = ctx.array_len
        assert L.xgpuCudaXengine(ctypes.byref(ctx), 1) == xg.XGPU_INVALID_ARGUMENT
        L.xgpuFree(ctypes.byref(ctx))
        assert not ctx.internal


def test_library_buffers_kept_when_set_again(xg, oracle_mod):
    """xgpuSetHostInputBuffer / xgpuSetHostOutputBuffer called again with the
    buffers the library allocated (array_h and matrix_h unchanged) keep them:
    the pointers stay valid, hold what the caller wrote, and the call after
    them is exact.  (Taken literally, the reference's steps would free the
    buffer and then register the freed pointer.)"""
    n, f, t = 32, 2, 128
    x = oracle_mod.gaussian_input(n, f, t, seed=8)
    exact = oracle_mod.xengine_i64(x, n, f, t).astype(np.int32)
    with xg.Correlator(n, f, t, ntimepipe=128, order="tri") as c:
        c.set_input(x)
        a, m = c.ctx.array_h, c.ctx.matrix_h
        L = xg.lib()
        for _ in range(2):
            assert L.xgpuSetHostInputBuffer(ctypes.byref(c.ctx)) == 0
            assert L.xgpuSetHostOutputBuffer(ctypes.byref(c.ctx)) == 0
        assert (c.ctx.array_h, c.ctx.matrix_h) == (a, m)
        assert np.array_equal(c.input_view()[: x.size], x)
        c.run(xg.SYNCOP_DUMP)
        assert np.array_equal(c.output_view()[: exact.size], exact)


def test_reference_api_default_context(xg, oracle_mod):
    """The unmodified xGPU calling sequence (cuda_correlator.c:145-253) at the
    default sizes: xgpuInit with library-allocated buffers, xgpuCudaXengine
    with SYNCOP_DUMP, xgpuReorderMatrix, compare with the CPU engine."""
    L = xg.lib()
    info = xg.default_info()
    ctx = xg.XGPUContext()
    assert L.xgpuInit(ctypes.byref(ctx), 0) == 0
    x = oracle_mod.gaussian_input(info.nstation, info.nfrequency, info.ntime, seed=1)
    ctypes.memmove(ctx.array_h, x.ctypes.data, x.size)
    assert L.xgpuCudaXengine(ctypes.byref(ctx), xg.SYNCOP_DUMP) == 0
    m = np.frombuffer((ctypes.c_float * (2 * info.matLength)).from_address(ctx.matrix_h),
                      dtype=np.float32).copy()
    L.xgpuReorderMatrix(m.ctypes.data)
    exact = oracle_mod.xengine_i64(x, info.nstation, info.nfrequency, info.ntime)
    assert np.array_equal(m[: exact.size], exact.astype(np.float32))
    L.xgpuFree(ctypes.byref(ctx))


@pytest.mark.parametrize("fmt", ["packed4", "dp4a_swizzled", "block32"])
def test_converted_inputs_back_to_back(xg, oracle_mod, fmt):
    """Several calls in flight: each call's input conversion runs on its own
    stream into one of two buffers, under the previous call's correlation."""
    n, f, t = 96, 3, 1024
    raws, feeds = [], []
    for s in range(4):
        if fmt == "packed4":
            p = oracle_mod.generate(t * f * n * 2, 1, 50 + s)
            raws.append(oracle_mod.unpack4(p))
            feeds.append(p)
        else:
            x = oracle_mod.gaussian_input(n, f, t, seed=50 + s)
            raws.append(x)
            feeds.append(oracle_mod.swizzle(x, n, f, t) if fmt == "dp4a_swizzled"
                         else oracle_mod.block32(x))
    with xg.Correlator(n, f, t, engine="tensor", input_format=fmt) as c:
        for q, feed in enumerate(feeds):
            c.set_input(feed)
            c.run(xg.SYNCOP_SYNC_TRANSFER if q < 3 else xg.SYNCOP_DUMP)
        got = c.dump_int64()
    assert np.array_equal(got, oracle_mod.xengine_i64(np.concatenate(raws), n, f, 4 * t))


def test_converted_device_input_on_caller_stream(xg, oracle_mod):
    import torch
    n, f, t = 64, 2, 512
    stream = torch.cuda.Stream()
    with xg.Correlator(n, f, t, engine="tensor", input_format="packed4") as c:
        c.set_stream(stream.cuda_stream)
        want = np.zeros(f * n * (n + 1) // 2 * 8, dtype=np.int64)
        for s in range(3):
            p = oracle_mod.generate(t * f * n * 2, 1, 70 + s)
            with torch.cuda.stream(stream):
                d = torch.from_numpy(p).to("cuda", non_blocking=False)
                c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
                stream.synchronize()
            oracle_mod.xengine_i64(oracle_mod.unpack4(p), n, f, t, acc=want)
        assert np.array_equal(c.dump_int64(), want)


@pytest.mark.parametrize("engine,pair,ksplit", [("tensor", 0, 1), ("tensor", 1, 1),
                                                ("tensor", 0, 3), ("tensor", 2, 1),
                                                ("plain", None, None)])
def test_overlapping_accumulating_calls(xg, oracle_mod, engine, pair, ksplit):
    """Back-to-back accumulating calls over device input on the context's own
    stream: each launch may start before the previous one has finished (the
    two only add into the integration; the plain dp4a engine's time splits
    too).  Sums stay exact, also across a dump in the middle and a clear."""
    import torch
    n, f, t = 128, 5, 1024
    xs = [oracle_mod.gaussian_input(n, f, t, seed=90 + q, sigma=30.0) for q in range(5)]
    ds = [torch.from_numpy(x).cuda() for x in xs]
    torch.cuda.synchronize()
    one = sum(oracle_mod.xengine_i64(x, n, f, t) for x in xs)
    with xg.Correlator(n, f, t, engine=engine) as c:
        if engine == "tensor":
            c.tune(ksplit, 0, pair)
        for _ in range(3):
            for d in ds:
                c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump_int64(), 3 * one)
        for d in ds:
            c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump_int64(), 4 * one)
        c.clear()
        for d in ds[::-1]:
            c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        c.run_device(ds[0].data_ptr(), xg.SYNCOP_SYNC_COMPUTE)
        assert np.array_equal(c.dump_int64(), one + oracle_mod.xengine_i64(xs[0], n, f, t))


@pytest.mark.parametrize("engine", ["tensor", "plain"])
def test_overlapping_calls_of_several_segments(xg, oracle_mod, engine):
    """Calls longer than one launch (several time segments) chained back to back."""
    import torch
    n, f, t = 32, 2, 65536 + 512
    xs = [oracle_mod.gaussian_input(n, f, t, seed=70 + q, sigma=20.0) for q in range(2)]
    ds = [torch.from_numpy(x).cuda() for x in xs]
    torch.cuda.synchronize()
    with xg.Correlator(n, f, t, ntimepipe=128, engine=engine) as c:
        for d in ds + ds:
            c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        got = c.dump_int64()
    want = 2 * sum(oracle_mod.xengine_i64(x, n, f, t) for x in xs)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("pair", [0, 1])
def test_long_overlapping_integration_past_int32(xg, oracle_mod, pair):
    """70 full-scale calls of 1024 samples overlapping on the device (sums past
    2^31) stay exact in int64, and three more after a dump too; the int32 dump
    wraps like xGPU's int32 buffer."""
    import torch
    n, f, t = 32, 2, 1024
    x = np.empty(t * f * n * 4, dtype=np.int8)
    x[0::2] = -128
    x[1::2] = 127
    x[5::16] = 3
    d = torch.from_numpy(x).cuda()
    torch.cuda.synchronize()
    one = oracle_mod.xengine_i64(x, n, f, t)
    with xg.Correlator(n, f, t, engine="tensor", output="int32") as c:
        c.tune(1, 0, pair)
        for _ in range(70):
            c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        got = c.dump_int64()
        assert np.abs(got).max() > 2**31
        assert np.array_equal(got, 70 * one)
        for _ in range(3):
            c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump(), (73 * one).astype(np.int32))


@pytest.mark.parametrize("n,f,t,tune", [(48, 2, 1040, (1, 0, 0)),    # partial block and stage
                                        (64, 3, 512, (3, 0, 0)),     # time splits
                                        (128, 2, 2048, (1, 0, 2)),   # stream-K shares
                                        (96, 1, 256, (1, 0, 1)),     # CTA pairs: expanded in-kernel
                                        (32, 1, 65536 + 256, (1, 0, 0))])   # three segments
def test_packed4_tensor_paths(xg, oracle_mod, n, f, t, tune):
    """Packed 4+4-bit input on the tensor engine (expanded by the pre-pass for
    the single-CTA kernel, in shared memory by the CTA-pair kernel), with each
    kernel choice, partial station blocks and stages, and long calls."""
    packed = oracle_mod.generate(t * f * n * 2, 1, n + t)
    exact = oracle_mod.xengine_i64(oracle_mod.unpack4(packed), n, f, t)
    with xg.Correlator(n, f, t, ntimepipe=16, engine="tensor", input_format="packed4") as c:
        c.tune(*tune)
        c.set_input(packed)
        c.run(xg.SYNCOP_SYNC_COMPUTE)     # stores into the cleared buffer
        c.run(xg.SYNCOP_DUMP)             # adds
        assert np.array_equal(c.dump_int64(), 2 * exact)


@pytest.mark.parametrize("n,f,t,tune", [(96, 1, 256, (1, 0, 1)),      # one diagonal tile, partial block
                                        (48, 3, 1040, (1, 0, 1)),     # partial stage
                                        (256, 4, 2048, (3, 0, 1)),    # off-diagonal tiles, time splits
                                        (512, 2, 1024, (1, 24, 1)),   # several items per CTA pair
                                        (64, 2, 32768 + 384, (1, 0, 1))])   # two segments
def test_packed4_expanded_in_pair_kernel(xg, oracle_mod, n, f, t, tune):
    """Packed input on the CTA-pair kernel is expanded in shared memory, with
    no pre-pass.  Random bytes cover every packed value (-8..7 in both
    nibbles); the sums must equal the oracle's, stored and then added."""
    rng = np.random.default_rng(n * 7 + t)
    packed = rng.integers(0, 256, t * f * n * 2, dtype=np.uint8).view(np.int8)
    exact = oracle_mod.xengine_i64(oracle_mod.unpack4(packed), n, f, t)
    with xg.Correlator(n, f, t, ntimepipe=16, engine="tensor", input_format="packed4") as c:
        c.tune(*tune)
        c.set_input(packed)
        c.run(xg.SYNCOP_SYNC_COMPUTE)     # stores into the cleared buffer
        c.run(xg.SYNCOP_DUMP)             # adds
        assert np.array_equal(c.dump_int64(), 2 * exact)


def test_packed4_overlapping_calls_on_cta_pairs(xg, oracle_mod):
    """Accumulating device calls of packed input on CTA pairs (expanded in the
    kernel, no conversion between them) overlap on the context's stream and
    stay exact, across a clear and with several 32768-sample segments."""
    import torch
    n, f, t = 128, 3, 65536 + 256
    ps = [oracle_mod.generate(t * f * n * 2, 1, 60 + q) for q in range(2)]
    ds = [torch.from_numpy(p.view(np.int8)).cuda() for p in ps]
    torch.cuda.synchronize()
    ex = [oracle_mod.xengine_i64(oracle_mod.unpack4(p), n, f, t) for p in ps]
    with xg.Correlator(n, f, t, ntimepipe=16, engine="tensor", input_format="packed4") as c:
        c.tune(1, 24, 1)
        for q in (0, 1, 0, 1, 1):
            c.run_device(ds[q].data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump_int64(), 2 * ex[0] + 3 * ex[1])
        c.clear()
        for q in (1, 0, 0):
            c.run_device(ds[q].data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump_int64(), ex[1] + 2 * ex[0])


def test_packed4_autotune_and_overlapping_device_calls(xg, oracle_mod):
    """Autotuning a packed context (its input buffers hold one byte per sample;
    the timing runs on its int8 conversion buffer), then several calls in
    flight, each converted on the side stream, stay exact."""
    import torch
    n, f, t = 256, 4, 1024
    ps = [oracle_mod.generate(t * f * n * 2, 1, 40 + q) for q in range(3)]
    ds = [torch.from_numpy(p.view(np.int8)).cuda() for p in ps]
    torch.cuda.synchronize()
    one = sum(oracle_mod.xengine_i64(oracle_mod.unpack4(p), n, f, t) for p in ps)
    with xg.Correlator(n, f, t, engine="tensor", input_format="packed4") as c:
        c.tune(0)
        for _ in range(2):
            for d in ds:
                c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        assert np.array_equal(c.dump_int64(), 2 * one)
