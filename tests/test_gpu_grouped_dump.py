"""A dumping xgpuCudaXengine call over host buffers whose int8 input spans
two or more MB moves its channels in groups (input of later groups copied in
while results of earlier ones are copied out).  These shapes take that path
with even and uneven groups, every output order and type, every engine,
accumulated calls before the dump, a dump that follows a clear, and offsets
into caller buffers; each result must equal the oracle's bit for bit.
"""
import ctypes

import numpy as np
import pytest

from test_gpu_parity import ENGINES, expected_words, page_aligned

pytestmark = pytest.mark.gpu

# (stations, channels, samples): 2 uneven groups (4+3 channels), 7 groups of
# one channel, 5 groups of two (xGPU's default shape)
SHAPES = [(64, 7, 1536), (128, 7, 2048), (256, 10, 1024)]


@pytest.mark.parametrize("engine,compute", ENGINES)
@pytest.mark.parametrize("order", ["tri", "ri", "rt"])
@pytest.mark.parametrize("output", ["int32", "float32"])
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "n%d_f%d_t%d" % s)
def test_grouped_dump_orders(xg, oracle_mod, engine, compute, order, output, shape):
    n, f, t = shape
    if compute == "fp32" and shape != SHAPES[0]:
        pytest.skip("one FP32 shape keeps the float sums below 2^24")
    sigma = 8.0 if compute == "fp32" else 40.0
    xs = [oracle_mod.gaussian_input(n, f, t, seed=300 + 7 * k + n, sigma=sigma) for k in range(2)]
    exact = sum(oracle_mod.xengine_i64(x, n, f, t) for x in xs)
    if compute == "fp32":
        assert np.abs(exact).max() < 2**24
    with xg.Correlator(n, f, t, engine=engine, compute=compute, output=output, order=order) as c:
        c.set_input(xs[0])
        c.run(xg.SYNCOP_SYNC_TRANSFER)
        c.set_input(xs[1])
        c.run(xg.SYNCOP_DUMP)
        out = c.output_view()[: c.info.matLength * 2].copy()
        assert np.array_equal(out, expected_words(oracle_mod, exact, n, f, order, output))
        if compute == "int8":
            assert np.array_equal(c.dump_int64(), exact)
        # the dump leaves the buffer integrating: one more call adds to it
        c.run(xg.SYNCOP_DUMP)
        more = exact + oracle_mod.xengine_i64(xs[1], n, f, t)
        out = c.output_view()[: c.info.matLength * 2].copy()
        assert np.array_equal(out, expected_words(oracle_mod, more, n, f, order, output))
        # after a clear the first groups store over the buffer
        c.clear()
        c.set_input(xs[0])
        c.run(xg.SYNCOP_DUMP)
        out = c.output_view()[: c.info.matLength * 2].copy()
        want = oracle_mod.xengine_i64(xs[0], n, f, t)
        assert np.array_equal(out, expected_words(oracle_mod, want, n, f, order, output))


@pytest.mark.parametrize("pair,ksplit,grid", [(0, 1, 0), (1, 3, 37), (1, 1, 24), (0, 5, 7)])
def test_grouped_dump_tensor_tunings(xg, oracle_mod, pair, ksplit, grid):
    """Channel ranges through each tensor-core kernel, with time splits that
    clear only their range's part of the buffer."""
    n, f, t = 256, 10, 1024
    x = oracle_mod.gaussian_input(n, f, t, seed=91 + ksplit, sigma=60.0)
    exact = oracle_mod.xengine_i64(x, n, f, t)
    with xg.Correlator(n, f, t, engine="tensor") as c:
        c.tune(ksplit, grid, pair)
        for k in range(3):
            if k == 2:
                c.clear()
            c.set_input(x)
            c.run(xg.SYNCOP_DUMP)
            mult = 1 if k == 2 else k + 1
            assert np.array_equal(c.dump_int64(), mult * exact), k
            assert np.array_equal(c.dump(), (mult * exact).astype(np.int32)), k


@pytest.mark.parametrize("flags", [0, "dont_register"])
def test_grouped_dump_caller_buffers_and_offsets(xg, oracle_mod, flags):
    """Caller buffers registered by xgpuInit or afterwards by
    xgpuSetHost*Buffer, with input and output offsets."""
    n, f, t = 128, 6, 1024
    x = oracle_mod.gaussian_input(n, f, t, seed=17, sigma=30.0)
    exact = oracle_mod.xengine_i64(x, n, f, t).astype(np.int32)
    flag = xg.XGPU_DONT_REGISTER if flags else 0
    cfg = xg.default_config()
    cfg.nstation, cfg.nfrequency, cfg.ntime, cfg.ntimepipe = n, f, t, 128
    cfg.output_type, cfg.matrix_order = xg.XGPU_INT32, xg.TRIANGULAR_ORDER
    off_in, off_out = 96, 5
    inbuf = page_aligned(x.size + 2 * off_in + 64, np.int8)
    inbuf[2 * off_in: 2 * off_in + x.size] = x
    outbuf = page_aligned(2 * (exact.size // 2 + off_out) + 16, np.int32)
    outbuf[:] = -1
    ctx = xg.XGPUContext()
    ctx.array_h = inbuf.ctypes.data
    ctx.array_len = inbuf.size // 2
    ctx.matrix_h = outbuf.ctypes.data
    ctx.matrix_len = outbuf.size // 2
    L = xg.lib()
    assert L.xgpuInitEx(ctypes.byref(ctx), flag, ctypes.byref(cfg)) == 0
    try:
        if flag:
            assert L.xgpuSetHostInputBuffer(ctypes.byref(ctx)) == 0
            assert L.xgpuSetHostOutputBuffer(ctypes.byref(ctx)) == 0
        ctx.input_offset, ctx.output_offset = off_in, off_out
        assert L.xgpuCudaXengine(ctypes.byref(ctx), xg.SYNCOP_DUMP) == 0
        assert np.array_equal(outbuf[2 * off_out: 2 * off_out + exact.size], exact)
        # words outside the dump are untouched
        assert (outbuf[: 2 * off_out] == -1).all()
        assert (outbuf[2 * off_out + exact.size:] == -1).all()
        # an output offset the dump does not fit behind is refused after the
        # call has integrated, as the whole-call path does
        ctx.output_offset = ctx.matrix_len - 1
        assert L.xgpuCudaXengine(ctypes.byref(ctx), xg.SYNCOP_DUMP) == xg.XGPU_INVALID_ARGUMENT
    finally:
        L.xgpuFree(ctypes.byref(ctx))


@pytest.mark.parametrize("engine,compute", [("tensor", "int8"), ("plain", "int8")])
def test_grouped_dump_on_caller_stream(xg, oracle_mod, engine, compute):
    """With the context's work on the caller's stream (xgpuSetComputeStream),
    the grouped dump orders its groups' engine launches after earlier work on
    that stream and returns complete results."""
    import torch
    n, f, t = 128, 6, 1024
    xs = [oracle_mod.gaussian_input(n, f, t, seed=500 + k, sigma=25.0) for k in range(2)]
    exact = sum(oracle_mod.xengine_i64(x, n, f, t) for x in xs)
    stream = torch.cuda.Stream()
    with xg.Correlator(n, f, t, engine=engine, compute=compute) as c:
        c.set_stream(stream.cuda_stream)
        c.set_input(xs[0])
        c.run(xg.SYNCOP_SYNC_TRANSFER)
        # unrelated work queued on the caller's stream between the calls
        with torch.cuda.stream(stream):
            torch.cuda._sleep(1000000)
        c.set_input(xs[1])
        c.run(xg.SYNCOP_DUMP)
        out = c.output_view()[: c.info.matLength * 2].copy()
        assert np.array_equal(out, exact.astype(np.int32))
        assert np.array_equal(c.dump_int64(), exact)
        c.set_stream(None)
        c.clear()
        c.set_input(xs[0])
        c.run(xg.SYNCOP_DUMP)
        out = c.output_view()[: c.info.matLength * 2].copy()
        assert np.array_equal(out, oracle_mod.xengine_i64(xs[0], n, f, t).astype(np.int32))


def test_grouped_dump_packed_input_on_cta_pairs(xg, oracle_mod):
    """Packed 4+4-bit input that the CTA-pair kernel expands also goes in
    channel groups (one packed byte per station and polarisation per row of
    the 2-D copies); every byte value, stored and then added."""
    n, f, t = 256, 16, 1024                 # 8.4 MB packed: 8 groups of 2 channels
    rng = np.random.default_rng(2024)
    packed = rng.integers(0, 256, t * f * n * 2, dtype=np.uint8).view(np.int8)
    exact = oracle_mod.xengine_i64(oracle_mod.unpack4(packed), n, f, t)
    with xg.Correlator(n, f, t, engine="tensor", input_format="packed4") as c:
        c.tune(1, 0, 1)
        c.set_input(packed)
        c.run(xg.SYNCOP_DUMP)
        out = c.output_view()[: c.info.matLength * 2].copy()
        assert np.array_equal(out, exact.astype(np.int32))
        c.run(xg.SYNCOP_DUMP)
        assert np.array_equal(c.dump_int64(), 2 * exact)
