"""Contexts over channel ranges of one full-band input (XGPUConfig's
channel_offset / input_nfrequency), the C-level form of sharding channels over
GPUs: each GPU's context correlates its channels of the shared
[t][f][s][p] buffer in place, with no re-packing by the caller.  xGPU has one
context per device (XGPU_DEVICE_MASK, xgpu.h:50; cuda_xengine.cu:193,225),
each over a buffer of its own.

Channels are independent, so the triangular dumps of contexts over
consecutive ranges, concatenated, must equal one context over the whole band,
bit for bit (int32 and int64 dumps; float32 for the FP32 engine).  These run
the ranges one after another on one GPU; on several GPUs each range's context
would sit on its own device.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RANGES = [(0, 5), (5, 10)]


def band_input(oracle_mod, fmt, n, f, t, seed):
    """(feed in the context's input format, the int8 samples it holds)."""
    if fmt == "packed4":
        p = oracle_mod.generate(t * f * n * 2, 1, seed)
        return p, oracle_mod.unpack4(p)
    x = oracle_mod.gaussian_input(n, f, t, seed=seed, sigma=24.0)
    if fmt == "dp4a_swizzled":
        return oracle_mod.swizzle(x, n, f, t), x
    if fmt == "block32":
        return oracle_mod.block32(x), x
    return x, x


def ranged(xg, n, f0, f1, fband, t, **kw):
    return xg.Correlator(n, f1 - f0, t, channel_offset=f0, input_nfrequency=fband, **kw)


@pytest.mark.parametrize("engine,compute,tune", [
    ("tensor", "int8", (1, 0, 0)), ("tensor", "int8", (1, 0, 1)), ("tensor", "int8", (2, 0, 1)),
    ("plain", "int8", None), ("plain", "fp32", None)])
@pytest.mark.parametrize("syncop", ["dump", "sync_compute"])
def test_ranges_of_host_input_concatenate_to_the_band(xg, oracle_mod, engine, compute, tune,
                                                      syncop):
    """Host buffers: each context copies its channels of the band (a 2-D copy;
    a dumping call in channel groups)."""
    n, f, t = 256, 10, 1024
    x = oracle_mod.gaussian_input(n, f, t, seed=31, sigma=20.0)
    output = "int32" if compute == "int8" else "float32"
    parts, parts64 = [], []
    for f0, f1 in RANGES:
        with ranged(xg, n, f0, f1, f, t, engine=engine, compute=compute, output=output,
                    order="tri") as c:
            assert c.info.vecLength == t * f * n * 2      # the caller's input is the band
            assert c.info.triLength == (f1 - f0) * n * (n + 1) // 2 * 4
            if tune:
                c.tune(*tune)
            c.set_input(x)
            if syncop == "dump":
                c.run(xg.SYNCOP_DUMP)
                parts.append(c.output_view()[: c.info.matLength * 2].copy())
            else:
                c.run(xg.SYNCOP_SYNC_COMPUTE)
                parts.append(c.dump())
            if compute == "int8":
                parts64.append(c.dump_int64())
    got = xg.merge_triangular(parts)
    if compute == "int8":
        exact = oracle_mod.xengine_i64(x, n, f, t)
        assert np.array_equal(xg.merge_triangular(parts64), exact)
        assert np.array_equal(got, exact.astype(np.int32))
    else:
        assert np.array_equal(got, oracle_mod.xengine_f32(x, n, f, t))


@pytest.mark.parametrize("fmt,tune", [("int8", (1, 0, 0)), ("int8", (1, 0, 1)),
                                      ("packed4", (1, 0, 1)), ("packed4", (1, 0, 0)),
                                      ("dp4a_swizzled", (1, 0, 0)), ("block32", (1, 0, 1))])
def test_ranges_of_device_input_read_in_place(xg, oracle_mod, fmt, tune):
    """Device-resident band: int8 (and packed input on CTA pairs) is read in
    place through strided tensor maps; the other formats gather the range
    before their conversion.  Two accumulating calls per context."""
    import torch
    n, f, t = 128, 7, 512
    ranges = [(0, 3), (3, 4), (4, 7)]
    feeds, xs = zip(*(band_input(oracle_mod, fmt, n, f, t, seed=40 + k) for k in range(2)))
    devs = [torch.from_numpy(np.ascontiguousarray(q)).cuda() for q in feeds]
    parts = []
    for f0, f1 in ranges:
        with ranged(xg, n, f0, f1, f, t, engine="tensor", input_format=fmt) as c:
            c.tune(*tune)
            c.run_device(devs[0].data_ptr(), xg.SYNCOP_NONE)
            c.run_device(devs[1].data_ptr(), xg.SYNCOP_SYNC_COMPUTE)
            parts.append(c.dump_int64())
    want = oracle_mod.xengine_i64(np.concatenate(xs), n, f, 2 * t)
    assert np.array_equal(xg.merge_triangular(parts), want)


@pytest.mark.parametrize("compute", ["int8", "fp32"])
def test_plain_engine_ranges_of_device_input_read_in_place(xg, oracle_mod, compute):
    """The plain engines read a range of a device-resident int8 band in place
    (their panel maps step the band's channels per sample); three calls per
    context, whose dp4a launches overlap (each only adds)."""
    import torch
    n, f, t = 96, 6, 512
    ranges = [(0, 2), (2, 5), (5, 6)]
    xs = [oracle_mod.gaussian_input(n, f, t, seed=60 + k, sigma=20.0) for k in range(3)]
    devs = [torch.from_numpy(x).cuda() for x in xs]
    output = "int32" if compute == "int8" else "float32"
    parts = []
    for f0, f1 in ranges:
        with ranged(xg, n, f0, f1, f, t, engine="plain", compute=compute, output=output,
                    order="tri") as c:
            for k, d in enumerate(devs):
                c.run_device(d.data_ptr(), xg.SYNCOP_SYNC_COMPUTE if k == 2 else xg.SYNCOP_NONE)
            parts.append(c.dump())
    got = xg.merge_triangular(parts)
    x3 = np.concatenate(xs)
    if compute == "int8":
        assert np.array_equal(got, oracle_mod.xengine_i64(x3, n, f, 3 * t).astype(np.int32))
    else:   # sums of 1536 samples at sigma 20 stay below 2^24: exact
        assert np.array_equal(got, oracle_mod.xengine_i64(x3, n, f, 3 * t).astype(np.float32))


@pytest.mark.parametrize("fmt", ["packed4", "dp4a_swizzled", "block32"])
def test_ranges_of_host_input_in_other_formats(xg, oracle_mod, fmt):
    n, f, t = 64, 6, 512
    feed, x = band_input(oracle_mod, fmt, n, f, t, seed=55)
    parts = []
    for f0, f1 in [(0, 1), (1, 4), (4, 6)]:
        with ranged(xg, n, f0, f1, f, t, engine="tensor", input_format=fmt) as c:
            c.set_input(feed)
            c.run(xg.SYNCOP_DUMP)
            parts.append(c.dump_int64())
    assert np.array_equal(xg.merge_triangular(parts), oracle_mod.xengine_i64(x, n, f, t))


def test_range_in_register_tile_order(xg, oracle_mod):
    """The host input buffer holds the band; the dump of a range in
    register-tile order is that range's own matrix."""
    n, f, t = 64, 8, 256
    x = oracle_mod.gaussian_input(n, f, t, seed=61)
    with ranged(xg, n, 2, 7, f, t, engine="tensor", order="rt") as c:
        view = c.input_view()
        assert view.size == x.size
        c.set_input(x)
        c.run(xg.SYNCOP_DUMP)
        got = c.output_view()[: c.info.matLength * 2].copy()   # the view dies with the context
    sub = np.ascontiguousarray(x.reshape(t, f, n * 4)[:, 2:7, :]).reshape(-1)
    exact = oracle_mod.xengine_i64(sub, n, 5, t)
    assert np.array_equal(got, oracle_mod.tri_to_order(exact.astype(np.int32), n, 5, 3000))


def test_shared_pinned_band_and_output_without_registration(xg, oracle_mod):
    """The multi-GPU calling pattern of the integration guide, on one GPU: one
    caller-pinned band and one caller-pinned triangular output shared by
    three contexts created with XGPU_DONT_REGISTER; each context dumps its
    range into its part of the output (ranges share pages at their ends), and
    the whole output is the band's matrix."""
    import ctypes
    import torch
    n, f, t = 128, 9, 512
    nb = n * (n + 1) // 2
    ranges = [(0, 4), (4, 5), (5, 9)]
    x = oracle_mod.gaussian_input(n, f, t, seed=71, sigma=18.0)
    band = torch.from_numpy(x).pin_memory()
    out = torch.zeros(f * nb * 8, dtype=torch.int32).pin_memory()
    ctxs = []
    try:
        for f0, f1 in ranges:
            c = ranged(xg, n, f0, f1, f, t, engine="tensor", order="tri",
                       flags=xg.XGPU_DONT_REGISTER)
            ctxs.append(c)
            c.ctx.array_h = band.data_ptr()
            c.ctx.array_len = t * f * n * 2
            c.ctx.matrix_h = out.data_ptr() + f0 * nb * 4 * 8
            c.ctx.matrix_len = (f1 - f0) * nb * 4
            xg.check("xgpuSetHostInputBuffer", xg.lib().xgpuSetHostInputBuffer(ctypes.byref(c.ctx)))
            xg.check("xgpuSetHostOutputBuffer",
                     xg.lib().xgpuSetHostOutputBuffer(ctypes.byref(c.ctx)))
        for c in ctxs:
            c.run(xg.SYNCOP_NONE)
        for c in ctxs:
            c.run(xg.SYNCOP_DUMP)           # a second integration step, dumped
    finally:
        for c in ctxs:
            c.close()
    want = (2 * oracle_mod.xengine_i64(x, n, f, t)).astype(np.int32)
    assert np.array_equal(out.numpy(), want)
