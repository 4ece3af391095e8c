"""xgpuCorrelateStatic: the correlation entry point that allocates nothing.

It exists for callers that cannot call cudaMalloc where they correlate (a
real-time thread that must not block on an allocation that can synchronise
the device, or a plugin whose host framework owns all device memory); its
integration buffer is a static device array inside libxgpu.so.  Two calls in
a row, with different inputs and output formats, must each give exactly what
the context-based entry point (xgpuCudaXengineDevice + dump) gives for the
same input, so the second call is not disturbed by what the first left in the
shared array.  The file name makes pytest collect it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def context_result(xg, x_dev, n, f, t, order, output):
    with xg.Correlator(n, f, t, engine="tensor", output=output, order=order) as c:
        c.run_device(x_dev.data_ptr(), xg.SYNCOP_SYNC_COMPUTE)
        return c.dump()


def static_result(xg, torch, x_dev, n, f, t, order, output):
    cfg = xg.default_config()
    cfg.nstation, cfg.nfrequency, cfg.ntime, cfg.ntimepipe = n, f, t, 128
    cfg.engine = xg.XGPU_ENGINE_TENSOR
    cfg.compute_type = xg.XGPU_INT8
    cfg.input_format = xg.XGPU_INPUT_INT8
    cfg.matrix_order = xg.ORDERS[order]
    cfg.output_type = xg.XGPU_INT32 if output == "int32" else xg.XGPU_FLOAT32
    mat_len = (f * (n // 2 + 1) * (n // 4) * 16 if order == "rt" else f * n * (n + 1) // 2 * 4)
    out = torch.full((mat_len * 2,), -1, dtype=torch.int32, device="cuda")
    rc = xg.lib().xgpuCorrelateStatic(ctypes.c_void_p(x_dev.data_ptr()),
                                      ctypes.c_void_p(out.data_ptr()), ctypes.byref(cfg),
                                      torch.cuda.current_device(), None)
    assert rc == xg.XGPU_OK, xg.ERROR_NAMES.get(rc, rc)
    words = out.cpu().numpy()
    return words.view(np.int32 if output == "int32" else np.float32)


def test_static_matches_context_path_twice(xg, oracle_mod):
    import torch
    n, f, t = 256, 10, 1024
    cases = [("tri", "int32", 101), ("rt", "float32", 102)]
    for order, output, seed in cases:
        x = oracle_mod.gaussian_input(n, f, t, seed=seed, sigma=16.0)
        x_dev = torch.from_numpy(x).cuda()
        want = context_result(xg, x_dev, n, f, t, order, output)
        got = static_result(xg, torch, x_dev, n, f, t, order, output)
        assert got.shape == want.shape
        assert np.array_equal(got, want), (order, output)


def test_static_at_the_size_limit(xg, oracle_mod):
    """N=256 with F=15 fills the static array to within 256 bytes of its end
    (64 * 15 * 32896 = 31,580,160 bytes <= 32 MiB - 256): accepted and equal
    to the context path; F=16 (33,685,504 bytes) is rejected."""
    import torch
    n, t = 256, 256
    x = oracle_mod.gaussian_input(n, 15, t, seed=151, sigma=30.0)
    x_dev = torch.from_numpy(x).cuda()
    want = context_result(xg, x_dev, n, 15, t, "tri", "int32")
    got = static_result(xg, torch, x_dev, n, 15, t, "tri", "int32")
    assert np.array_equal(got, want)
    cfg = xg.default_config()
    cfg.nstation, cfg.nfrequency, cfg.ntime, cfg.ntimepipe = n, 16, t, 128
    cfg.engine, cfg.input_format = xg.XGPU_ENGINE_TENSOR, xg.XGPU_INPUT_INT8
    big = torch.zeros(n * 16 * t * 4, dtype=torch.int8, device="cuda")
    out = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = xg.lib().xgpuCorrelateStatic(ctypes.c_void_p(big.data_ptr()),
                                      ctypes.c_void_p(out.data_ptr()), ctypes.byref(cfg),
                                      torch.cuda.current_device(), None)
    assert rc == xg.XGPU_INVALID_ARGUMENT


def test_static_with_cta_pairs_at_n512(xg, oracle_mod):
    """From 384 stations on the static path runs the CTA-pair kernel, as a
    context does before it is tuned: N=512, F=3 (the largest F the static
    array takes at that N), T=1152 (a partial stage), checked against the
    oracle in int64-exact int32 words and against the context path."""
    import torch
    n, f, t = 512, 3, 1152
    x = oracle_mod.gaussian_input(n, f, t, seed=171, sigma=30.0)
    x_dev = torch.from_numpy(x).cuda()
    got = static_result(xg, torch, x_dev, n, f, t, "tri", "int32")
    assert np.array_equal(got, oracle_mod.xengine_i64(x, n, f, t).astype(np.int32))
    assert np.array_equal(got, context_result(xg, x_dev, n, f, t, "tri", "int32"))


def test_static_rejects_sizes_beyond_the_array(xg):
    import torch
    cfg = xg.default_config()
    cfg.nstation, cfg.nfrequency, cfg.ntime, cfg.ntimepipe = 512, 4, 128, 128
    cfg.engine, cfg.input_format = xg.XGPU_ENGINE_TENSOR, xg.XGPU_INPUT_INT8
    x = torch.zeros(512 * 4 * 128 * 4, dtype=torch.int8, device="cuda")
    out = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = xg.lib().xgpuCorrelateStatic(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                      ctypes.byref(cfg), torch.cuda.current_device(), None)
    assert rc == xg.XGPU_INVALID_ARGUMENT
