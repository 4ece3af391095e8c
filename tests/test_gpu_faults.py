"""Failure detection without a GPU fault.

Every wait of the tensor-core and plain kernels is bounded (about 2 s); when
one expires the kernel records an error code, the other roles stop, TMEM (if
any) is released and the kernel returns without touching the integration.  xgpuInjectTimeout makes the engine withhold
its input loads so the waits expire on purpose (a flag nothing sets); the
host must report XGPU_CUDA_ERROR and the context must keep working."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pair", [0, 1])
def test_expired_device_wait_is_reported_and_recoverable(xg, oracle_mod, pair):
    n, f, t = 64, 2, 1024
    x = oracle_mod.gaussian_input(n, f, t, seed=5)
    with xg.Correlator(n, f, t, engine="tensor") as c:
        c.tune(1, 0, pair)
        c.set_input(x)
        assert xg.lib().xgpuInjectTimeout(ctypes.byref(c.ctx), 1) == 0
        with pytest.raises(xg.XGPUError) as err:
            c.run(xg.SYNCOP_SYNC_COMPUTE)
        assert err.value.code == xg.XGPU_CUDA_ERROR
        assert xg.lib().xgpuInjectTimeout(ctypes.byref(c.ctx), 0) == 0
        c.clear()
        c.run(xg.SYNCOP_DUMP)
        got = c.dump_int64()
    assert np.array_equal(got, oracle_mod.xengine_i64(x, n, f, t))


@pytest.mark.parametrize("compute", ["int8", "fp32"])
def test_plain_engine_expired_wait_is_reported_and_recoverable(xg, oracle_mod, compute):
    """The plain engines' panel waits (TMA on mbarriers) expire the same way."""
    n, f, t = 64, 2, 512
    x = oracle_mod.gaussian_input(n, f, t, seed=6)
    out = "int32" if compute == "int8" else "float32"
    with xg.Correlator(n, f, t, engine="plain", compute=compute, output=out) as c:
        c.set_input(x)
        assert xg.lib().xgpuInjectTimeout(ctypes.byref(c.ctx), 1) == 0
        with pytest.raises(xg.XGPUError) as err:
            c.run(xg.SYNCOP_SYNC_COMPUTE)
        assert err.value.code == xg.XGPU_CUDA_ERROR
        assert xg.lib().xgpuInjectTimeout(ctypes.byref(c.ctx), 0) == 0
        c.clear()
        c.run(xg.SYNCOP_DUMP)
        got = c.output_view()[: c.info.matLength * 2].copy()
    exact = oracle_mod.xengine_i64(x, n, f, t)
    assert np.array_equal(got, exact.astype(got.dtype))


def test_packed_input_pair_kernel_expired_wait_is_reported_and_recoverable(xg, oracle_mod):
    """Packed input expanded inside the CTA-pair kernel: with the loads
    withheld, the converter warps' waits expire the same way."""
    n, f, t = 128, 2, 1024
    packed = oracle_mod.generate(t * f * n * 2, 1, 77)
    with xg.Correlator(n, f, t, engine="tensor", input_format="packed4") as c:
        c.tune(1, 0, 1)
        c.set_input(packed)
        assert xg.lib().xgpuInjectTimeout(ctypes.byref(c.ctx), 1) == 0
        with pytest.raises(xg.XGPUError) as err:
            c.run(xg.SYNCOP_SYNC_COMPUTE)
        assert err.value.code == xg.XGPU_CUDA_ERROR
        assert xg.lib().xgpuInjectTimeout(ctypes.byref(c.ctx), 0) == 0
        c.clear()
        c.run(xg.SYNCOP_DUMP)
        got = c.dump_int64()
    assert np.array_equal(got, oracle_mod.xengine_i64(oracle_mod.unpack4(packed), n, f, t))


@pytest.mark.parametrize("engine,pair", [("tensor", 1), ("tensor", 0), ("plain", None)])
def test_expired_waits_in_a_chain_of_overlapping_calls(xg, oracle_mod, engine, pair):
    """Device-input calls that overlap (programmatic launches that only add)
    with their waits expiring: each launch gives up on its own bounded waits,
    waits for its predecessor and returns, the error is reported at the next
    synchronising call, and the context then works normally."""
    import torch
    n, f, t = 64, 2, 512
    x = oracle_mod.gaussian_input(n, f, t, seed=8)
    d = torch.from_numpy(x).cuda()
    torch.cuda.synchronize()
    exact = oracle_mod.xengine_i64(x, n, f, t)
    L = xg.lib()
    with xg.Correlator(n, f, t, engine=engine) as c:
        if pair is not None:
            c.tune(1, 0, pair)
        c.run_device(d.data_ptr(), xg.SYNCOP_SYNC_COMPUTE)     # a stored call, intact
        assert L.xgpuInjectTimeout(ctypes.byref(c.ctx), 1) == 0
        c.run_device(d.data_ptr(), xg.SYNCOP_NONE)             # adding calls, overlapping
        c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        with pytest.raises(xg.XGPUError) as err:
            c.run_device(d.data_ptr(), xg.SYNCOP_SYNC_COMPUTE)
        assert err.value.code == xg.XGPU_CUDA_ERROR
        assert L.xgpuInjectTimeout(ctypes.byref(c.ctx), 0) == 0
        c.clear()
        for _ in range(3):
            c.run_device(d.data_ptr(), xg.SYNCOP_NONE)
        got = c.dump_int64()
    assert np.array_equal(got, 3 * exact)
