"""The C ABI of libxgpu.so, without a GPU.

* the library loads and exports exactly the functions include/xgpu.h declares;
* include/xgpu.h is layout- and value-compatible with the reference header
  (sizes, offsets and macro values recorded from it in tests/golden);
* the host helpers of the reference API (cpu_util.c / omp_xengine.c
  counterparts) agree with the reference's outputs and with the oracle;
* host-side error paths return the documented codes (no device present here,
  bad arguments, use before init, double free).
"""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "xgpu.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(xgpu[A-Za-z0-9]+)\s*\(", text)))


def test_exports_match_header(xg):
    declared = header_functions()
    out = subprocess.run(["nm", "-D", "--defined-only", xg.LIB_PATH], check=True,
                         capture_output=True, text=True).stdout
    exported = sorted({line.split()[-1] for line in out.splitlines() if " T " in line})
    assert exported == declared
    assert sorted(xg.EXPORTED) == declared
    for name in declared:
        assert getattr(xg.lib(), name) is not None


@pytest.mark.parametrize("tag,flags", [("plain", []), ("dp4a", ["-DDP4A"])])
def test_header_layout_matches_reference(golden, tag, flags):
    meta, _ = golden
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "probe")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), *flags, "-o", exe,
                        os.path.join(ROOT, "tests", "golden", "abi_probe.c")], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    ours = {k: int(v) for k, v in (line.split() for line in out.splitlines())}
    assert ours == meta["abi"][tag]


def test_ctypes_structs_match_header(xg, golden):
    meta, _ = golden
    abi = meta["abi"]["plain"]
    assert ctypes.sizeof(xg.XGPUInfo) == abi["sizeof.XGPUInfo"]
    assert ctypes.sizeof(xg.XGPUContext) == abi["sizeof.XGPUContext"]
    for f, _ in xg.XGPUInfo._fields_:
        assert getattr(xg.XGPUInfo, f).offset == abi[f"XGPUInfo.{f}"]
    for f, _ in xg.XGPUContext._fields_:
        assert getattr(xg.XGPUContext, f).offset == abi[f"XGPUContext.{f}"]


def test_default_info(xg):
    i = xg.default_info()
    assert (i.npol, i.nstation, i.nfrequency, i.ntime, i.ntimepipe) == (2, 256, 10, 1024, 128)
    assert i.nbaseline == 256 * 257 // 2
    assert i.vecLength == 10 * 1024 * 256 * 2
    assert i.vecLengthPipe == 10 * 128 * 256 * 2
    # register-tile order by default, as xgpu_info.h:68-74
    assert i.matrix_order == xg.REGISTER_TILE_TRIANGULAR_ORDER
    assert i.matLength == 10 * (256 // 2 + 1) * (256 // 4) * 16
    assert i.triLength == 10 * (256 * 257 // 2) * 4
    assert "xgpu-b200" in xg.version()


def test_random_complex_matches_reference(xg, golden):
    _, arr = golden
    ref = arr["s16_random_complex_seed1"]
    libc = ctypes.CDLL(None)
    libc.srand(1)
    out = np.zeros(ref.size, dtype=np.int8)
    xg.lib().xgpuRandomComplex(out.ctypes.data, ref.size // 2)
    assert np.array_equal(out, ref)


def test_reorder_matches_oracle_at_default_size(xg, oracle_mod):
    i = xg.default_info()
    n, f = i.nstation, i.nfrequency
    rng = np.random.default_rng(5)
    tri = rng.integers(-2**31, 2**31 - 1, size=i.triLength * 2, dtype=np.int64).astype(np.int32)
    m = oracle_mod.tri_to_order(tri, n, f, 3000)
    buf = m.copy()
    xg.lib().xgpuReorderMatrix(buf.ctypes.data)
    assert np.array_equal(buf[: tri.size], tri)
    assert np.array_equal(buf[: tri.size], oracle_mod.reorder(m, n, f, 3000)[: tri.size])


def test_swizzle_extract_omp_at_default_size(xg, oracle_mod):
    i = xg.default_info()
    n, f, t = i.nstation, i.nfrequency, i.ntime
    x = oracle_mod.gaussian_input(n, f, t, seed=21)
    sw = np.zeros_like(x)
    xg.lib().xgpuSwizzleInput(sw.ctypes.data, x.ctypes.data)
    assert np.array_equal(sw, oracle_mod.swizzle(x, n, f, t))
    omp = np.zeros(i.triLength * 2, dtype=np.float32)
    xg.lib().xgpuOmpXengine(omp.ctypes.data, x.ctypes.data)
    exact = oracle_mod.xengine_i64(x, n, f, t)
    assert np.array_equal(omp, exact.astype(np.float32))
    full = np.zeros(f * n * n * 8, dtype=np.float32)
    xg.lib().xgpuExtractMatrix(full.ctypes.data, omp.ctypes.data)
    assert np.array_equal(full, oracle_mod.extract_f32(omp, n, f))


def test_check_result_reports(xg, capfd):
    i = xg.default_info()
    a = np.zeros(i.triLength * 2, dtype=np.float32)
    b = a.copy()
    xg.lib().xgpuCheckResult(a.ctypes.data, b.ctypes.data, 0, None)
    assert "successful" in capfd.readouterr().out
    a[10] = 5.0
    xg.lib().xgpuCheckResult(a.ctypes.data, b.ctypes.data, 0, None)
    assert "failed with 1 deviations" in capfd.readouterr().out


def test_check_result_rounds_float_matrix_in_place(xg, capfd):
    """xGPU's fixed-point float build rounds the GPU matrix in place before
    comparing (cpu_util.c:164-167); the caller sees the rounded values."""
    i = xg.default_info()
    assert not xg.default_config().output_type == xg.XGPU_INT32   # float Complex build
    cpu = np.zeros(i.triLength * 2, dtype=np.float32)
    cpu[::7] = 1000.0
    gpu = cpu + np.float32(0.375)
    gpu[1::7] = -2.625
    xg.lib().xgpuCheckResult(gpu.ctypes.data, cpu.ctypes.data, 0, None)
    out = capfd.readouterr().out
    assert np.array_equal(gpu, np.round(gpu))
    assert gpu[0] == 1000.0 and gpu[1] == -3.0
    assert "failed" in out       # the -3 entries deviate from zero


def test_check_result_verbose_prints_samples_and_sum(xg, capfd):
    i = xg.default_info()
    n, f, t = i.nstation, i.nfrequency, i.ntime
    cpu = np.zeros(i.triLength * 2, dtype=np.float32)
    gpu = cpu.copy()
    gpu[0] = 7.0      # f=0, baseline (0,0), pols (0,0), real part
    x = np.zeros(t * f * n * 4, dtype=np.int8)
    x[0], x[1] = 3, -2          # t=0, f=0, station 0, pol 0: 3 - 2i
    xg.lib().xgpuCheckResult(gpu.ctypes.data, cpu.ctypes.data, 2, x.ctypes.data)
    out = capfd.readouterr().out
    assert "(   3,  -2) (   3,  -2) -> (    13,      0)" in out
    lines = out.splitlines()
    last = max(k for k, ln in enumerate(lines) if ln.startswith(f" {t - 1:4d} "))
    assert lines[last + 1].strip() == "(    13,      0)"     # the sum after the samples


def _ctx(xg):
    return xg.XGPUContext()


def test_errors_before_init(xg):
    L = xg.lib()
    ctx = _ctx(xg)
    p = ctypes.byref(ctx)
    assert L.xgpuCudaXengine(p, xg.SYNCOP_DUMP) == xg.XGPU_NOT_INITIALIZED
    assert L.xgpuClearDeviceIntegrationBuffer(p) == xg.XGPU_NOT_INITIALIZED
    assert L.xgpuSetHostInputBuffer(p) == xg.XGPU_NOT_INITIALIZED
    assert L.xgpuSetHostOutputBuffer(p) == xg.XGPU_NOT_INITIALIZED
    assert L.xgpuDumpDeviceIntegrationBuffer(p) == xg.XGPU_NOT_INITIALIZED
    assert L.xgpuCudaXengineDevice(p, None, 0) == xg.XGPU_NOT_INITIALIZED
    assert L.xgpuFlushIntegrationBuffer(p) == xg.XGPU_NOT_INITIALIZED
    L.xgpuFree(p)
    L.xgpuFree(p)  # idempotent, as cuda_xengine.cu:537


def test_core_peak_arguments_checked_before_any_device_call(xg):
    L = xg.lib()
    v = ctypes.c_double(-1.0)
    assert L.xgpuMeasureCorePeak(0, 2, ctypes.byref(v)) == xg.XGPU_INVALID_ARGUMENT
    assert L.xgpuMeasureCorePeak(0, -1, ctypes.byref(v)) == xg.XGPU_INVALID_ARGUMENT
    assert L.xgpuMeasureCorePeak(0, 0, None) == xg.XGPU_INVALID_ARGUMENT
    assert v.value == -1.0


@pytest.mark.parametrize("field,value", [
    ("nstation", 24), ("nstation", 0), ("nfrequency", 0), ("ntimepipe", 8),
    ("ntime", 100), ("compute_type", 7), ("output_type", 0), ("matrix_order", 1234),
    ("engine", 9), ("input_format", 5), ("ntime", 2**31 - 128), ("ntime", 2**32 - 128),
])
def test_invalid_config_rejected_before_any_device_call(xg, field, value):
    cfg = xg.default_config()
    setattr(cfg, field, value)
    ctx = _ctx(xg)
    assert xg.lib().xgpuInitEx(ctypes.byref(ctx), 0, ctypes.byref(cfg)) == xg.XGPU_INVALID_ARGUMENT
    assert not ctx.internal


def test_tensor_engine_needs_integer_compute(xg):
    cfg = xg.default_config()
    cfg.engine = xg.XGPU_ENGINE_TENSOR
    cfg.compute_type = xg.XGPU_FLOAT32
    ctx = _ctx(xg)
    assert xg.lib().xgpuInitEx(ctypes.byref(ctx), 0, ctypes.byref(cfg)) == xg.XGPU_INVALID_ARGUMENT


def test_init_without_device_returns_error_not_exit(xg):
    """xGPU calls exit(-1) with no device (cuda_xengine.cu:208-213); this
    library returns XGPU_CUDA_ERROR.  Runs in a child so a GPU host still
    exercises the no-device path (CUDA_VISIBLE_DEVICES empty)."""
    code = (
        "import ctypes, sys; sys.path.insert(0, %r); import xgpu_b200 as xg;"
        "ctx = xg.XGPUContext();"
        "r = xg.lib().xgpuInit(ctypes.byref(ctx), 0);"
        "print('RC', r, bool(ctx.internal))" % ROOT)
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run(["python", "-c", code], capture_output=True, text=True, env=env,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    assert "RC 2 False" in out.stdout


@pytest.mark.parametrize("offset,band,nfreq", [
    (1, 0, 10),      # an offset needs the band's channel count
    (3, 12, 10),     # range past the band's last channel
    (0, 5, 10),      # band narrower than the range
    (0, 70000, 10),  # band beyond the channel limit
])
def test_invalid_channel_range_rejected(xg, offset, band, nfreq):
    cfg = xg.default_config()
    cfg.nfrequency, cfg.channel_offset, cfg.input_nfrequency = nfreq, offset, band
    ctx = _ctx(xg)
    assert xg.lib().xgpuInitEx(ctypes.byref(ctx), 0, ctypes.byref(cfg)) == xg.XGPU_INVALID_ARGUMENT
    assert not ctx.internal


def _static_cfg(xg, n, f, t):
    cfg = xg.default_config()
    cfg.nstation, cfg.nfrequency, cfg.ntime, cfg.ntimepipe = n, f, t, 128
    cfg.engine, cfg.input_format = xg.XGPU_ENGINE_TENSOR, xg.XGPU_INPUT_INT8
    return cfg


@pytest.mark.parametrize("change", [
    {"nstation": 256, "nfrequency": 16},          # 64*F*N(N+1)/2 just past 32 MiB - 256
    {"ntime": 2**31 - 128},                        # past the engines' sample count
    {"channel_offset": 2, "input_nfrequency": 8},  # a channel range
    {"input_nfrequency": 12},                      # input wider than the correlated channels
    {"input_format": 1},                           # packed input
])
def test_static_entry_point_rejects_before_any_device_call(xg, change):
    """xgpuCorrelateStatic checks every argument before touching a device:
    the pointers below are never dereferenced."""
    cfg = _static_cfg(xg, 256, 4, 1024)
    for k, v in change.items():
        setattr(cfg, k, v)
    rc = xg.lib().xgpuCorrelateStatic(ctypes.c_void_p(1 << 20), ctypes.c_void_p(1 << 21),
                                      ctypes.byref(cfg), 0, None)
    assert rc == xg.XGPU_INVALID_ARGUMENT


@pytest.mark.parametrize("change", [
    {"ntime": 2**31 - 128},      # past the planner's int stage count
    {"nfrequency": 70000},       # past xgpuInitEx's channel range
    {"nstation": 8208},          # past the station limit
    {"ntime": 1000},             # not a multiple of 16
    {"nstation": 40},            # not a multiple of 16
])
def test_batch_job_sizes_rejected_before_any_device_call(xg, change):
    """xgpuBatchCreate applies xgpuInitEx's size checks to every job before
    touching a device (the buffer addresses below are never dereferenced)."""
    jobs = (xg.XGPUBatchJob * 2)()
    for q in range(2):
        jobs[q].device_input = 1 << 20
        jobs[q].device_state = 1 << 21
        jobs[q].nstation, jobs[q].nfrequency, jobs[q].ntime = 64, 2, 256
    for k, v in change.items():
        setattr(jobs[1], k, v)
    b = ctypes.c_void_p()
    rc = xg.lib().xgpuBatchCreate(ctypes.byref(b), jobs, 2, 0, None, 0)
    assert rc == xg.XGPU_INVALID_ARGUMENT
    assert not b.value
