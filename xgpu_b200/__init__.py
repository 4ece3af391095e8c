"""Python binding of libxgpu.so, the B200 X-engine behind xGPU's xgpu.h C ABI.

The functions and structures mirror ``include/xgpu.h`` one for one (ctypes),
so code here reads like a C caller of the library: ``xgpuInit``,
``xgpuCudaXengine(ctx, SYNCOP_DUMP)``, ``xgpuReorderMatrix`` ...  The
:class:`Correlator` class wraps one context for tests and benchmarks.

The CUDA library is the only implementation: if ``libxgpu.so`` is missing or
cannot load, every entry point raises instead of falling back to anything.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxgpu.so")

# ---- constants of include/xgpu.h ----------------------------------------
XGPU_INT8, XGPU_FLOAT32, XGPU_INT32 = 0, 1, 2
TRIANGULAR_ORDER = 1000
REAL_IMAG_TRIANGULAR_ORDER = 2000
REGISTER_TILE_TRIANGULAR_ORDER = 3000
XGPU_DEVICE_MASK = (1 << 16) - 1
XGPU_DONT_REGISTER_ARRAY = 1 << 16
XGPU_DONT_REGISTER_MATRIX = 1 << 17
XGPU_DONT_REGISTER = XGPU_DONT_REGISTER_ARRAY | XGPU_DONT_REGISTER_MATRIX
XGPU_OK = 0
XGPU_OUT_OF_MEMORY = 1
XGPU_CUDA_ERROR = 2
XGPU_INSUFFICIENT_TEXTURE_MEMORY = 3
XGPU_NOT_INITIALIZED = 4
XGPU_HOST_BUFFER_NOT_SET = 5
XGPU_INVALID_ARGUMENT = 6
SYNCOP_NONE, SYNCOP_DUMP, SYNCOP_SYNC_TRANSFER, SYNCOP_SYNC_COMPUTE = 0, 1, 2, 3
XGPU_ENGINE_DEFAULT, XGPU_ENGINE_PLAIN, XGPU_ENGINE_TENSOR = 0, 1, 2
XGPU_INPUT_INT8, XGPU_INPUT_PACKED4, XGPU_INPUT_DP4A_SWIZZLED, XGPU_INPUT_BLOCK32 = 0, 1, 2, 3

ERROR_NAMES = {
    XGPU_OK: "XGPU_OK",
    XGPU_OUT_OF_MEMORY: "XGPU_OUT_OF_MEMORY",
    XGPU_CUDA_ERROR: "XGPU_CUDA_ERROR",
    XGPU_INSUFFICIENT_TEXTURE_MEMORY: "XGPU_INSUFFICIENT_TEXTURE_MEMORY",
    XGPU_NOT_INITIALIZED: "XGPU_NOT_INITIALIZED",
    XGPU_HOST_BUFFER_NOT_SET: "XGPU_HOST_BUFFER_NOT_SET",
    XGPU_INVALID_ARGUMENT: "XGPU_INVALID_ARGUMENT",
}


class XGPUInfo(ctypes.Structure):
    """xgpu.h XGPUInfo (byte-identical to xGPU's, xgpu.h:61-92)."""
    _fields_ = [
        ("npol", ctypes.c_uint), ("nstation", ctypes.c_uint), ("nbaseline", ctypes.c_uint),
        ("nfrequency", ctypes.c_uint), ("ntime", ctypes.c_uint), ("ntimepipe", ctypes.c_uint),
        ("input_type", ctypes.c_uint), ("compute_type", ctypes.c_uint),
        ("vecLength", ctypes.c_ulonglong), ("vecLengthPipe", ctypes.c_ulonglong),
        ("matLength", ctypes.c_ulonglong), ("triLength", ctypes.c_ulonglong),
        ("matrix_order", ctypes.c_uint), ("shared_atomic_size", ctypes.c_size_t),
        ("complex_block_size", ctypes.c_size_t),
    ]


class XGPUContext(ctypes.Structure):
    """xgpu.h XGPUContext (byte-identical to xGPU's, xgpu.h:94-113)."""
    _fields_ = [
        ("array_h", ctypes.c_void_p), ("matrix_h", ctypes.c_void_p),
        ("array_len", ctypes.c_size_t), ("matrix_len", ctypes.c_size_t),
        ("input_offset", ctypes.c_size_t), ("output_offset", ctypes.c_size_t),
        ("internal", ctypes.c_void_p),
    ]


class XGPUBatchJob(ctypes.Structure):
    """xgpu.h XGPUBatchJob (extension: one subarray of a batch)."""
    _fields_ = [
        ("device_input", ctypes.c_void_p), ("device_state", ctypes.c_void_p),
        ("nstation", ctypes.c_uint), ("nfrequency", ctypes.c_uint), ("ntime", ctypes.c_uint),
        ("accumulate", ctypes.c_int),
    ]


XGPU_BATCH_AUTOTUNE, XGPU_BATCH_GRAPH, XGPU_BATCH_PAIR = 1, 2, 4
XGPU_SERVE_BATCHED, XGPU_SERVE_PLAIN_SERIAL = 0, 1


class XGPUServeJob(ctypes.Structure):
    _fields_ = [
        ("nstation", ctypes.c_uint), ("nfrequency", ctypes.c_uint), ("ntime", ctypes.c_uint),
        ("nblocks", ctypes.c_uint), ("dump_every", ctypes.c_uint), ("seed", ctypes.c_ulonglong),
        ("sigma", ctypes.c_double), ("arrival_s", ctypes.c_double),
    ]


class XGPUServeOptions(ctypes.Structure):
    _fields_ = [
        ("sample_rate_hz", ctypes.c_double), ("device_budget_bytes", ctypes.c_size_t),
        ("host_budget_bytes", ctypes.c_size_t), ("mode", ctypes.c_int), ("device", ctypes.c_int),
    ]


class XGPUServeStats(ctypes.Structure):
    _fields_ = [
        ("jobs", ctypes.c_longlong), ("blocks", ctypes.c_longlong), ("dumps", ctypes.c_longlong),
        ("ops", ctypes.c_double), ("wall_s", ctypes.c_double), ("tops", ctypes.c_double),
        ("gpu_busy_s", ctypes.c_double), ("dump_p50_ms", ctypes.c_double),
        ("dump_p99_ms", ctypes.c_double), ("dump_max_ms", ctypes.c_double),
        ("period_ratio_p99", ctypes.c_double), ("late_dumps", ctypes.c_longlong),
        ("admitted_peak", ctypes.c_longlong), ("device_peak_bytes", ctypes.c_double),
    ]


class XGPUConfig(ctypes.Structure):
    """xgpu.h XGPUConfig (extension: runtime sizing and engine choice)."""
    _fields_ = [
        ("nstation", ctypes.c_uint), ("nfrequency", ctypes.c_uint), ("ntime", ctypes.c_uint),
        ("ntimepipe", ctypes.c_uint), ("compute_type", ctypes.c_uint),
        ("output_type", ctypes.c_uint), ("matrix_order", ctypes.c_uint),
        ("engine", ctypes.c_uint), ("input_format", ctypes.c_uint),
        ("channel_offset", ctypes.c_uint), ("input_nfrequency", ctypes.c_uint),
    ]


# (name, restype, argtypes) of every function include/xgpu.h declares.
_PROTOTYPES = [
    ("xgpuVersionString", ctypes.c_char_p, []),
    ("xgpuInfo", None, [ctypes.POINTER(XGPUInfo)]),
    ("xgpuInit", ctypes.c_int, [ctypes.POINTER(XGPUContext), ctypes.c_int]),
    ("xgpuClearDeviceIntegrationBuffer", ctypes.c_int, [ctypes.POINTER(XGPUContext)]),
    ("xgpuSetHostInputBuffer", ctypes.c_int, [ctypes.POINTER(XGPUContext)]),
    ("xgpuSetHostOutputBuffer", ctypes.c_int, [ctypes.POINTER(XGPUContext)]),
    ("xgpuFree", None, [ctypes.POINTER(XGPUContext)]),
    ("xgpuCudaXengine", ctypes.c_int, [ctypes.POINTER(XGPUContext), ctypes.c_int]),
    ("xgpuDumpDeviceIntegrationBuffer", ctypes.c_int, [ctypes.POINTER(XGPUContext)]),
    ("xgpuRandomComplex", None, [ctypes.c_void_p, ctypes.c_ulonglong]),
    ("xgpuReorderMatrix", None, [ctypes.c_void_p]),
    ("xgpuCheckResult", None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    ("xgpuSwizzleInput", None, [ctypes.c_void_p, ctypes.c_void_p]),
    ("xgpuExtractMatrix", None, [ctypes.c_void_p, ctypes.c_void_p]),
    ("xgpuOmpXengine", None, [ctypes.c_void_p, ctypes.c_void_p]),
    ("xgpuDefaultConfig", None, [ctypes.POINTER(XGPUConfig)]),
    ("xgpuInitEx", ctypes.c_int, [ctypes.POINTER(XGPUContext), ctypes.c_int,
                                  ctypes.POINTER(XGPUConfig)]),
    ("xgpuContextInfo", ctypes.c_int, [ctypes.POINTER(XGPUContext), ctypes.POINTER(XGPUInfo)]),
    ("xgpuCudaXengineDevice", ctypes.c_int, [ctypes.POINTER(XGPUContext), ctypes.c_void_p,
                                             ctypes.c_int]),
    ("xgpuDumpDeviceIntegrationBufferInt64", ctypes.c_int, [ctypes.POINTER(XGPUContext),
                                                            ctypes.c_void_p]),
    ("xgpuFlushIntegrationBuffer", ctypes.c_int, [ctypes.POINTER(XGPUContext)]),
    ("xgpuGenerateDevice", ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                                          ctypes.c_ulonglong, ctypes.c_double, ctypes.c_int]),
    ("xgpuMeasureCorePeak", ctypes.c_int, [ctypes.c_int, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_double)]),
    ("xgpuSetComputeStream", ctypes.c_int, [ctypes.POINTER(XGPUContext), ctypes.c_void_p]),
    ("xgpuComputeStream", ctypes.c_void_p, [ctypes.POINTER(XGPUContext)]),
    ("xgpuTuning", ctypes.c_int, [ctypes.POINTER(XGPUContext), ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    ("xgpuEngineName", ctypes.c_char_p, [ctypes.POINTER(XGPUContext)]),
    ("xgpuCorrelateStatic", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.POINTER(XGPUConfig), ctypes.c_int,
                                           ctypes.c_void_p]),
    ("xgpuTune", ctypes.c_int, [ctypes.POINTER(XGPUContext), ctypes.c_int, ctypes.c_int,
                                ctypes.c_int]),
    ("xgpuBatchCreate", ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p),
                                       ctypes.POINTER(XGPUBatchJob), ctypes.c_int, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.c_int]),
    ("xgpuBatchRun", ctypes.c_int, [ctypes.c_void_p]),
    ("xgpuBatchSync", ctypes.c_int, [ctypes.c_void_p]),
    ("xgpuBatchInfo", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    ("xgpuBatchDestroy", None, [ctypes.c_void_p]),
    ("xgpuInjectTimeout", ctypes.c_int, [ctypes.POINTER(XGPUContext), ctypes.c_int]),
    ("xgpuServeRun", ctypes.c_int, [ctypes.POINTER(XGPUServeJob), ctypes.c_int,
                                    ctypes.POINTER(XGPUServeOptions),
                                    ctypes.POINTER(XGPUServeStats),
                                    ctypes.POINTER(ctypes.POINTER(ctypes.c_int))]),
]
EXPORTED = [p[0] for p in _PROTOTYPES]

_lib = None


def build(jobs=8):
    """Compile libxgpu.so in place (nvcc, sm_100a)."""
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", HERE], check=True)


def lib():
    """The loaded libxgpu.so; raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built: run `make -C {HERE}` "
                               "(there is no non-CUDA fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in _PROTOTYPES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class XGPUError(RuntimeError):
    def __init__(self, where, code):
        super().__init__(f"{where} returned {ERROR_NAMES.get(code, code)}")
        self.code = code


def check(where, code):
    if code != XGPU_OK:
        raise XGPUError(where, code)
    return code


def version():
    return lib().xgpuVersionString().decode()


def default_info():
    info = XGPUInfo()
    lib().xgpuInfo(ctypes.byref(info))
    return info


def default_config():
    cfg = XGPUConfig()
    lib().xgpuDefaultConfig(ctypes.byref(cfg))
    return cfg


ENGINES = {"default": XGPU_ENGINE_DEFAULT, "plain": XGPU_ENGINE_PLAIN, "tensor": XGPU_ENGINE_TENSOR}
ORDERS = {"tri": TRIANGULAR_ORDER, "ri": REAL_IMAG_TRIANGULAR_ORDER,
          "rt": REGISTER_TILE_TRIANGULAR_ORDER}
FORMATS = {"int8": XGPU_INPUT_INT8, "packed4": XGPU_INPUT_PACKED4,
           "dp4a_swizzled": XGPU_INPUT_DP4A_SWIZZLED, "block32": XGPU_INPUT_BLOCK32}


class Correlator:
    """One xgpu context with host buffers allocated (pinned) by the library.

    ``compute`` is "int8" (exact integer engines) or "fp32" (plain FP32),
    ``output`` the Complex member type ("int32" or "float32"), ``order`` one
    of "tri", "ri", "rt", ``engine`` "tensor" or "plain".  With
    ``input_nfrequency`` set, the input holds that many channels per sample
    and the context correlates ``nfrequency`` of them from ``channel_offset``
    on (XGPUConfig's channel range).
    """

    def __init__(self, nstation, nfrequency, ntime, ntimepipe=None, compute="int8",
                 output="int32", order="tri", engine="tensor", input_format="int8",
                 device=0, flags=0, channel_offset=0, input_nfrequency=0):
        cfg = default_config()
        cfg.nstation, cfg.nfrequency, cfg.ntime = nstation, nfrequency, ntime
        cfg.ntimepipe = ntimepipe if ntimepipe else min(ntime, 128)
        cfg.compute_type = XGPU_INT8 if compute == "int8" else XGPU_FLOAT32
        cfg.output_type = XGPU_INT32 if output == "int32" else XGPU_FLOAT32
        cfg.matrix_order = ORDERS.get(order, order)
        cfg.engine = ENGINES.get(engine, engine)
        cfg.input_format = FORMATS.get(input_format, input_format)
        cfg.channel_offset, cfg.input_nfrequency = channel_offset, input_nfrequency
        self.cfg = cfg
        self.ctx = XGPUContext()
        check("xgpuInitEx", lib().xgpuInitEx(ctypes.byref(self.ctx), device | flags,
                                             ctypes.byref(cfg)))
        self.info = XGPUInfo()
        check("xgpuContextInfo", lib().xgpuContextInfo(ctypes.byref(self.ctx),
                                                       ctypes.byref(self.info)))
        self.out_dtype = np.int32 if output == "int32" else np.float32

    @property
    def engine_name(self):
        return lib().xgpuEngineName(ctypes.byref(self.ctx)).decode()

    # -- host buffers (views of the library's pinned allocations) --
    def input_view(self):
        nbytes = self.ctx.array_len * 2
        buf = (ctypes.c_int8 * nbytes).from_address(self.ctx.array_h)
        return np.frombuffer(buf, dtype=np.int8)

    def output_view(self):
        nwords = self.ctx.matrix_len * 2
        buf = (ctypes.c_uint32 * nwords).from_address(self.ctx.matrix_h)
        return np.frombuffer(buf, dtype=np.uint32).view(self.out_dtype)

    def set_input(self, x):
        v = self.input_view()
        x = np.ascontiguousarray(x).view(np.int8).ravel()
        v[: x.size] = x

    # -- calls --
    def run(self, syncop=SYNCOP_DUMP):
        return check("xgpuCudaXengine", lib().xgpuCudaXengine(ctypes.byref(self.ctx), syncop))

    def run_device(self, ptr, syncop=SYNCOP_NONE):
        return check("xgpuCudaXengineDevice",
                     lib().xgpuCudaXengineDevice(ctypes.byref(self.ctx), ctypes.c_void_p(ptr),
                                                 syncop))

    def dump(self):
        check("xgpuDumpDeviceIntegrationBuffer",
              lib().xgpuDumpDeviceIntegrationBuffer(ctypes.byref(self.ctx)))
        return self.output_view()[: self.info.matLength * 2].copy()

    def dump_int64(self):
        out = np.empty(self.info.triLength * 2, dtype=np.int64)
        check("xgpuDumpDeviceIntegrationBufferInt64",
              lib().xgpuDumpDeviceIntegrationBufferInt64(ctypes.byref(self.ctx), out.ctypes.data))
        return out

    def flush(self):
        """Queue the addition of pending short-term sums into the integration
        buffer on the compute stream (no host wait)."""
        return check("xgpuFlushIntegrationBuffer",
                     lib().xgpuFlushIntegrationBuffer(ctypes.byref(self.ctx)))

    def clear(self):
        return check("xgpuClearDeviceIntegrationBuffer",
                     lib().xgpuClearDeviceIntegrationBuffer(ctypes.byref(self.ctx)))

    def tune(self, ksplit=0, grid=0, pair=0):
        """Tensor-core kernel choice: ksplit=0 autotunes; else fixed time splits,
        grid (0 = one CTA per SM) and kernel (pair=1: CTA pairs, 256x256 tiles;
        pair=2: single CTAs with stream-K shares for accumulating calls)."""
        return check("xgpuTune", lib().xgpuTune(ctypes.byref(self.ctx), ksplit, grid, pair))

    def set_stream(self, stream_handle):
        return check("xgpuSetComputeStream",
                     lib().xgpuSetComputeStream(ctypes.byref(self.ctx),
                                                ctypes.c_void_p(stream_handle)))

    def tuning(self):
        """The tensor-engine setting in use: {"ksplit", "grid", "pair"}."""
        k, g, p = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check("xgpuTuning", lib().xgpuTuning(ctypes.byref(self.ctx), ctypes.byref(k),
                                             ctypes.byref(g), ctypes.byref(p)))
        return {"ksplit": k.value, "grid": g.value, "pair": p.value}

    @property
    def stream(self):
        """Handle (cudaStream_t as int) of the stream the context queues work on;
        wrap it with torch.cuda.ExternalStream to record events on it."""
        return lib().xgpuComputeStream(ctypes.byref(self.ctx)) or 0

    def close(self):
        if self.ctx.internal:
            lib().xgpuFree(ctypes.byref(self.ctx))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """A planned batch of uneven subarrays (xgpuBatchCreate ... xgpuBatchDestroy).

    ``jobs`` is a list of dicts with keys input (device pointer), state (device
    pointer to the int64 triangular buffer), nstation, nfrequency, ntime and
    optionally accumulate (default 0)."""

    def __init__(self, jobs, device=0, stream=None, autotune=False, graph=False, pair=False):
        arr = (XGPUBatchJob * len(jobs))()
        for a, j in zip(arr, jobs):
            a.device_input = j["input"]
            a.device_state = j["state"]
            a.nstation, a.nfrequency, a.ntime = j["nstation"], j["nfrequency"], j["ntime"]
            a.accumulate = int(j.get("accumulate", 0))
        self.handle = ctypes.c_void_p()
        flags = ((XGPU_BATCH_AUTOTUNE if autotune else 0) | (XGPU_BATCH_GRAPH if graph else 0) |
                 (XGPU_BATCH_PAIR if pair else 0))
        check("xgpuBatchCreate", lib().xgpuBatchCreate(ctypes.byref(self.handle), arr, len(jobs),
                                                       device, ctypes.c_void_p(stream), flags))

    def run(self):
        return check("xgpuBatchRun", lib().xgpuBatchRun(self.handle))

    def sync(self):
        return check("xgpuBatchSync", lib().xgpuBatchSync(self.handle))

    def info(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check("xgpuBatchInfo", lib().xgpuBatchInfo(self.handle, ctypes.byref(a), ctypes.byref(b),
                                                   ctypes.byref(c)))
        return {"work_items": a.value, "grid": b.value, "max_steps": c.value}

    def close(self):
        if self.handle:
            lib().xgpuBatchDestroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def serve(requests, sample_rate_hz, device_budget_bytes, mode=XGPU_SERVE_BATCHED, device=0,
          host_budget_bytes=0, collect=False):
    """Run xgpuServeRun on a list of request dicts (nstation, nfrequency, ntime,
    nblocks, dump_every, seed, sigma, arrival_s).  Returns (stats dict, results)
    where results are the final int32 triangular dumps when collect=True, or,
    when collect is a collection of request indices, a dict index -> dump of
    those requests only."""
    arr = (XGPUServeJob * len(requests))()
    for a, r in zip(arr, requests):
        a.nstation, a.nfrequency, a.ntime = r["nstation"], r["nfrequency"], r["ntime"]
        a.nblocks, a.dump_every = r["nblocks"], r.get("dump_every", 0)
        a.seed, a.sigma, a.arrival_s = r["seed"], r.get("sigma", 16.0), r["arrival_s"]
    opt = XGPUServeOptions(sample_rate_hz, device_budget_bytes, host_budget_bytes, mode, device)
    st = XGPUServeStats()
    res_ptrs = None
    results = None

    def words(r):
        return np.zeros(r["nfrequency"] * r["nstation"] * (r["nstation"] + 1) // 2 * 8,
                        dtype=np.int32)
    if collect is True:
        results = [words(r) for r in requests]
        res_ptrs = (ctypes.POINTER(ctypes.c_int) * len(requests))(
            *[x.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) for x in results])
    elif collect:
        results = {q: words(requests[q]) for q in sorted(set(collect))}
        res_ptrs = (ctypes.POINTER(ctypes.c_int) * len(requests))()
        for q, x in results.items():
            res_ptrs[q] = x.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    check("xgpuServeRun", lib().xgpuServeRun(arr, len(requests), ctypes.byref(opt),
                                             ctypes.byref(st), res_ptrs))
    stats = {name: getattr(st, name) for name, _ in XGPUServeStats._fields_}
    return stats, results


def channel_shard(nfrequency, world, rank):
    """Channels [f0, f1) of one GPU when nfrequency channels are split over
    `world` GPUs (one context per GPU, no collective: channels are
    independent).  The first nfrequency % world GPUs take one extra channel."""
    base, extra = divmod(nfrequency, world)
    f0 = rank * base + min(rank, extra)
    return f0, f0 + base + (1 if rank < extra else 0)


def shard_input(x, nstation, nfrequency, ntime, f0, f1):
    """The [t][f][s][p][c] samples of channels [f0, f1), contiguous."""
    a = np.asarray(x).reshape(ntime, nfrequency, nstation * 4)
    return np.ascontiguousarray(a[:, f0:f1, :]).reshape(-1)


def merge_triangular(parts):
    """Full triangular-order output from per-GPU outputs of consecutive channel
    ranges: triangular order is channel-major ([f][baseline][p1][p2][re,im]), so
    the shards concatenate."""
    return np.concatenate([np.asarray(q).reshape(-1) for q in parts])


def state_elems(nstation, nfrequency):
    """int64 values of a triangular integration buffer."""
    return nfrequency * nstation * (nstation + 1) // 2 * 8


def generate_device(ptr, nbytes, kind, seed, sigma=16.0, device=0):
    """Fill device memory with the seeded generator (same bytes as the host one)."""
    return check("xgpuGenerateDevice",
                 lib().xgpuGenerateDevice(ctypes.c_void_p(ptr), nbytes, kind, seed, sigma, device))


def core_peak(kind, device=0):
    """Measured CUDA-core rate in X-engine operations per second: kind
    "dp4a" (8 per dp4a) or "fp32" (2 per FMA)."""
    v = ctypes.c_double()
    check("xgpuMeasureCorePeak",
          lib().xgpuMeasureCorePeak(device, {"dp4a": 0, "fp32": 1}[kind], ctypes.byref(v)))
    return v.value


def ops_per_integration(n, f, t):
    """Useful X-engine operations for t samples: 16*F*T*N(N+1) (8 per complex
    MAC over N(N+1)/2 baselines x 4 polarisation products), the flop count of
    xGPU's kernel (kernel.cuh:419)."""
    return 16 * f * t * n * (n + 1)
