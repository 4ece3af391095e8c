"""TEST INFRASTRUCTURE, not product code.

numpy/ctypes front end of the CPU checkers built by ``oracle/Makefile``:

* ``liboracle.so`` -- this directory's C restatement of the reference's CPU
  engine and utilities (``xgpu_oracle.c``, following xGPU ``src/omp_xengine.c``
  and ``src/cpu_util.c``) with runtime sizes and exact int64 sums;
* ``_ref/libref_<shape>_<variant>.so`` -- the reference's own
  ``omp_xengine.c`` + ``cpu_util.c`` compiled per shape.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg use this package.  The library under test (``libxgpu.so``) never does.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

# name -> (NSTATION, NFREQUENCY, NTIME, NTIME_PIPE); must match oracle/Makefile
REF_SHAPES = {
    "s16": (16, 2, 64, 16),
    "s32": (32, 3, 256, 128),
    "c1": (64, 10, 1024, 128),
    "c2": (256, 10, 1024, 128),
}
ORDERS = {"tri": 1000, "ri": 2000, "rt": 3000}
ORDER_CODE_TO_NAME = {v: k for k, v in ORDERS.items()}

_lib = None


def build():
    """Compile liboracle.so (and _ref/ where the reference sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        c_i8p = ctypes.POINTER(ctypes.c_int8)
        L.oracle_xengine_i64.argtypes = [c_i8p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
        L.oracle_xengine_f32.argtypes = [c_i8p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_float)]
        L.oracle_mat_length.restype = ctypes.c_long
        L.oracle_mat_length.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_tri_to_order.argtypes = [ctypes.POINTER(ctypes.c_uint32), ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_uint32)]
        L.oracle_reorder_matrix.argtypes = [ctypes.POINTER(ctypes.c_uint32), ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int]
        L.oracle_swizzle_input.argtypes = [c_i8p, ctypes.c_int, ctypes.c_int, ctypes.c_int, c_i8p]
        L.oracle_extract_matrix_f32.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_int,
                                                ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
        L.oracle_gauss_thresholds.argtypes = [ctypes.c_double, ctypes.POINTER(ctypes.c_uint32)]
        L.oracle_generate.argtypes = [c_i8p, ctypes.c_size_t, ctypes.c_int, ctypes.c_uint64,
                                      ctypes.c_double]
        L.oracle_generate_range.argtypes = [c_i8p, ctypes.c_size_t, ctypes.c_int, ctypes.c_uint64,
                                            ctypes.c_double, ctypes.c_uint64]
        L.oracle_block32_input.argtypes = [c_i8p, ctypes.c_size_t, c_i8p]
        L.oracle_unpack4.argtypes = [ctypes.POINTER(ctypes.c_uint8), ctypes.c_size_t, c_i8p]
        L.oracle_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def nbaseline(n):
    return n * (n + 1) // 2


def tri_length(n, f):
    """Complex elements in triangular order (xgpu_info.h:46, cuda_xengine.cu:138)."""
    return f * nbaseline(n) * 4


def mat_length(n, f, order):
    """Complex elements of the dumped matrix (cuda_xengine.cu:132-137)."""
    return int(lib().oracle_mat_length(n, f, order))


def generate(nbytes, kind, seed, sigma=16.0, offset=0):
    """Seeded synthetic bytes [offset, offset+nbytes) of a stream; kind 0 Gaussian
    int8, 1 packed 4+4-bit, 2 uniform [-7,7]."""
    out = np.empty(nbytes, dtype=np.int8)
    lib().oracle_generate_range(_p(out, ctypes.c_int8), nbytes, kind, seed, sigma, offset)
    return out


SERVE_SIGMAS = (4.0, 8.0, 16.0, 32.0)


def serve_block_input(nstation, nfrequency, ntime, seed, sigma, block):
    """Input of block `block` of a served request, as xgpuServeRun defines it:
    bytes [off, off+len) of the Gaussian stream of the sigma bucket nearest
    (in log2) to sigma, seed 0x5EED0000 + bucket, off = 256 * (splitmix64(
    seed * 1000003 + block) mod 2^20)."""
    import math
    nb = 4 * nstation * nfrequency * ntime
    bucket = min(range(len(SERVE_SIGMAS)),
                 key=lambda q: abs(math.log2(sigma) - math.log2(SERVE_SIGMAS[q])))
    m = (1 << 64) - 1
    z = (seed * 1000003 + block + 0x9E3779B97F4A7C15) & m
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    z ^= z >> 31
    off = 256 * (z % (1 << 20))
    return generate(nb, 0, 0x5EED0000 + bucket, SERVE_SIGMAS[bucket], off)


def gaussian_input(n, f, t, seed, sigma=16.0):
    """[t][f][s][p][c] int8 input as a flat array."""
    return generate(t * f * n * 4, 0, seed, sigma)


def unpack4(packed):
    packed = np.ascontiguousarray(packed).view(np.uint8)
    out = np.empty(packed.size * 2, dtype=np.int8)
    lib().oracle_unpack4(_p(packed, ctypes.c_uint8), packed.size, _p(out, ctypes.c_int8))
    return out


def xengine_i64(inp, n, f, t, acc=None):
    """Exact triangular visibilities, int64 [f][k][p1][p2][re,im] (flat)."""
    inp = np.ascontiguousarray(inp, dtype=np.int8)
    assert inp.size == t * f * n * 4
    out = acc if acc is not None else np.zeros(tri_length(n, f) * 2, dtype=np.int64)
    lib().oracle_xengine_i64(_p(inp, ctypes.c_int8), n, f, t, _p(out, ctypes.c_int64),
                             1 if acc is not None else 0)
    return out


def xengine_f32(inp, n, f, t):
    """The reference's float arithmetic, triangular float re/im pairs (flat)."""
    inp = np.ascontiguousarray(inp, dtype=np.int8)
    out = np.zeros(tri_length(n, f) * 2, dtype=np.float32)
    lib().oracle_xengine_f32(_p(inp, ctypes.c_int8), n, f, t, _p(out, ctypes.c_float))
    return out


def tri_to_order(tri_words, n, f, order):
    """Triangular 32-bit re/im words -> matrix order (same word type)."""
    src = np.ascontiguousarray(tri_words)
    u = src.view(np.uint32)
    out = np.empty(mat_length(n, f, order) * 2, dtype=np.uint32)
    lib().oracle_tri_to_order(_p(u, ctypes.c_uint32), n, f, order, _p(out, ctypes.c_uint32))
    return out.view(src.dtype)


def reorder(matrix_words, n, f, order):
    """In-place style reorder (returns a copy) to triangular order."""
    m = np.ascontiguousarray(matrix_words).copy()
    u = m.view(np.uint32)
    lib().oracle_reorder_matrix(_p(u, ctypes.c_uint32), n, f, order)
    return m


def block32(inp):
    """Standard input -> xGPU's COMPLEX_BLOCK_SIZE=32 layout (omp_xengine.c:61-78)."""
    inp = np.ascontiguousarray(inp, dtype=np.int8)
    assert inp.size % 64 == 0
    out = np.empty_like(inp)
    lib().oracle_block32_input(_p(inp, ctypes.c_int8), inp.size, _p(out, ctypes.c_int8))
    return out


def swizzle(inp, n, f, t):
    inp = np.ascontiguousarray(inp, dtype=np.int8)
    out = np.empty_like(inp)
    lib().oracle_swizzle_input(_p(inp, ctypes.c_int8), n, f, t, _p(out, ctypes.c_int8))
    return out


def extract_f32(packed, n, f):
    packed = np.ascontiguousarray(packed, dtype=np.float32)
    out = np.zeros(f * n * n * 4 * 2, dtype=np.float32)
    lib().oracle_extract_matrix_f32(_p(packed, ctypes.c_float), n, f, _p(out, ctypes.c_float))
    return out


def num_threads():
    return int(lib().oracle_num_threads())


# ---------------------------------------------------------------------------
# The reference's own CPU code, compiled per shape under _ref/.


def ref_path(shape, variant):
    return os.path.join(HERE, "_ref", f"libref_{shape}_{variant}.so")


def ref_available(shape="s16", variant="fp32_rt"):
    return os.path.exists(ref_path(shape, variant))


class RefLib:
    """One compiled instance of src/omp_xengine.c + src/cpu_util.c."""

    def __init__(self, shape, variant):
        self.shape = shape
        self.variant = variant
        self.n, self.f, self.t, self.tp = REF_SHAPES[shape]
        self.dp4a = variant.startswith("dp4a")
        self.order = ORDERS[variant.split("_")[1]]
        path = ref_path(shape, variant)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        # RTLD_LOCAL keeps the reference's symbols private to this handle.
        self.L = ctypes.CDLL(path, mode=os.RTLD_LOCAL if hasattr(os, "RTLD_LOCAL") else 0)
        self.L.xgpuOmpXengine.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self.L.xgpuReorderMatrix.argtypes = [ctypes.c_void_p]
        self.L.xgpuSwizzleInput.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self.L.xgpuExtractMatrix.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self.L.xgpuRandomComplex.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong]
        self.libc = ctypes.CDLL(None)

    @property
    def word_dtype(self):
        return np.int32 if self.dp4a else np.float32

    def omp_xengine(self, inp):
        """xgpuOmpXengine (omp_xengine.c:36-93): triangular re/im words."""
        inp = np.ascontiguousarray(inp, dtype=np.int8)
        assert inp.size == self.t * self.f * self.n * 4
        out = np.zeros(tri_length(self.n, self.f) * 2, dtype=self.word_dtype)
        self.L.xgpuOmpXengine(out.ctypes.data, inp.ctypes.data)
        return out

    def reorder(self, matrix_words):
        m = np.ascontiguousarray(matrix_words).copy()
        self.L.xgpuReorderMatrix(m.ctypes.data)
        return m

    def swizzle(self, inp):
        inp = np.ascontiguousarray(inp, dtype=np.int8)
        out = np.zeros_like(inp)
        self.L.xgpuSwizzleInput(out.ctypes.data, inp.ctypes.data)
        return out

    def extract(self, packed):
        packed = np.ascontiguousarray(packed)
        out = np.zeros(self.f * self.n * self.n * 4 * 2, dtype=packed.dtype)
        self.L.xgpuExtractMatrix(out.ctypes.data, packed.ctypes.data)
        return out

    def random_complex(self, seed, length):
        """xgpuRandomComplex after srand(seed) (cpu_util.c:13-55)."""
        self.libc.srand(ctypes.c_uint(seed))
        out = np.zeros(length * 2, dtype=np.int8)
        self.L.xgpuRandomComplex(out.ctypes.data, length)
        return out
