"""The oracle restatement against the reference's own outputs (CPU only).

The fixtures in tests/golden were produced by the reference's CPU code
(src/omp_xengine.c, src/cpu_util.c compiled per shape) on seeded inputs; see
tests/golden/make_golden.py.  These tests pin the oracle before any GPU result
is compared with it.
"""
import hashlib

import numpy as np
import pytest


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_generator_pins(oracle_mod, golden):
    _, arr = golden
    for kind, sigma in [(0, 16.0), (0, 40.0), (0, 4.0), (1, 0.0), (2, 0.0)]:
        got = oracle_mod.generate(4096, kind, 7, sigma)
        assert np.array_equal(got, arr[f"gen_k{kind}_s{int(sigma)}"]), (kind, sigma)


@pytest.mark.parametrize("shape", ["s16", "s32"])
def test_xengine_matches_reference_exactly(oracle_mod, golden, shape):
    meta, arr = golden
    e = meta["shapes"][shape]
    n, f, t = e["n"], e["f"], e["t"]
    x = oracle_mod.gaussian_input(n, f, t, seed=e["seed"], sigma=e["sigma"])
    assert np.array_equal(x, arr[f"{shape}_input"])
    exact = oracle_mod.xengine_i64(x, n, f, t)
    # reference DP4A build: int32 words; its float sums are exact at this size
    assert np.array_equal(exact, arr[f"{shape}_omp_dp4a"].astype(np.int64))
    # reference float build, term for term
    assert np.array_equal(oracle_mod.xengine_f32(x, n, f, t), arr[f"{shape}_omp_fp32"])


@pytest.mark.parametrize("shape", ["c1", "c2"])
def test_xengine_matches_reference_digest(oracle_mod, golden, shape):
    """Configs 1 and 2 (N=64 and N=256, F=10, T=1024, sigma 16, seeds 0 and 1)."""
    meta, _ = golden
    e = meta["shapes"][shape]
    n, f, t = e["n"], e["f"], e["t"]
    x = oracle_mod.gaussian_input(n, f, t, seed=e["seed"], sigma=e["sigma"])
    assert sha(x) == e["input_sha"]
    exact = oracle_mod.xengine_i64(x, n, f, t)
    assert sha(exact.astype(np.int32)) == e["omp_dp4a_sha"]
    assert sha(exact.astype(np.float32)) == e["omp_fp32_sha"]


def test_full_range_including_minus_128(oracle_mod, golden):
    _, arr = golden
    x = arr["s16_fullrange_input"]
    n, f, t, _ = oracle_mod.REF_SHAPES["s16"]
    assert (x == -128).sum() >= 64
    exact = oracle_mod.xengine_i64(x, n, f, t)
    assert np.array_equal(exact, arr["s16_fullrange_omp_dp4a"].astype(np.int64))


@pytest.mark.parametrize("shape", ["s16", "s32"])
@pytest.mark.parametrize("var,order", [("dp4a_rt", 3000), ("dp4a_ri", 2000),
                                       ("fp32_rt", 3000), ("fp32_ri", 2000)])
def test_orders_and_reorder(oracle_mod, golden, shape, var, order):
    """Forward index maps of the three orders and the reference's reorder."""
    meta, arr = golden
    e = meta["shapes"][shape]
    n, f = e["n"], e["f"]
    words = arr[f"{shape}_omp_dp4a"] if var.startswith("dp4a") else arr[f"{shape}_omp_fp32"]
    m = oracle_mod.tri_to_order(words, n, f, order)
    assert np.array_equal(m, arr[f"{shape}_{var}_matrix"])
    back = oracle_mod.reorder(m, n, f, order)[: words.size]
    assert np.array_equal(back, arr[f"{shape}_{var}_reordered"])
    assert np.array_equal(back, words)


@pytest.mark.parametrize("shape", ["s16", "s32"])
def test_swizzle_and_extract(oracle_mod, golden, shape):
    meta, arr = golden
    e = meta["shapes"][shape]
    n, f, t = e["n"], e["f"], e["t"]
    x = arr[f"{shape}_input"]
    assert np.array_equal(oracle_mod.swizzle(x, n, f, t), arr[f"{shape}_swizzled"])
    assert np.array_equal(oracle_mod.extract_f32(arr[f"{shape}_omp_fp32"], n, f),
                          arr[f"{shape}_extract_fp32"])


@pytest.mark.parametrize("shape", ["s16", "s32"])
def test_block32_layout_matches_reference_reader(oracle_mod, golden, shape):
    """The reference built with COMPLEX_BLOCK_SIZE=32 (its reader,
    omp_xengine.c:61-78) sees the oracle's blocked copy of an input as the
    same samples: its output equals the standard build's on the plain input."""
    _, arr = golden
    n, f, t, _ = oracle_mod.REF_SHAPES[shape]
    x = arr[f"{shape}_input"]
    assert np.array_equal(arr[f"{shape}_omp_dp4a_b32"], arr[f"{shape}_omp_dp4a"])
    assert np.array_equal(oracle_mod.xengine_i64(x, n, f, t),
                          arr[f"{shape}_omp_dp4a_b32"].astype(np.int64))
    b = oracle_mod.block32(x)
    assert np.array_equal(np.sort(b), np.sort(x))      # a permutation of the bytes
    if oracle_mod.ref_available(shape, "dp4a_rt_b32"):
        ref = oracle_mod.RefLib(shape, "dp4a_rt_b32").omp_xengine(b)
        assert np.array_equal(ref, arr[f"{shape}_omp_dp4a"])


def test_oracle_accumulates(oracle_mod):
    n, f, t = 16, 2, 64
    a = oracle_mod.gaussian_input(n, f, t, seed=3)
    b = oracle_mod.gaussian_input(n, f, t, seed=4)
    acc = oracle_mod.xengine_i64(a, n, f, t)
    oracle_mod.xengine_i64(b, n, f, t, acc=acc)
    both = oracle_mod.xengine_i64(np.concatenate([a, b]), n, f, 2 * t)
    assert np.array_equal(acc, both)


def test_unpack4_roundtrip(oracle_mod):
    p = oracle_mod.generate(4096, 1, 9)
    u = oracle_mod.unpack4(p)
    assert u.min() >= -7 and u.max() <= 7
    repacked = ((u[0::2].astype(np.int32) & 0xF) << 4) | (u[1::2].astype(np.int32) & 0xF)
    assert np.array_equal(repacked.astype(np.uint8), p.view(np.uint8))


def test_scaled_packed_expansion_is_exact(oracle_mod):
    """The arithmetic the CTA-pair kernel uses for packed input, restated on
    the CPU: each nibble kept in (or moved to) the high half of its byte is 16
    times its 4-bit value, so every sum of products is 256 times the true one
    and an arithmetic shift by 8 recovers it exactly -- over every byte value,
    including the nibble -8 (byte -128)."""
    n, f, t = 16, 2, 256
    rng = np.random.default_rng(5)
    packed = rng.integers(0, 256, t * f * n * 2, dtype=np.uint8)
    packed[:256] = np.arange(256, dtype=np.uint8)          # every value at least once
    hi = (packed & 0xF0).view(np.int8).astype(np.int64)   # 16 x real part
    lo = ((packed.astype(np.uint16) << 4) & 0xF0).astype(np.uint8).view(np.int8).astype(np.int64)
    scaled = np.empty(packed.size * 2, dtype=np.int64)
    scaled[0::2], scaled[1::2] = hi, lo
    assert scaled.min() == -128 and scaled.max() == 112
    exact = oracle_mod.xengine_i64(oracle_mod.unpack4(packed.view(np.int8)), n, f, t)
    # the Gram formulation on the scaled bytes: x[t][f][s][p][c]
    x = scaled.reshape(t, f, n, 2, 2)
    re = np.einsum("tfip,tfjq->fijpq", x[..., 0], x[..., 0]) + \
        np.einsum("tfip,tfjq->fijpq", x[..., 1], x[..., 1])
    im = np.einsum("tfip,tfjq->fijpq", x[..., 1], x[..., 0]) - \
        np.einsum("tfip,tfjq->fijpq", x[..., 0], x[..., 1])
    assert not (re % 256).any() and not (im % 256).any()
    i, j = np.tril_indices(n)
    got = np.stack([re[:, i, j] >> 8, im[:, i, j] >> 8], axis=-1)   # [f][k][p][q][re,im]
    assert np.array_equal(got.reshape(-1), exact)
