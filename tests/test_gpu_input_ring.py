"""Accumulating calls over a ring of more device input buffers than the
context keeps tensor maps for.

A context caches one TMA descriptor per input buffer it has read (16 entries,
the oldest replaced once all are in use), so that a pipeline rotating over a
ring of input buffers does not encode a descriptor on every call.  Here every
call reads one of 20 distinct buffers -- in order, in reverse, then in a
seeded random order -- so entries are replaced while earlier launches over
other buffers are still queued.  The integration must equal the sum of each
call's sums from the oracle (exact int64; omp_xengine.c:36-93 restated in
oracle/), for both tensor-core kernels and for packed 4+4-bit input expanded
by the CTA-pair kernel.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, F, T = 64, 2, 512
NBUF = 20


def call_order():
    rng = np.random.default_rng(17)
    return (list(range(NBUF)) + list(reversed(range(NBUF))) +
            [int(b) for b in rng.integers(0, NBUF, 40)])


def run_ring(xg, torch, inputs, sums, pair, input_format="int8"):
    dev = [torch.from_numpy(x).cuda() for x in inputs]
    torch.cuda.synchronize()
    seq = call_order()
    want = np.zeros_like(sums[0])
    for b in seq:
        want += sums[b]
    with xg.Correlator(N, F, T, engine="tensor", output="int32", order="tri",
                       input_format=input_format) as c:
        c.tune(1, 0, pair)
        for b in seq:
            c.run_device(dev[b].data_ptr(), xg.SYNCOP_NONE)
        got = c.dump_int64()
    assert np.array_equal(got, want)


@pytest.mark.parametrize("pair", [0, 1], ids=["single_cta", "cta_pair"])
def test_int8_input_ring(xg, oracle_mod, pair):
    import torch
    xs = [oracle_mod.gaussian_input(N, F, T, seed=100 + b, sigma=30.0) for b in range(NBUF)]
    sums = [oracle_mod.xengine_i64(x, N, F, T) for x in xs]
    run_ring(xg, torch, xs, sums, pair)


def test_packed_input_ring(xg, oracle_mod):
    import torch
    packed = [oracle_mod.generate(T * F * N * 2, 1, 200 + b) for b in range(NBUF)]
    sums = [oracle_mod.xengine_i64(oracle_mod.unpack4(p), N, F, T) for p in packed]
    run_ring(xg, torch, packed, sums, 1, input_format="packed4")
