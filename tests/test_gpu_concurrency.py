"""Contexts used from several host threads at once.

xGPU keeps its input textures in file-scope globals (cuda_xengine.cu:73-87),
so two contexts of one process must not run at the same time there.  Here
every context owns its state, streams, buffers and tensor maps; the
library's shared state (per-device attribute set-up, the SM-count cache, the
batch tuning cache) is synchronised.  The threads below each drive their own
context -- different engines, kernels and shapes -- through dumping calls
concurrently (ctypes releases the GIL for every library call), and every
dump must equal the oracle's.
"""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [  # (engine, compute, tune, n, f, t)
    ("tensor", "int8", (1, 0, 1), 256, 6, 1024),
    ("tensor", "int8", (2, 0, 0), 128, 4, 2048),
    ("plain", "int8", None, 96, 5, 1024),
    ("plain", "fp32", None, 64, 3, 512),
]


def test_contexts_on_concurrent_host_threads(xg, oracle_mod):
    inputs, wants = [], []
    for k, (engine, compute, tune, n, f, t) in enumerate(CASES):
        xs = [oracle_mod.gaussian_input(n, f, t, seed=300 + 10 * k + q, sigma=20.0) for q in range(3)]
        inputs.append(xs)
        # every sum below 2^24: the FP32 engine is exact too
        wants.append([oracle_mod.xengine_i64(x, n, f, t) for x in xs])
    errors, checked = [], []
    start = threading.Barrier(len(CASES))

    def worker(k):
        engine, compute, tune, n, f, t = CASES[k]
        output = "int32" if compute == "int8" else "float32"
        try:
            with xg.Correlator(n, f, t, engine=engine, compute=compute, output=output,
                               order="tri") as c:
                if tune:
                    c.tune(*tune)
                start.wait()
                for it in range(12):
                    q = it % 3
                    c.clear()
                    c.set_input(inputs[k][q])
                    c.run(xg.SYNCOP_DUMP)
                    got = c.output_view()[: c.info.matLength * 2]
                    if not np.array_equal(got, wants[k][q].astype(got.dtype)):
                        errors.append(f"{engine}/{compute} case {k} iteration {it}: dump differs")
                        return
                    checked.append(k)
        except Exception as e:   # noqa: BLE001 -- reported below
            errors.append(f"case {k}: {e!r}")

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(len(CASES))]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=300)
    assert not any(th.is_alive() for th in threads), "a worker did not finish"
    assert not errors, errors
    assert len(checked) == len(CASES) * 12


def test_contexts_created_and_freed_concurrently(xg, oracle_mod):
    """xgpuInitEx / xgpuFree from several threads at once, each thread checking
    one call of its own context."""
    n, f, t = 64, 2, 256
    x = oracle_mod.gaussian_input(n, f, t, seed=7, sigma=16.0)
    want = oracle_mod.xengine_i64(x, n, f, t).astype(np.int32)
    errors, checked = [], []

    def worker(k):
        try:
            for _ in range(4):
                with xg.Correlator(n, f, t, engine="tensor" if k % 2 == 0 else "plain",
                                   order="tri") as c:
                    c.set_input(x)
                    c.run(xg.SYNCOP_DUMP)
                    if not np.array_equal(c.output_view()[: c.info.matLength * 2], want):
                        errors.append(f"thread {k}: dump differs")
                        return
                    checked.append(k)
        except Exception as e:   # noqa: BLE001 -- reported below
            errors.append(f"thread {k}: {e!r}")

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(6)]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=300)
    assert not any(th.is_alive() for th in threads), "a worker did not finish"
    assert not errors, errors
    assert len(checked) == 6 * 4
