"""Generate the golden fixtures in this directory from the reference itself.

Run where the reference sources are (the _ref/ libraries are built from them
by ``make -C oracle``), with XGPU_REF_SRC naming the reference's src/
directory unless it is checked out beside this repository::

    XGPU_REF_SRC=<xGPU>/src python tests/golden/make_golden.py

Every array stored here is an output of the reference's own CPU code
(xGPU ``src/omp_xengine.c`` and ``src/cpu_util.c`` compiled per shape), on
inputs from the seeded generator in ``oracle/``.  Large outputs are stored as
SHA-256 digests.  The tests then check the oracle restatement, and through it
the CUDA library, against these files without needing the reference tree.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402


def reference_src():
    """The reference's src/ directory: $XGPU_REF_SRC, else a checkout beside
    this repository (../reference/src)."""
    path = os.environ.get("XGPU_REF_SRC") or os.path.join(
        os.path.dirname(os.path.dirname(HERE)), "..", "reference", "src")
    if not os.path.exists(os.path.join(path, "omp_xengine.c")):
        sys.exit("make_golden.py: the reference's src/ directory was not found; "
                 "set XGPU_REF_SRC to it")
    return os.path.abspath(path)


def abi_facts(include_dir, flags):
    """Compile abi_probe.c against the xgpu.h in include_dir and parse it."""
    import subprocess
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "probe")
        subprocess.run(["gcc", "-I", include_dir, *flags, "-o", exe,
                        os.path.join(HERE, "abi_probe.c")], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    return {k: int(v) for k, v in (line.split() for line in out.splitlines())}


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    ref_src = reference_src()
    os.environ["XGPU_REF_SRC"] = ref_src
    oracle.build()
    if not oracle.ref_available("s16", "fp32_rt"):
        raise SystemExit("reference libraries missing: run make -C oracle where the reference exists")

    arrays = {}
    meta = {"generator": {}, "shapes": {}}

    # Generator pins: first bytes of each kind, and the Gaussian CDF table.
    for kind, sigma in [(0, 16.0), (0, 40.0), (0, 4.0), (1, 0.0), (2, 0.0)]:
        g = oracle.generate(4096, kind, 7, sigma)
        arrays[f"gen_k{kind}_s{int(sigma)}"] = g
    thr = np.zeros(254, dtype=np.uint32)
    oracle.lib().oracle_gauss_thresholds(16.0, thr.ctypes.data_as(oracle.ctypes.POINTER(oracle.ctypes.c_uint32)))
    arrays["thr_s16"] = thr

    for shape in ["s16", "s32", "c1", "c2"]:
        n, f, t, tp = oracle.REF_SHAPES[shape]
        seed = {"s16": 11, "s32": 12, "c1": 0, "c2": 1}[shape]
        x = oracle.gaussian_input(n, f, t, seed=seed, sigma=16.0)
        ref_int = oracle.RefLib(shape, "dp4a_rt").omp_xengine(x)
        ref_flt = oracle.RefLib(shape, "fp32_rt").omp_xengine(x)
        entry = {"n": n, "f": f, "t": t, "tp": tp, "seed": seed, "sigma": 16.0,
                 "input_sha": sha(x), "omp_dp4a_sha": sha(ref_int), "omp_fp32_sha": sha(ref_flt)}
        if shape in ("s16", "s32"):
            arrays[f"{shape}_input"] = x
            arrays[f"{shape}_omp_dp4a"] = ref_int
            arrays[f"{shape}_omp_fp32"] = ref_flt
            for var, order in [("dp4a_rt", 3000), ("dp4a_ri", 2000), ("fp32_rt", 3000), ("fp32_ri", 2000)]:
                R = oracle.RefLib(shape, var)
                words = ref_int if R.dp4a else ref_flt
                # A dumped matrix in `order`, built by placing each triangular
                # element where the reference's reorder reads it from.
                m = oracle.tri_to_order(words, n, f, order)
                arrays[f"{shape}_{var}_matrix"] = m
                arrays[f"{shape}_{var}_reordered"] = R.reorder(m)[: words.size]
            # The reference's COMPLEX_BLOCK_SIZE=32 reader on the oracle's
            # blocked copy of the same input.
            arrays[f"{shape}_omp_dp4a_b32"] = oracle.RefLib(shape, "dp4a_rt_b32").omp_xengine(
                oracle.block32(x))
            R = oracle.RefLib(shape, "fp32_rt")
            arrays[f"{shape}_swizzled"] = R.swizzle(x)
            arrays[f"{shape}_extract_fp32"] = R.extract(ref_flt)
            arrays[f"{shape}_random_complex_seed1"] = R.random_complex(1, n * f * t * 2)
        meta["shapes"][shape] = entry

    # Full-range int8 (including -128) at a size where the reference's float
    # sums are still exact, so its DP4A output is the exact answer.
    n, f, t, _ = oracle.REF_SHAPES["s16"]
    rng = np.random.default_rng(123)
    x = rng.integers(-128, 128, size=n * f * t * 4, dtype=np.int16).astype(np.int8)
    x[:64] = -128
    arrays["s16_fullrange_input"] = x
    arrays["s16_fullrange_omp_dp4a"] = oracle.RefLib("s16", "dp4a_rt").omp_xengine(x)

    # ABI facts of the reference header, plain and with DP4A.
    meta["abi"] = {}
    for tag, flags in [("plain", []), ("dp4a", ["-DDP4A"])]:
        meta["abi"][tag] = abi_facts(ref_src, flags)

    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)
    with open(os.path.join(HERE, "golden.json"), "w") as fh:
        json.dump(meta, fh, indent=1, sort_keys=True)
    print("wrote", len(arrays), "arrays")


if __name__ == "__main__":
    main()
