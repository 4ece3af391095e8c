"""xGPU's own test driver, unmodified, on this library.

oracle/_ref/cuda_correlator is the reference's src/cuda_correlator.c (with its
CPU engine and utilities) compiled exactly as xGPU compiles it -- against the
reference's xgpu.h -- and linked to libxgpu.so from this repository.  Its
built-in self-check (cuda_correlator.c:186-189, 250-253: reorder the GPU
matrix and compare it with xgpuOmpXengine) must report success.
"""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "cuda_correlator")


@pytest.mark.parametrize("args", [[], ["-r"], ["-s", "7"]])
def test_reference_driver_self_check(args):
    if not os.path.exists(EXE):
        pytest.skip("reference driver not built (needs the reference sources at build time)")
    out = subprocess.run([EXE, *args], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "Outer product summation successful" in out.stdout, out.stdout


def test_reference_driver_streaming_calls():
    """Several calls per integration with SYNCOP_NONE / SYNCOP_SYNC_TRANSFER
    (xGPU's test program checks only single-call integrations, so this checks that the
    pipelined calling pattern runs cleanly)."""
    if not os.path.exists(EXE):
        pytest.skip("reference driver not built")
    for op in ("0", "2", "3"):
        out = subprocess.run([EXE, "-c", "8", "-C", "2", "-o", op], capture_output=True, text=True,
                             timeout=600)
        assert out.returncode == 0, out.stdout + out.stderr
        assert "ms/call" in out.stdout
