"""Host-side tools without a GPU: the xgpuinfo program's autoconf-visible
lines, and channel sharding over several GPUs (exercised with two gloo ranks
on the CPU, each correlating its channels with the oracle)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_xgpuinfo_lines_parse_like_xgpu_m4(xg):
    exe = os.path.join(ROOT, "xgpu_b200", "xgpuinfo")
    if not os.path.exists(exe):
        xg.build()
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout

    def sed(label):   # the sed expressions of xgpu.m4:57-67
        for line in out.splitlines():
            if label in line:
                return line.split(": ", 1)[1]
        return None

    assert sed("Number of stations: ") == "256"
    assert sed("Number of frequencies: ") == "10"
    assert sed("time samples per GPU integration: ") == "1024"
    assert "register tile triangular" in out


@pytest.mark.parametrize("nf,world", [(10, 2), (10, 3), (3, 4), (64, 8)])
def test_channel_shards_cover_all_channels(xg, nf, world):
    ranges = [xg.channel_shard(nf, world, r) for r in range(world)]
    assert ranges[0][0] == 0 and ranges[-1][1] == nf
    for a, b in zip(ranges, ranges[1:]):
        assert a[1] == b[0]
    sizes = [b - a for a, b in ranges]
    assert max(sizes) - min(sizes) <= 1


def _rank_main(rank, world, port, n, f, t, result_path):
    import torch
    import torch.distributed as dist
    import sys
    sys.path.insert(0, ROOT)
    import oracle
    import xgpu_b200 as xg
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    import ctypes
    x = oracle.gaussian_input(n, f, t, seed=42)
    f0, f1 = xg.channel_shard(f, world, rank)
    part = oracle.xengine_i64(xg.shard_input(x, n, f, t, f0, f1), n, f1 - f0, t)
    # The library takes this rank's range as a context of the full band
    # (XGPUConfig channel_offset / input_nfrequency): without a device the
    # call gets past argument checking and fails only for want of a GPU.
    cfg = xg.default_config()
    cfg.nstation, cfg.ntime, cfg.ntimepipe = n, t, 128
    cfg.nfrequency, cfg.channel_offset, cfg.input_nfrequency = f1 - f0, f0, f
    ctx = xg.XGPUContext()
    rc = xg.lib().xgpuInitEx(ctypes.byref(ctx), 0, ctypes.byref(cfg))   # device 0 on any host
    accepted = rc in (xg.XGPU_OK, xg.XGPU_CUDA_ERROR)
    if rc == xg.XGPU_OK:
        xg.lib().xgpuFree(ctypes.byref(ctx))
    parts = [None] * world
    dist.all_gather_object(parts, (part, accepted))
    if rank == 0:
        full = xg.merge_triangular([q[0] for q in parts])
        ok = np.array_equal(full, oracle.xengine_i64(x, n, f, t)) and all(q[1] for q in parts)
        np.save(result_path, np.array([ok]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_channel_sharding_matches_single(tmp_path, oracle_mod, xg):
    import socket
    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    res = str(tmp_path / "ok.npy")
    mp.start_processes(_rank_main, args=(2, port, 48, 5, 128, res), nprocs=2, join=True,
                       start_method="spawn")
    assert bool(np.load(res)[0])
