"""Time one engine on one shape with the input resident in device memory.

    python -m xgpu_b200.profile_case --n 512 --f 32 --t 8192 [--engine tensor|plain|fp32]
                                     [--reps 5] [--warmup 3] [--ksplit K] [--pair P]
                                     [--grid G] [--accumulate] [--caller-stream]
                                     [--format int8|packed4|dp4a_swizzled|block32] [--dump]
                                     [--flush]

Prints one JSON line: milliseconds per xgpuCudaXengineDevice call (CUDA
events on the engine's stream), X-engine TOPS (16*F*T*N(N+1) ops per call)
(with --flush the timed region ends with xgpuFlushIntegrationBuffer, which
adds the CTA-pair kernel's short-term per-call sums into the integration
buffer) and the host time to queue one call (when it approaches the device time, the
caller, not the GPU, sets the pace).  Useful to size a deployment and as a small, self-contained case for
profilers.
"""
import argparse
import json
import time

import xgpu_b200 as xg


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--f", type=int, default=32)
    ap.add_argument("--t", type=int, default=8192)
    ap.add_argument("--engine", default="tensor", choices=["tensor", "plain", "fp32"])
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--ksplit", type=int, default=-1, help="-1: engine default, 0: autotune")
    ap.add_argument("--pair", type=int, default=0,
                    help="1: CTA-pair kernel (256x256 tiles), 2: stream-K")
    ap.add_argument("--grid", type=int, default=0, help="CTAs per launch (0: one per SM)")
    ap.add_argument("--accumulate", action="store_true",
                    help="add into the integration (default: every call starts a new one)")
    ap.add_argument("--sigma", type=float, default=16.0)
    ap.add_argument("--caller-stream", action="store_true",
                    help="run on a caller stream (xgpuSetComputeStream) instead of the context's")
    ap.add_argument("--format", default="int8", choices=sorted(xg.FORMATS),
                    help="input format (converted on the device before the engine)")
    ap.add_argument("--dump", action="store_true",
                    help="dump (device formatting + copy to the host) after every call")
    ap.add_argument("--flush", action="store_true",
                    help="end the timed region with xgpuFlushIntegrationBuffer")
    args = ap.parse_args()

    import torch
    compute = "fp32" if args.engine == "fp32" else "int8"
    engine = "plain" if args.engine in ("plain", "fp32") else "tensor"
    c = xg.Correlator(args.n, args.f, args.t, ntimepipe=16, engine=engine, compute=compute,
                      output="int32" if compute == "int8" else "float32", order="tri",
                      input_format=args.format)
    if args.ksplit >= 0 or args.pair or args.grid:
        c.tune(max(args.ksplit, 0) if args.ksplit != -1 else 1, args.grid, args.pair)
    if args.caller_stream:
        stream = torch.cuda.Stream()
        c.set_stream(stream.cuda_stream)
    else:
        stream = torch.cuda.ExternalStream(c.stream)
    packed = args.format == "packed4"
    nbytes = int(c.info.vecLength) * (1 if packed else 2)
    x = torch.empty(nbytes, dtype=torch.int8, device="cuda")
    xg.generate_device(x.data_ptr(), nbytes, 1 if packed else 0, 7, args.sigma,
                       torch.cuda.current_device())
    sync = xg.SYNCOP_DUMP if args.dump else xg.SYNCOP_NONE
    for _ in range(args.warmup):
        if not args.accumulate:
            c.clear()
        c.run_device(x.data_ptr(), sync)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    h0 = time.perf_counter()
    for _ in range(args.reps):
        if not args.accumulate:
            c.clear()
        c.run_device(x.data_ptr(), sync)
    host_ms = (time.perf_counter() - h0) * 1e3 / args.reps
    if args.flush:
        c.flush()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.reps
    ops = xg.ops_per_integration(args.n, args.f, args.t)
    tuning = c.tuning() if engine == "tensor" else None
    print(json.dumps({"engine": c.engine_name, "n": args.n, "f": args.f, "t": args.t,
                      "ms": ms, "tops": ops / (ms * 1e-3) / 1e12, "host_enqueue_ms": host_ms,
                      "accumulate": args.accumulate, "flush": args.flush,
                      "tuning": tuning}))
    c.close()


if __name__ == "__main__":
    main()
