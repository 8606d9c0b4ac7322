"""Side-by-side timing of the reference's own CUDA push/pull kernels
(nitorch's CUDA backend compiled for sm_100a by oracle/build_ref_cuda.py)
and this library's, on the same B200, the same inputs and the same chain --
a measurement script, not a test (pytest does not collect it).

    python tests/perf_reference_cuda.py [--size 192] [--steps 5] [--warmup 3]

Workload: the config-2 chain without the prefilter (the reference's
prefilter is Python code in a third-party package that is not present):
1x3xS^3 float32 image, grid = identity + smoothed displacement (std 4),
cubic, dct2, no extrapolation:
    y = pull(x, g);  z = push(y, g);  loss = <z, w>;  d x, d g
run through each backend's native functions (grid_pull, grid_push,
grid_push_backward, grid_pull_backward with the same requires_grad
wiring).  Each op is timed with CUDA events on the current stream, L2
flushed between steps.  The outputs of the two backends are compared
(max relative difference) as a full-size parity check on the GPU.  Prints
one JSON line.
"""
import argparse
import json
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def chain(mod, x, g, w):
    """The step through one backend's native module; returns the outputs and
    the per-op events."""
    b, o = [mod.BoundType.dct2], [mod.InterpolationType.cubic]
    ev = {}

    def rec(name, fn):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        out = fn()
        e.record()
        ev[name] = (s, e)
        return out

    y = rec("pull_fwd", lambda: mod.grid_pull(x, g, b, o, 0))
    z = rec("push_fwd", lambda: mod.grid_push(y, g, list(x.shape[2:]), b, o, 0))
    yr = y.detach().requires_grad_(True)
    gr = g.detach().requires_grad_(True)
    dy, dg1 = rec("push_bwd", lambda: mod.grid_push_backward(w, yr, gr, b, o, 0))
    xr = x.detach().requires_grad_(True)
    dx, dg2 = rec("pull_bwd", lambda: mod.grid_pull_backward(dy, xr, gr, b, o, 0))
    return (y, z, dx, dg1 + dg2), ev


def timed(mod, x, g, w, steps, warmup, flush):
    for _ in range(warmup):
        chain(mod, x, g, w)
    torch.cuda.synchronize()
    per = {}
    tot = []
    for _ in range(steps):
        flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        out, ev = chain(mod, x, g, w)
        e.record()
        torch.cuda.synchronize()
        tot.append(s.elapsed_time(e))
        for k, (a, b) in ev.items():
            per.setdefault(k, []).append(a.elapsed_time(b))
    return out, float(np.median(tot)), {k: round(float(np.median(v)), 4) for k, v in per.items()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=192)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    args = ap.parse_args()
    from nitorch_b200 import spatial, workloads
    from oracle.reference import load_compiled_cuda
    ref = load_compiled_cuda()
    if ref is None:
        print(json.dumps({"unavailable": "reference CUDA backend not built (oracle/build_ref_cuda.py)"}))
        return
    dev = torch.device("cuda")
    x, g = workloads.config2(size=args.size, channels=3)
    w = torch.randn(x.shape, generator=torch.Generator().manual_seed(13), dtype=torch.float64)
    x, g, w = x.float().to(dev), g.float().to(dev), w.float().to(dev)
    flush = torch.empty(64 * 1024 * 1024, device=dev)
    res = {"workload": f"1x3x{args.size}^3 float32, cubic, dct2, no prefilter: pull, push, push_backward, "
                       "pull_backward (config-2 chain)", "steps": args.steps}
    outs = {}
    for name, mod in (("reference_cuda", ref), ("b200", spatial)):
        out, ms, per = timed(mod, x, g, w, args.steps, args.warmup, flush)
        outs[name] = out
        res[name] = {"ms_per_step": round(ms, 4), "Gvox_per_s": round(args.size ** 3 / (ms * 1e-3) / 1e9, 4),
                     "ops_ms": per}
    res["speedup"] = round(res["reference_cuda"]["ms_per_step"] / res["b200"]["ms_per_step"], 2)
    names = ("pull", "push", "dx", "dgrid")
    res["max_rel_diff"] = {}
    for k, a, b in zip(names, outs["b200"], outs["reference_cuda"]):
        a, b = a.double(), b.double()
        res["max_rel_diff"][k] = float((a - b).abs().max() / b.abs().max().clamp_min(1e-30))
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
