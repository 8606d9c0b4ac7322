"""Per-kernel timing of the push/pull entry points on a benchmark workload.

    python -m nitorch_b200.opbench [--size 192] [--channels 3] [--orders 1,3]
                                   [--ops pull,push,...] [--reps 10] [--smooth]

Times each entry point with CUDA events on the current stream (median of
`reps`, L2 flushed between repetitions) on the config-2 workload (smoothed
image, identity + smoothed displacement, dct2, no extrapolation) and prints
JSON: milliseconds, Gvoxel/s and algorithmic GB/s per op.  ``--smooth``
uses a smoother, smaller displacement (sigma 4, std 2: configs 1 and 4).
``--reps 3 --ops <one op>`` is the small case used for ncu captures.
"""
import argparse
import json

import numpy as np
import torch

from . import coeff, spatial, workloads
from .enums import BoundType, InterpolationType

OPS = ("pull", "push", "sgrad", "pull_bwd", "push_bwd", "count", "prefilter")


def algo_bytes(op, C, s=4):
    """Algorithmic HBM bytes per output voxel (float32 grids)."""
    return {"pull": 12 + 2 * s * C, "push": 12 + 2 * s * C, "sgrad": 12 + 4 * s * C,
            "pull_bwd": 24 + 3 * s * C, "push_bwd": 24 + 3 * s * C, "count": 16,
            "prefilter": 3 * 2 * s * C}[op]


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=192)
    ap.add_argument("--channels", type=int, default=3)
    ap.add_argument("--orders", default="3")
    ap.add_argument("--ops", default=",".join(OPS))
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--bound", default="dct2")
    ap.add_argument("--dtype", default="float32")
    ap.add_argument("--smooth", action="store_true")
    ap.add_argument("--order-mode", default="auto", choices=["auto", "natural", "sorted"])
    args = ap.parse_args(argv)

    spatial.set_sample_order(args.order_mode)
    dev = torch.device("cuda")
    dt = getattr(torch, args.dtype)
    size, C = args.size, args.channels
    if args.smooth:
        shape = (size,) * 3
        x = torch.rand((1, C, *shape), generator=torch.Generator().manual_seed(1), dtype=torch.float64)
        grid = workloads.identity_grid(shape)[None] + workloads.smooth_displacement(shape, 4.0, 2.0, seed=2)
    else:
        x, grid = workloads.config2(size=size, channels=C)
    x = x.to(dev, dt)
    grid = grid.to(dev, torch.float32 if dt != torch.float64 else torch.float64)
    w = torch.randn_like(x)
    flush = torch.empty(64 * 1024 * 1024, device=dev)
    bnd = [getattr(BoundType, args.bound)]
    nv = size ** 3
    s = torch.finfo(dt).bits // 8

    def timeit(fn):
        for _ in range(min(3, args.reps)):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(args.reps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return float(np.median(ts))

    res = {}
    for order in [int(o) for o in args.orders.split(",")]:
        o = [InterpolationType(order)]
        xr = x.clone().requires_grad_(True)
        gr = grid.clone().requires_grad_(True)
        y = spatial.grid_pull(x, grid, bnd, o, 0)
        yr = y.clone().requires_grad_(True)
        fns = {
            "pull": lambda: spatial.grid_pull(x, grid, bnd, o, 0),
            "push": lambda: spatial.grid_push(y, grid, [], bnd, o, 0),
            "sgrad": lambda: spatial.grid_grad(x, grid, bnd, o, 0),
            "pull_bwd": lambda: spatial.grid_pull_backward(w, xr, gr, bnd, o, 0),
            "push_bwd": lambda: spatial.grid_push_backward(w, yr, gr, bnd, o, 0),
            "count": lambda: spatial.grid_count(grid, [], bnd, o, 0),
            "prefilter": lambda: coeff.spline_coeff_nd(x, [3], [order], dim=3),
        }
        out = {}
        for op in args.ops.split(","):
            ms = timeit(fns[op])
            out[op] = {"ms": round(ms, 4), "Gvox/s": round(nv / ms / 1e6, 3),
                       "GB/s": round(algo_bytes(op, C, s) * nv / ms / 1e6, 1)}
        res[f"order{order}"] = out
    # cost of the (per-grid, cached) sample sort itself
    if args.order_mode != "natural":
        res["sample_order_ms"] = round(timeit(lambda: spatial.sample_order(grid, (size,) * 3)), 4)
    print(json.dumps({"size": size, "channels": C, "dtype": args.dtype, "smooth": args.smooth,
                      "order_mode": args.order_mode, "results": res}))


if __name__ == "__main__":
    main()
