#!/usr/bin/env python
"""Headline benchmark: 3-D cubic spline pull + push, forward + backward.

Workload (default, one step): 1x3x192^3 float32 image, grid = identity +
smoothed displacement (std ~4 voxels, ~5 % of samples outside), order 3,
dct2, extrapolate=False, prefilter=True:
    c = spline_coeff_nd(x);  y = pull(c, grid);  z = push(y, grid)
    loss = <z, w>;  loss.backward()  -> d x, d grid
Metric: output-grid voxels per second (Gvox/s) of that step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

--impl b200 (default) prints one JSON line with the device-timed value, the
end-to-end value through the public API with host buffers (`e2e`), the
roofline of the dominant kernel, the CPU baseline (the reference's own C++
backend on a bounded sample), clocks and kernel-launch counts.
--impl reference times the reference's CPU implementation of the same step
on the host cores (bounded sample) and prints the same metric.
With N > 1 (torchrun), every rank runs an independent replica of the step
(the workload does not shard; "replicas only"); value = all ranks' voxels
/ max-over-ranks time.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "3D pull+push fwd+bwd Gvox/s, % HBM roofline; batched vs plain at <=1e-5 rel"
ORDER, BOUND, EXTRAP = 3, "dct2", False


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------- #
# clocks                                                                 #
# ---------------------------------------------------------------------- #
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_bench_{os.getpid()}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------- #
# per-op instrumentation (CUDA events around each product call)          #
# ---------------------------------------------------------------------- #
class OpTimer:
    """Wraps the nitorch_b200 entry points the step calls so that each call
    is bracketed by CUDA events on the launching (current) stream."""

    def __init__(self):
        self.events = {}
        self.enabled = False
        self._orig = []

    def install(self):
        from nitorch_b200 import coeff, spatial
        for mod, name, label in ((spatial, "grid_pull", "pull_fwd"),
                                 (spatial, "grid_push", "push_fwd"),
                                 (spatial, "grid_push_backward", "push_bwd"),
                                 (spatial, "grid_pull_backward", "pull_bwd"),
                                 (coeff, "spline_coeff_nd", "prefilter")):
            fn = getattr(mod, name)
            self._orig.append((mod, name, fn))
            setattr(mod, name, self._wrap(fn, label))

    def uninstall(self):
        for mod, name, fn in self._orig:
            setattr(mod, name, fn)
        self._orig = []

    def _wrap(self, fn, label):
        def inner(*a, **k):
            if not self.enabled:
                return fn(*a, **k)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            out = fn(*a, **k)
            e.record()
            self.events.setdefault(label, []).append((s, e))
            return out
        return inner

    def summary(self):
        out = {}
        for label, evs in self.events.items():
            ms = [s.elapsed_time(e) for s, e in evs]
            out[label] = {"launches": len(ms), "avg_ms": float(np.mean(ms)), "total_ms": float(np.sum(ms))}
        return out


# algorithmic HBM bytes per output voxel (images s bytes, C channels; grids
# and grid gradients float32): each tensor read or written once.
def algo_bytes(label, s, C):
    return {"pull_fwd": 12 + 2 * s * C, "push_fwd": 12 + 2 * s * C,
            "push_bwd": 24 + 3 * s * C, "pull_bwd": 24 + 3 * s * C,
            "prefilter": 3 * 2 * s * C}[label]


# ---------------------------------------------------------------------- #
# the step                                                               #
# ---------------------------------------------------------------------- #
def make_inputs(size, channels, device):
    from nitorch_b200 import workloads
    x, grid = workloads.config2(size=size, channels=channels)
    oob = workloads.oob_fraction(grid[0], (size,) * 3)
    w = torch.randn(x.shape, generator=torch.Generator().manual_seed(13), dtype=torch.float64)
    return (x.float().to(device), grid.float().to(device), w.float().to(device), oob)


def step(x, grid, w):
    import nitorch_b200 as nb
    from nitorch_b200 import spatial
    # a step sees a new grid in practice: recompute the (cached) sample order
    spatial._orders.clear()
    x.grad = None
    grid.grad = None
    y = nb.grid_pull(x, grid, ORDER, BOUND, EXTRAP, prefilter=True)
    z = nb.grid_push(y, grid, None, ORDER, BOUND, EXTRAP)
    loss = (z * w).sum()
    loss.backward()
    return loss


def flush_l2(buf):
    buf.zero_()


def run_b200(args, rank, world, device):
    from nitorch_b200 import _lib
    size, C = args.size, 3
    x, grid, w, oob = make_inputs(size, C, device)
    x.requires_grad_(True)
    grid.requires_grad_(True)
    nvox = size ** 3
    l2buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    for _ in range(args.warmup):
        step(x, grid, w)
    torch.cuda.synchronize()

    timer = OpTimer()
    timer.install()
    clocks = ClockSampler(device.index or 0) if rank == 0 else None
    if clocks:
        clocks.start()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = _lib.kernel_launches()
    timer.enabled = True
    for i in range(args.steps):
        flush_l2(l2buf)                 # between timed steps, outside the timed window
        starts[i].record()
        step(x, grid, w)
        ends[i].record()
    timer.enabled = False
    torch.cuda.synchronize()
    launches = _lib.kernel_launches() - launches0
    if world > 1:
        torch.distributed.barrier()
    clk = clocks.stop() if clocks else None
    timer.uninstall()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = float(np.sum(step_ms))
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * nvox * args.steps / (total_ms * 1e-3) / 1e9

    ops = timer.summary()

    # ---- end to end: public API, host buffers, H2D inputs + D2H loss -------
    xh = x.detach().cpu().pin_memory()
    gh = grid.detach().cpu().pin_memory()
    wh = w.detach().cpu().pin_memory()
    lh = torch.empty((), dtype=torch.float32).pin_memory()

    def e2e_step():
        xd = xh.to(device, non_blocking=True).requires_grad_(True)
        gd = gh.to(device, non_blocking=True).requires_grad_(True)
        wd = wh.to(device, non_blocking=True)
        loss = step(xd, gd, wd)
        lh.copy_(loss.detach(), non_blocking=True)
        return lh

    for _ in range(max(1, min(args.warmup, 3))):
        e2e_step()
    torch.cuda.synchronize()
    e_s = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e_e = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if world > 1:
        torch.distributed.barrier()
    for i in range(args.steps):
        flush_l2(l2buf)
        e_s[i].record()
        e2e_step()
        e_e[i].record()
    torch.cuda.synchronize()
    e2e_ms = float(np.sum([s.elapsed_time(e) for s, e in zip(e_s, e_e)]))
    if world > 1:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * nvox * args.steps / (e2e_ms * 1e-3) / 1e9
    h2d = (xh.numel() + gh.numel() + wh.numel()) * 4

    if rank != 0:
        return None

    # ---- roofline of the dominant op -----------------------------------------
    hbm, src = peaks()
    dom = max(ops, key=lambda k: ops[k]["total_ms"])
    per = algo_bytes(dom, 4, C) * nvox
    achieved = per / (ops[dom]["avg_ms"] * 1e-3) / 1e9
    step_bytes = sum(algo_bytes(k, 4, C) for k in ("pull_fwd", "push_fwd", "push_bwd", "pull_bwd")) * nvox
    roof = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": hbm,
            "unit": "GB/s", "frac": round(achieved / hbm, 4), "peak_source": src,
            "algorithmic_bytes_per_launch": per, "traffic": args.traffic,
            "step_frac": round(step_bytes / (ms_per_step * 1e-3) / 1e9 / hbm, 4)}

    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "Gvox/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; smoothed N(0,1) image, smoothed displacement)",
        "config": {"workload": f"1x{C}x{size}^3 order-3 dct2 prefilter pull+push fwd+bwd (cfg2)",
                   "voxels_per_step": nvox, "channels": C, "oob_fraction": round(oob, 4),
                   "l2": "flushed (256 MiB write) between timed steps; inputs > L2",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": round(e2e_value, 4), "unit": "Gvox/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": 4},
        "roofline": roof,
        "ops": {k: {kk: round(vv, 4) if isinstance(vv, float) else vv for kk, vv in v.items()}
                for k, v in ops.items()},
        "gpu_launches": int(launches),
        "gpu_launches_per_step": round(launches / args.steps, 2),
        "clocks": clk,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.cpu_size, steps=2, warmup=1)
    return line


# ---------------------------------------------------------------------- #
# reference CPU implementation of the same step                          #
# ---------------------------------------------------------------------- #
def reference_step_fn():
    """The step through the reference's own compiled CPU backend (its native
    API: the functions GridPull / GridPush call) with the prefilter from the
    CPU oracle port (the reference's prefilter lives in a third-party Python
    package that is not present on the benchmark host)."""
    from oracle import oracle as O
    from oracle import reference as R
    ref = R.load_compiled()
    if ref is None:
        return None, "port"
    b, o = [ref.BoundType.dct2], [ref.InterpolationType.cubic]

    def prefilter(a):
        return torch.from_numpy(O.spline_coeff_nd(a.numpy(), [3], [3], dim=3).astype(np.float32))

    def run(x, grid, w):
        c = prefilter(x)
        y = ref.grid_pull(c, grid, b, o, 0)
        z = ref.grid_push(y, grid, list(x.shape[2:]), b, o, 0)
        loss = (z * w).sum()
        yr = y.detach().requires_grad_(True)
        gr = grid.detach().requires_grad_(True)
        dy, dg1 = ref.grid_push_backward(w, yr, gr, b, o, 0)
        cr = c.detach().requires_grad_(True)
        dc, dg2 = ref.grid_pull_backward(dy, cr, gr, b, o, 0)
        dx = prefilter(dc)
        return loss, dx, dg1 + dg2
    return run, "reference"


def cpu_baseline(size, steps=2, warmup=1):
    torch.set_num_threads(os.cpu_count() or 1)
    x, grid, w, _ = make_inputs(size, 3, torch.device("cpu"))
    run, kind = reference_step_fn()
    if run is None:
        return {"value": None, "unit": "Gvox/s", "cores": os.cpu_count(), "kind": "port",
                "sample": "reference CPU backend not built"}
    for _ in range(warmup):
        run(x, grid, w)
    t0 = time.perf_counter()
    for _ in range(steps):
        run(x, grid, w)
    dt = (time.perf_counter() - t0) / steps
    return {"value": round(size ** 3 / dt / 1e9, 6), "unit": "Gvox/s", "cores": torch.get_num_threads(),
            "kind": kind,
            "sample": f"1x3x{size}^3 (1/{(192 // size) ** 3} of the 192^3 voxels), same chain, "
                      f"{steps} steps after {warmup} warm-up; pull/push via the reference's compiled "
                      "C++ CPU backend, prefilter via the CPU oracle port", "sec_per_step": round(dt, 4)}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    size = args.cpu_size
    torch.set_num_threads(os.cpu_count() or 1)
    x, grid, w, _ = make_inputs(size, 3, torch.device("cpu"))
    run, kind = reference_step_fn()
    if run is None:
        return {"impl": "reference", "unavailable": "reference CPU backend not built (oracle/_ref missing)"}
    for _ in range(args.warmup):
        run(x, grid, w)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        run(x, grid, w)
    total = time.perf_counter() - t0
    value = size ** 3 * args.steps / total / 1e9
    sample = (f"1x3x{size}^3 bounded sample of the 1x3x192^3 workload per step, "
              f"{torch.get_num_threads()} threads; reference compiled C++ CPU backend "
              "(prefilter via the CPU oracle port)")
    return {"impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": "Gvox/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "1x3x192^3 order-3 dct2 prefilter pull+push fwd+bwd (cfg2)",
                       "sample_size": size},
            "cpu_baseline": {"value": round(value, 6), "unit": "Gvox/s", "cores": torch.get_num_threads(),
                             "kind": kind, "sample": sample},
            "e2e": {"value": round(value, 6), "unit": "Gvox/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=192)
    ap.add_argument("--cpu-size", type=int, default=96)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--traffic", type=float, default=None,
                    help="ncu dram bytes per launch of the dominant kernel, if measured")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "b200" else args.warmup

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=device)
    try:
        line = run_b200(args, rank, world, device)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
