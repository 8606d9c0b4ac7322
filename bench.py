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
backend on the full workload), `reference_cuda` (the reference's own CUDA
kernels on the same chain and inputs), clocks and kernel-launch counts;
`fused` reports the same step through the fused pull_push operator, and
`batched` the config-4 workload (64 uneven volumes, float32 and bfloat16) as
one captured batched step against the per-call loop; `svf` times config-5
registration iterations (velocity exponentiation, warp, MSE, backward);
`resize` times nitorch's resize (256^3 -> 320^3, cubic) through the
separable TMA-staged kernel beside the per-point affine pull.
--impl reference times the reference's CPU implementation of the same step
(full size) on the host cores and prints the same metric.
With N > 1 (torchrun), every rank runs an independent replica of the
single-volume step (it does not shard; "replicas only"); value = all ranks'
voxels / max-over-ranks time.  The batched volumes are sharded over the
ranks (LPT on points x channels), timed as max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
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
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(prefix="clocks_bench_", suffix=".csv")
            self.fh = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # the timed region starts once the sampler is running: lines up to
        # here were taken before it and are skipped in stop()
        t0 = time.time()
        self.skip = 0
        while time.time() - t0 < 5.0:
            self.fh.flush()
            with open(self.path) as f:
                n = sum(1 for _ in f)
            if n > 0:
                self.skip = n
                break
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        with open(self.path) as f:
            lines = f.readlines()
        os.unlink(self.path)
        return self.parse(lines, getattr(self, "skip", 0))

    @staticmethod
    def parse(lines, skip=0):
        """Median SM clock, max clock and active throttle reasons of the
        samples after the first `skip` lines (taken before the timed region;
        the last line stands in if none came after)."""
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        during = lines[skip:] or lines[-1:]
        for line in during:
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

    CHAIN = {"grid_pull": "pull_fwd", "grid_push": "push_fwd", "grid_push_backward": "push_bwd",
             "grid_pull_backward": "pull_bwd", "spline_coeff_nd": "prefilter"}
    FUSED = {"grid_pull_push": "pp_fwd", "grid_pull_push_backward": "pp_bwd", "spline_coeff_nd": "prefilter"}

    def __init__(self, labels=None):
        self.labels = labels or self.CHAIN
        self.events = {}
        self.kernels = {}
        self.enabled = False
        self._orig = []

    def install(self):
        from nitorch_b200 import coeff, spatial
        for name, label in self.labels.items():
            mod = coeff if name == "spline_coeff_nd" else spatial
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
            from nitorch_b200 import _lib
            self.kernels[label] = _lib.last_kernel()
            return out
        return inner

    def summary(self):
        out = {}
        for label, evs in self.events.items():
            ms = [s.elapsed_time(e) for s, e in evs]
            out[label] = {"launches": len(ms), "avg_ms": float(np.mean(ms)), "total_ms": float(np.sum(ms)),
                          "kernel": self.kernels.get(label, "")}
        return out


# algorithmic HBM bytes per output voxel (images s bytes, C channels; grids
# and grid gradients float32): each tensor read or written once.
def algo_bytes(label, s, C):
    return {"pull_fwd": 12 + 2 * s * C, "push_fwd": 12 + 2 * s * C,
            "push_bwd": 24 + 3 * s * C, "pull_bwd": 24 + 3 * s * C,
            "pp_fwd": 12 + 2 * s * C, "pp_bwd": 24 + 3 * s * C,
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


def step_fused(x, grid, w):
    """The same step through the fused normal operator (one pass forward,
    one pass backward); same outputs as `step` up to summation order."""
    import nitorch_b200 as nb
    from nitorch_b200 import spatial
    spatial._orders.clear()
    x.grad = None
    grid.grad = None
    z = nb.pull_push(x, grid, ORDER, BOUND, EXTRAP, prefilter=True)
    loss = (z * w).sum()
    loss.backward()
    return loss


def timed_steps(fn, args, world, device, l2buf, timer=None, clocks=None, steps=None):
    """Device time (ms, max over ranks) of `steps` calls of fn(), L2 flushed
    between steps outside the timed windows; the library's kernel launches
    and the clock record of the window."""
    from nitorch_b200 import _lib
    steps = steps or args.steps
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
    launches0 = _lib.kernel_launches()
    if timer:
        timer.enabled = True
    for i in range(steps):
        flush_l2(l2buf)
        starts[i].record()
        fn()
        ends[i].record()
    if timer:
        timer.enabled = False
    torch.cuda.synchronize()
    launches = _lib.kernel_launches() - launches0
    clk = clocks.stop() if clocks else None
    if world > 1:
        torch.distributed.barrier()
    total_ms = float(np.sum([s.elapsed_time(e) for s, e in zip(starts, ends)]))
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    return total_ms, launches, clk


# Ceiling of the per-tap scatter kernels: float reductions (RED) per second
# that this GPU's atomic path sustains when fully coalesced (1.46 T scalar
# adds/s, vector forms 1.6 T; measured on B200 with a reduction probe).
ATOMIC_ADDS_PER_S = 1.46e12
HBM_SPEC_GBS = 8000.0  # B200 HBM3e specification (the measured copy bandwidth is the roofline)
SCATTER_OPS = ("push_fwd", "pull_bwd", "pp_fwd", "pp_bwd")


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one op call
# on the default workload (1x3x192^3, cubic, dct2, brick-major order), from
# one ncu capture of its kernels, keyed by the kernel string pp_last_kernel
# reports after the op.  Push and pull backward include the copy of their
# channel-interleaved accumulator into the output (store_interleaved_vox).
# A kernel not listed here reports traffic null.
MEASURED_TRAFFIC = {
    "pp_brick_gather_kernel mode=0 order=3 cb=3": 291_602_176,
    "pp_brick_scatter_kernel mode=2 order=3 cb=3": 413_647_360 + 152_769_792,
    "pp_kernel mode=4 order=3 cb=3": 492_331_520,
    "pp_brick_pullbwd_kernel mode=5 order=3 cb=3": 583_946_240 + 151_942_400,
    # resize 1x3x256^3 -> 320^3, cubic, dct2
    "resize_sep_kernel tma mode=0 order=3 cb=1": 566_675_200,
}


def roofline(ops, labels, nvox, C, ms_per_step, traffic):
    hbm, src = peaks()
    dom = max(ops, key=lambda k: ops[k]["total_ms"])
    kernel = ops[dom].get("kernel", "")
    traffic_src = "--traffic" if traffic is not None else None
    if traffic is None and kernel in MEASURED_TRAFFIC and nvox == 192 ** 3 and C == 3:
        traffic, traffic_src = MEASURED_TRAFFIC[kernel], f"ncu capture of the {dom} kernels (last: {kernel}) on this workload"
    per = algo_bytes(dom, 4, C) * nvox
    achieved = per / (ops[dom]["avg_ms"] * 1e-3) / 1e9
    step_bytes = sum(algo_bytes(k, 4, C) for k in labels) * nvox
    step_gbs = step_bytes / (ms_per_step * 1e-3) / 1e9
    out = {"bound": "hbm", "op": dom, "kernel": kernel, "achieved": round(achieved, 1), "peak": hbm,
           "unit": "GB/s", "frac": round(achieved / hbm, 4), "peak_source": src,
           "algorithmic_bytes_per_launch": per, "traffic": traffic, "traffic_source": traffic_src,
           "step_frac": round(step_gbs / hbm, 4),
           # the same against the 8 TB/s HBM3e specification
           "spec_gbs": HBM_SPEC_GBS, "frac_of_spec": round(achieved / HBM_SPEC_GBS, 4),
           "step_frac_of_spec": round(step_gbs / HBM_SPEC_GBS, 4)}
    if dom in SCATTER_OPS:
        # the scatter's tap additions (64 taps x C channels per point, cubic
        # 3-D) against the ceiling of one global reduction per tap
        adds = 64 * C * nvox
        rate = adds / (ops[dom]["avg_ms"] * 1e-3)
        out["atomic"] = {"adds_per_launch": adds, "achieved_adds_per_s": round(rate / 1e9, 1),
                         "ceiling_adds_per_s": ATOMIC_ADDS_PER_S / 1e9, "unit": "G adds/s",
                         "frac": round(rate / ATOMIC_ADDS_PER_S, 3),
                         "ceiling_source": "coalesced global float reductions measured on B200"}
    return out


def run_b200(args, rank, world, device):
    size, C = args.size, 3
    x, grid, w, oob = make_inputs(size, C, device)
    x.requires_grad_(True)
    grid.requires_grad_(True)
    nvox = size ** 3
    l2buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    xh = x.detach().cpu().pin_memory()
    gh = grid.detach().cpu().pin_memory()
    wh = w.detach().cpu().pin_memory()
    lh = torch.empty((), dtype=torch.float32).pin_memory()
    h2d = (xh.numel() + gh.numel() + wh.numel()) * 4

    def measure(stepfn, labels, with_clocks, traffic):
        for _ in range(args.warmup):
            stepfn(x, grid, w)
        torch.cuda.synchronize()
        timer = OpTimer(labels)
        timer.install()
        clocks = ClockSampler(device.index or 0) if (rank == 0 and with_clocks) else None
        total_ms, launches, clk = timed_steps(lambda: stepfn(x, grid, w), args, world, device, l2buf,
                                              timer, clocks)
        timer.uninstall()

        # end to end: public API from pinned host buffers.  Every step copies
        # its inputs host -> device and reads its loss back inside the timed
        # region; the copies are double-buffered the way a data loader
        # prefetches: step k+1's inputs cross PCIe on a copy stream while
        # step k computes.  Inputs (255 MB per step) exceed L2: no flush.
        cs = torch.cuda.Stream(device=device)
        bufs = [tuple(torch.empty(h.shape, dtype=h.dtype, device=device) for h in (xh, gh, wh))
                for _ in range(2)]
        ready = [torch.cuda.Event() for _ in range(2)]
        free = [torch.cuda.Event() for _ in range(2)]

        def prefetch(slot, after=None):
            with torch.cuda.stream(cs):
                cs.wait_event(free[slot])
                if after is not None:
                    cs.wait_event(after)
                for d, h in zip(bufs[slot], (xh, gh, wh)):
                    d.copy_(h, non_blocking=True)
                ready[slot].record(cs)

        def e2e_run(nsteps, start=None):
            for e in free:
                e.record()
            prefetch(0, start)
            for k in range(nsteps):
                slot = k % 2
                if k + 1 < nsteps:
                    prefetch(1 - slot)
                torch.cuda.current_stream().wait_event(ready[slot])
                xb, gb, wb = bufs[slot]
                loss = stepfn(xb.detach().requires_grad_(True), gb.detach().requires_grad_(True), wb)
                lh.copy_(loss.detach(), non_blocking=True)
                free[slot].record()
            return lh

        e2e_run(max(1, min(args.warmup, 3)))
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        e2e_run(args.steps, t0)
        t1.record()
        torch.cuda.synchronize()
        e2e_ms = t0.elapsed_time(t1)
        if world > 1:
            t = torch.tensor([e2e_ms], dtype=torch.float64, device=device)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e2e_ms = float(t.item())
        ms_per_step = total_ms / args.steps
        ops = timer.summary()
        return {
            "value": round(world * nvox * args.steps / (total_ms * 1e-3) / 1e9, 4),
            "ms_per_step": round(ms_per_step, 4),
            "e2e": {"value": round(world * nvox * args.steps / (e2e_ms * 1e-3) / 1e9, 4), "unit": "Gvox/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 4,
                    "copies": "pinned host -> device every step, double-buffered on a copy stream "
                              "(step k+1's inputs during step k); loss read back every step"},
            "roofline": roofline(ops, [k for k in labels.values() if k != "prefilter"], nvox, C, ms_per_step,
                                 traffic),
            "ops": {k: {kk: round(vv, 4) if isinstance(vv, float) else vv for kk, vv in v.items()}
                    for k, v in ops.items()},
            "gpu_launches": int(launches),
            "gpu_launches_per_step": round(launches / args.steps, 2),
            "clocks": clk,
        }

    chain = measure(step, OpTimer.CHAIN, True, args.traffic)
    fused = None if args.no_fused else measure(step_fused, OpTimer.FUSED, False, None)
    if rank != 0:
        return None

    line = {
        "metric": METRIC, "value": chain["value"], "unit": "Gvox/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": chain["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; smoothed N(0,1) image, smoothed displacement)",
        "config": {"workload": f"1x{C}x{size}^3 order-3 dct2 prefilter pull+push fwd+bwd (cfg2)",
                   "api": "grid_pull -> grid_push (the nitorch call chain), autograd",
                   "voxels_per_step": nvox, "channels": C, "oob_fraction": round(oob, 4),
                   "l2": "flushed (256 MiB write) between timed steps; inputs > L2",
                   "parallelism": f"replicas x{world}"},
        "e2e": chain["e2e"],
        "roofline": chain["roofline"],
        "ops": chain["ops"],
        "gpu_launches": chain["gpu_launches"],
        "gpu_launches_per_step": chain["gpu_launches_per_step"],
        "clocks": chain["clocks"],
    }
    if fused is not None:
        line["fused"] = {"api": "pull_push (fused normal operator, same outputs), autograd",
                         **{k: fused[k] for k in ("value", "ms_per_step", "e2e", "roofline", "ops", "gpu_launches",
                                                  "gpu_launches_per_step")}}
    if not args.no_reference_cuda and world == 1:
        line["reference_cuda"] = reference_cuda_leg(args, device, x, grid, w, chain["ms_per_step"])
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.cpu_size or size, steps=1, warmup=1)
    return line


# ---------------------------------------------------------------------- #
# batched configuration: many uneven volumes                              #
# ---------------------------------------------------------------------- #
def cfg4_volumes(n):
    from nitorch_b200 import workloads
    items = workloads.config4(n_volumes=n)
    return [it[0] for it in items], [it[1] for it in items], [it[2] for it in items]


def fill_cfg4(batch, seed=31):
    """Seeded synthetic inputs drawn on the GPU: images U[0,1); grids =
    identity + smooth displacement (coarse normal field, trilinear
    upsampling, std 2 voxels)."""
    g = torch.Generator(device=batch.device).manual_seed(seed)
    for i, s in enumerate(batch.shapes):
        batch.x[i].copy_(torch.rand(batch.x[i].shape, generator=g, device=batch.device))
        batch.w[i].copy_(torch.randn(batch.w[i].shape, generator=g, device=batch.device))
        coarse = tuple(max(4, v // 8) for v in s)
        d = torch.randn((1, 3, *coarse), generator=g, device=batch.device)
        d = torch.nn.functional.interpolate(d, size=s, mode="trilinear", align_corners=True)
        d = d * (2.0 / d.std())
        mesh = torch.stack(torch.meshgrid(*[torch.arange(n, dtype=torch.float32, device=batch.device)
                                            for n in s], indexing="ij"), -1)
        batch.grid[i].copy_(mesh[None] + d.movedim(1, -1))


def plain_step(batch):
    """The per-call form: the public API volume by volume, autograd (what a
    loop over subjects does with nitorch's own functions)."""
    import nitorch_b200 as nb
    from nitorch_b200 import spatial
    spatial._orders.clear()
    loss = torch.zeros((), device=batch.device)
    for i in range(batch.n):
        x = batch.x[i].detach().requires_grad_(True)
        g = batch.grid[i].detach().requires_grad_(True)
        y = nb.grid_pull(x, g, batch.orders[i], "dct2", False)
        z = nb.grid_push(y, g, None, batch.orders[i], "dct2", False)
        li = (z.float() * batch.w[i].float()).sum()
        li.backward()
        loss = loss + li.detach()
    return loss


def run_batched(args, rank, world, device):
    from nitorch_b200.batch import Autotuner, PullPushBatch, plan_shards
    shapes, chans, orders = cfg4_volumes(args.batch_volumes)
    costs = [int(np.prod(s)) * c for s, c in zip(shapes, chans)]
    shards, _ = plan_shards(costs, world)
    mine = shards[rank]
    shapes_r = [shapes[i] for i in mine]
    chans_r = [chans[i] for i in mine]
    orders_r = [orders[i] for i in mine]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    total_points = sum(int(np.prod(s)) for s in shapes)
    out = {"workload": f"cfg4: {len(shapes)} volumes, axes U{{96..256}}, C U{{1..4}}, orders 1/3 "
                       "alternating, dct2; pull -> push -> <z,w> -> backward",
           "points_per_step": total_points, "channels_total": int(sum(chans)),
           "sharding": f"LPT over {world} rank(s), no collective on the data path"}
    for dtype in (torch.float32, torch.bfloat16):
        tag = "f32" if dtype == torch.float32 else "bf16"
        tuner = Autotuner()
        form, ctas, srt, tried = tuner.choose(shapes_r, chans_r, orders_r, dtype=dtype, device=device,
                                              init=fill_cfg4)
        b = PullPushBatch(shapes_r, chans_r, orders_r, dtype=dtype, device=device, sorted_order=srt, ctas=ctas,
                          form=form)
        fill_cfg4(b)
        b.capture()
        for _ in range(args.warmup):
            b.step()
        torch.cuda.synchronize(device)
        ms_graph, _, _ = timed_steps(b.step, args, world, device, flush, steps=args.batch_steps)
        for _ in range(max(1, min(args.warmup, 2))):
            plain_step(b)
        torch.cuda.synchronize(device)
        ms_plain, _, _ = timed_steps(lambda: plain_step(b), args, world, device, flush, steps=args.batch_steps)
        res = {"batched_graph": {"value": round(total_points * args.batch_steps / (ms_graph * 1e-3) / 1e9, 4),
                                 "unit": "Gvox/s", "ms_per_step": round(ms_graph / args.batch_steps, 3),
                                 "gpu_launches_per_step": b.graph_launches},
               "plain_per_call": {"value": round(total_points * args.batch_steps / (ms_plain * 1e-3) / 1e9, 4),
                                  "unit": "Gvox/s", "ms_per_step": round(ms_plain / args.batch_steps, 3)},
               "speedup": round(ms_plain / ms_graph, 3),
               "roofline": batched_roofline(shapes, chans, 4 if dtype == torch.float32 else 2,
                                            ms_graph / args.batch_steps, world),
               "autotune": {"form": form, "ctas": ctas, "sorted_order": srt, "candidates_ms": tried}}
        if rank == 0 and dtype == torch.float32:
            res["max_rel_err_vs_plain"] = batched_vs_plain(b)
        if rank == 0 and dtype == torch.bfloat16 and not args.no_cpu_baseline:
            res["error_vs_fp64_oracle"] = bf16_error(b)
        out[tag] = res
        b.release()
        del b
        import gc
        gc.collect()
        torch.cuda.empty_cache()
    return out


def batched_roofline(shapes, chans, s, ms_per_step, world):
    """Algorithmic HBM bytes of the batched step (every volume's pull, push
    and both backward passes, each tensor read or written once: algo_bytes
    per point with the volume's channel count and storage size s) against
    the measured copy bandwidth of all ranks."""
    hbm, src = peaks()
    labels = ("pull_fwd", "push_fwd", "push_bwd", "pull_bwd")
    step_bytes = sum(int(np.prod(sh)) * sum(algo_bytes(k, s, c) for k in labels) for sh, c in zip(shapes, chans))
    achieved = step_bytes / (ms_per_step * 1e-3) / 1e9
    return {"bound": "hbm", "algorithmic_bytes_per_step": int(step_bytes), "achieved": round(achieved, 1),
            "peak": hbm * world, "unit": "GB/s", "frac": round(achieved / (hbm * world), 4), "peak_source": src}


def batched_vs_plain(b):
    """Largest relative difference (max |err| / max |ref|, per volume and
    output) between the batched float32 step and the per-volume public API
    on the same stored inputs: z = push(pull(x)), d loss / d x and
    d loss / d grid, over every volume."""
    import nitorch_b200 as nb
    b.step_eager()
    worst = {"z": 0.0, "dx": 0.0, "dgrid": 0.0}
    for i in range(b.n):
        x = b.x[i].detach().clone().requires_grad_(True)
        g = b.grid[i].detach().clone().requires_grad_(True)
        z = nb.grid_push(nb.grid_pull(x, g, b.orders[i], "dct2", False), g, None, b.orders[i], "dct2", False)
        (z * b.w[i]).sum().backward()
        for k, mine, ref in (("z", b.z[i], z), ("dx", b.dx[i], x.grad), ("dgrid", b.dgrid[i], g.grad)):
            mine, ref = mine.detach().double(), ref.detach().double()
            e = float((mine - ref).abs().max() / ref.abs().max().clamp_min(1e-30))
            worst[k] = max(worst[k], e)
    return worst


def bf16_error(b):
    """Max relative error of the batched bfloat16 step's forward output z =
    push(pull(x)) against the FP64 CPU oracle chain on the same stored (bf16)
    input, on the smallest volume of each (order, channel count) present."""
    from oracle import oracle as O
    b.step_eager()
    torch.cuda.synchronize(b.device)
    picks = {}
    for i in sorted(range(b.n), key=lambda k: int(np.prod(b.shapes[k]))):
        picks.setdefault((b.orders[i], b.channels[i]), i)
    rows = []
    for (order, c), i in sorted(picks.items()):
        x = b.x[i].double().cpu().numpy()
        g = b.grid[i].double().cpu().numpy()
        ref = O.grid_push(O.grid_pull(x, g, [2], [order], 0), g, x.shape[2:], [2], [order], 0)
        z = b.z[i].double().cpu().numpy()
        rows.append({"volume": list(b.shapes[i]), "channels": c, "order": order,
                     "push_of_pull_max_rel_err": float(np.abs(z - ref).max() / np.abs(ref).max())})
    return {"volumes": rows, "max": max(r["push_of_pull_max_rel_err"] for r in rows),
            "bound": "2^-8 (one bf16 rounding of the pulled values) + 2^-8 (the bf16 push output) + 1e-5"}


# ---------------------------------------------------------------------- #
# config 5: registration iterations through the SVF exponentiation        #
# ---------------------------------------------------------------------- #
def run_svf(args, rank, world, device):
    """Config 5: velocity 1x160x192x160x3 (N(0,1) smoothed sigma 3), moving
    and fixed images 1x1x160x192x160; one iteration = exp(v) by 8 squarings
    (linear, dft, extrapolate) -> pull of the moving image at order 3, dct2
    -> MSE -> backward through every pull -> gradient step on v."""
    import nitorch_b200 as nb
    from nitorch_b200 import svf, workloads
    v, mov, fix = workloads.config5()
    v, mov, fix = v.float().to(device), mov.float().to(device), fix.float().to(device)
    nvox = int(np.prod(v.shape[1:-1]))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    def iteration():
        vr = v.detach().requires_grad_(True)
        phi = svf.exp(vr)
        w = nb.grid_pull(mov, phi, 3, "dct2", False)
        loss = ((w - fix) ** 2).mean()
        loss.backward()
        with torch.no_grad():
            v.sub_(vr.grad, alpha=1.0)
        return loss

    for _ in range(args.warmup):
        iteration()
    torch.cuda.synchronize()
    total_ms, launches, _ = timed_steps(iteration, args, world, device, flush, steps=args.svf_steps)

    # the two kernels of every squaring, alone on a field of this size in the
    # iteration's layout: composition (field in, field out: 2 x 12 B per voxel
    # algorithmic) and its backward (field and gradient in, accumulator out:
    # 12 + 12 + 16 B per voxel)
    def kernel_ms(fn, reps=10):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return float(np.median(ts))

    from nitorch_b200 import _lib
    u = torch.mul(v, 1.0 / 256, out=svf._field_like(v))
    g = torch.randn_like(v)
    fwd_ms = kernel_ms(lambda: svf.compose(u))
    fwd_kernel = _lib.last_kernel()
    bwd_ms = kernel_ms(lambda: svf.compose_backward(g, u))
    bwd_kernel = _lib.last_kernel()
    hbm, src = peaks()
    kernels = {}
    for name, ms, per_vox, kern in (("compose", fwd_ms, 24, fwd_kernel), ("compose_backward", bwd_ms, 40, bwd_kernel)):
        algo = per_vox * nvox
        achieved = algo / (ms * 1e-3) / 1e9
        kernels[name] = {"kernel": kern, "ms": round(ms, 4),
                         "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                                      "frac": round(achieved / hbm, 4), "peak_source": src,
                                      "algorithmic_bytes_per_launch": algo}}
    return {"workload": "cfg5: exp(v) by 8 squarings (linear, dft) -> pull moving (cubic, dct2) -> MSE -> "
                        "backward -> step; 1x160x192x160",
            "ms_per_iteration": round(total_ms / args.svf_steps, 3),
            "value": round(world * nvox * args.svf_steps / (total_ms * 1e-3) / 1e9, 4), "unit": "Gvox/s",
            "gpu_launches_per_iteration": round(launches / args.svf_steps, 1), "kernels": kernels}


# ---------------------------------------------------------------------- #
# resize: separable sampling at a diagonal affine map                     #
# ---------------------------------------------------------------------- #
def run_resize(args, rank, world, device):
    """nitorch's resize of a 1x3x256^3 float32 image to 320^3 (factor 1.25,
    anchor "c", cubic, dct2, no prefilter): the separable TMA-staged kernel
    (pp_resize) against the per-point affine pull of the same map.  Roofline:
    the image read once and the output written once (algorithmic bytes)."""
    from nitorch_b200 import affine
    import nitorch_b200 as nb
    size, out = 256, 320
    g = torch.Generator(device=device).manual_seed(51)
    x = torch.randn((1, 3, size, size, size), generator=g, device=device)
    _, _, scales, shifts = nb.api._resize_transform([size] * 3, None, [out] * 3, "c")
    mat = torch.zeros((1, 3, 4), dtype=torch.float32, device=device)
    for d in range(3):
        mat[0, d, d] = scales[d]
        mat[0, d, 3] = shifts[d]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    shape = (out,) * 3

    def timeit(fn, reps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return float(np.median(ts))

    from nitorch_b200 import _lib
    sep = timeit(lambda: affine.resize_pull(x, scales, shifts, shape, 3, "dct2", False), args.steps)
    kernel = _lib.last_kernel()
    per_point = timeit(lambda: affine.affine_pull(x, mat, shape, 3, "dct2", False), max(3, args.steps // 4))
    a = affine.resize_pull(x, scales, shifts, shape, 3, "dct2", False)
    r = affine.affine_pull(x, mat, shape, 3, "dct2", False)
    diff = float((a - r).abs().max() / r.abs().max())
    hbm, src = peaks()
    algo = (x.numel() + 3 * out ** 3) * 4
    achieved = algo / (sep * 1e-3) / 1e9
    nvox = out ** 3
    return {"workload": f"resize 1x3x{size}^3 -> 1x3x{out}^3 float32, factor 1.25, anchor c, cubic, dct2",
            "kernel": kernel, "ms": round(sep, 4), "value": round(nvox / (sep * 1e-3) / 1e9, 3), "unit": "Gvox/s",
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                         "frac": round(achieved / hbm, 4), "peak_source": src, "algorithmic_bytes_per_launch": algo,
                         "traffic": MEASURED_TRAFFIC.get(kernel)},
            "per_point_affine_pull_ms": round(per_point, 4), "speedup_over_per_point": round(per_point / sep, 2),
            "max_rel_diff_vs_per_point": diff, "resize_status": affine.resize_status()}


def run_regulariser(args, rank, world, device):
    """The native solvers' regularisers (nitorch._C.solve): the grid
    regulariser of a 1x192^3x3 float32 displacement field with nitorch's
    registration penalties (absolute 1e-4, membrane 1e-3, bending 0.2, Lame
    (0.05, 0.2), dft; every term of the stencil) and the field regulariser
    of a 1x3x192^3 image (membrane, dct2).  Roofline: the field read once and
    the output written once (algorithmic bytes).  Beside it, the reference's
    own CPU regulariser on the same input (one call, all host threads)."""
    from nitorch_b200 import _lib, solve
    n = 192
    g = torch.Generator(device=device).manual_seed(61)
    v = torch.randn((1, n, n, n, 3), generator=g, device=device)
    x = torch.randn((1, 3, n, n, n), generator=g, device=device)
    ov, ox = torch.empty_like(v), torch.empty_like(x)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    pen = dict(absolute=1e-4, membrane=1e-3, bending=0.2, lame=(0.05, 0.2))

    def timeit(fn, reps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return float(np.median(ts))

    l0 = _lib.kernel_launches()
    grid_ms = timeit(lambda: solve.c_regulariser_grid(v, **pen, bound="dft", output=ov), args.steps)
    field_ms = timeit(lambda: solve.c_regulariser(x, None, None, 3, 0.0, 1.0, 0.0, bound="dct2", output=ox),
                      args.steps)
    launches = _lib.kernel_launches() - l0
    hbm, src = peaks()
    algo = 2 * v.numel() * 4
    out = {}
    for name, ms in (("grid", grid_ms), ("field", field_ms)):
        achieved = algo / (ms * 1e-3) / 1e9
        out[name] = {"ms": round(ms, 4), "value": round(n ** 3 / (ms * 1e-3) / 1e9, 3), "unit": "Gvox/s",
                     "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                                  "frac": round(achieved / hbm, 4), "peak_source": src,
                                  "algorithmic_bytes_per_launch": algo}}
    res = {"workload": f"regulariser_grid 1x{n}^3x3 float32 (absolute 1e-4, membrane 1e-3, bending 0.2, "
                       f"lame (0.05, 0.2), dft); regulariser 1x3x{n}^3 (membrane 1, dct2)",
           "gpu_launches": launches, **out}
    if not args.no_cpu_baseline:
        from oracle import reference as R
        ref = R.load_compiled()
        if ref is not None:
            vc = v.cpu().movedim(-1, 1).contiguous()
            E = torch.Tensor()
            dft = ref.BoundType.dft
            ref.regulariser_grid(vc, E, E, E, 1e-4, 1e-3, 0.2, 0.05, 0.2, [1.0], [dft])  # warm-up
            t0 = time.perf_counter()
            r = ref.regulariser_grid(vc, E, E, E, 1e-4, 1e-3, 0.2, 0.05, 0.2, [1.0], [dft])
            cpu_ms = (time.perf_counter() - t0) * 1e3
            ours = solve.c_regulariser_grid(v, **pen, bound="dft").cpu().movedim(-1, 1)
            res["reference_cpu"] = {"ms": round(cpu_ms, 1), "threads": torch.get_num_threads(),
                                    "kind": "reference", "max_rel_diff": float((ours - r).abs().max() / r.abs().max())}
    return res


def run_all(args, rank, world, device):
    import gc
    if args.only_resize:
        return {"resize": run_resize(args, rank, world, device)} if rank == 0 else None
    if args.only_svf:
        r = run_svf(args, rank, world, device)
        return {"svf": r} if rank == 0 else None
    if args.only_regulariser:
        r = run_regulariser(args, rank, world, device)
        return {"regulariser": r} if rank == 0 else None
    line = run_b200(args, rank, world, device)
    gc.collect()
    torch.cuda.empty_cache()
    if not args.no_batched:
        from nitorch_b200 import _lib
        l0 = _lib.kernel_launches()
        b = run_batched(args, rank, world, device)
        if line is not None:
            b["gpu_launches"] = _lib.kernel_launches() - l0
            line["batched"] = b
        gc.collect()
        torch.cuda.empty_cache()
    if not args.no_svf:
        r = run_svf(args, rank, world, device)
        if line is not None:
            line["svf"] = r
    if not args.no_resize:
        gc.collect()
        torch.cuda.empty_cache()
        r = run_resize(args, rank, world, device)
        if line is not None:
            line["resize"] = r
    if not args.no_regulariser:
        gc.collect()
        torch.cuda.empty_cache()
        r = run_regulariser(args, rank, world, device)
        if line is not None:
            line["regulariser"] = r
    return line


# ---------------------------------------------------------------------- #
# reference CPU implementation of the same step                          #
# ---------------------------------------------------------------------- #
def reference_step_fn():
    """The step through the reference's own compiled CPU backend (its native
    API: the functions GridPull / GridPush call).  The prefilter -- in the
    reference a third-party Python package that is not present on the
    benchmark host -- is the oracle's restatement of it, vectorised over
    lines with torch CPU operations in float32 as the reference's own runs
    (0.33 s for 3x192^3 on 8 cores against the reference's 0.325 s)."""
    from oracle import prefilter_torch as P
    from oracle import reference as R
    ref = R.load_compiled()
    if ref is None:
        return None, "port"
    b, o = [ref.BoundType.dct2], [ref.InterpolationType.cubic]

    def prefilter(a):
        return P.spline_coeff_nd(a, [3], [3], 3)

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


CPU_SAMPLE = ("1x3x{size}^3 float32, the same chain (prefilter -> pull -> push -> <z,w> -> backward to the "
              "image and the grid); pull / push and their backward passes through the reference's compiled "
              "C++ CPU backend, prefilter through the oracle's line-vectorised torch restatement")


def cpu_baseline(size, steps=1, warmup=1):
    """The reference's CPU implementation of the step on the host cores (all
    threads), full size: one warm-up and `steps` timed steps."""
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
            "kind": kind, "sample": CPU_SAMPLE.format(size=size) + f"; {steps} step(s) after {warmup} warm-up",
            "sec_per_step": round(dt, 4)}


def reference_cuda_leg(args, device, x, grid, w, ours_ms):
    """The reference's own CUDA push/pull kernels (nitorch's CUDA backend,
    compiled for sm_100a from its sources into oracle/_ref/cuda) timed on the
    same inputs and chain as the headline step, with the same CUDA events and
    L2 flush: the GPU implementation this library replaces.  Its prefilter
    is this library's (the reference's prefilter is a third-party package
    that is not present); the rest runs through the reference's native
    functions with the requires_grad wiring of nitorch/_C/grid.py.  Also
    reports the largest relative difference of the outputs."""
    from oracle import reference as R
    ref = R.load_compiled_cuda()
    if ref is None:
        return {"unavailable": "reference CUDA backend not built (oracle/build_ref_cuda.py)"}
    import nitorch_b200 as nb
    b, o = [ref.BoundType.dct2], [ref.InterpolationType.cubic]
    l2buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    marks = []  # (op, event) after each op of a step

    def mark(op):
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        marks.append((op, ev))

    def chain():
        c = nb.spline_coeff_nd(x.detach(), ORDER, BOUND, dim=3)
        mark("prefilter")
        y = ref.grid_pull(c, grid.detach(), b, o, 0)
        mark("pull_fwd")
        z = ref.grid_push(y, grid.detach(), list(x.shape[2:]), b, o, 0)
        mark("push_fwd")
        loss = (z * w).sum()
        yr = y.detach().requires_grad_(True)
        gr = grid.detach().requires_grad_(True)
        mark("loss")
        dy, dg1 = ref.grid_push_backward(w, yr, gr, b, o, 0)
        mark("push_bwd")
        cr = c.detach().requires_grad_(True)
        dc, dg2 = ref.grid_pull_backward(dy, cr, gr, b, o, 0)
        mark("pull_bwd")
        dx = nb.spline_coeff_nd(dc, ORDER, BOUND, dim=3)
        mark("prefilter_bwd")
        return z, dx, dg1 + dg2, loss

    for _ in range(max(1, min(args.warmup, 3))):
        chain()
    torch.cuda.synchronize()
    steps = max(1, min(args.steps, 5))
    ts = []
    per_op = {}
    clocks = ClockSampler(device.index or 0)
    clocks.start()
    for _ in range(steps):
        l2buf.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        marks.clear()
        s.record()
        out = chain()
        e.record()
        torch.cuda.synchronize()
        ts.append(s.elapsed_time(e))
        prev = s
        for op, ev in marks:
            per_op.setdefault(op, []).append(prev.elapsed_time(ev))
            prev = ev
    clk = clocks.stop()
    ms = float(np.mean(ts))
    # this library's outputs on the same inputs
    xr = x.detach().requires_grad_(True)
    gr = grid.detach().requires_grad_(True)
    z = nb.grid_push(nb.grid_pull(xr, gr, ORDER, BOUND, EXTRAP, prefilter=True), gr, None, ORDER, BOUND, EXTRAP)
    (z * w).sum().backward()
    diff = {}
    for k, a_, r_ in (("push", z, out[0]), ("dx", xr.grad, out[1]), ("dgrid", gr.grad, out[2])):
        a_, r_ = a_.detach().double(), r_.detach().double()
        diff[k] = float((a_ - r_).abs().max() / r_.abs().max().clamp_min(1e-30))
    nvox = int(np.prod(x.shape[2:]))
    return {"ms_per_step": round(ms, 4), "value": round(nvox / (ms * 1e-3) / 1e9, 4), "unit": "Gvox/s",
            "steps": steps, "speedup_of_this_library": round(ms / ours_ms, 2),
            "ops_ms": {k: round(float(np.mean(v)), 4) for k, v in per_op.items()}, "clocks": clk,
            "max_rel_diff_vs_this_library": diff,
            "note": "nitorch's CUDA pushpull_kernel built for sm_100a from the reference sources; "
                    "prefilter from this library"}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    size = args.cpu_size or args.size
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
    sample = CPU_SAMPLE.format(size=size) + f"; {torch.get_num_threads()} threads"
    return {"impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": "Gvox/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"1x3x{args.size}^3 order-3 dct2 prefilter pull+push fwd+bwd (cfg2)",
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
    ap.add_argument("--cpu-size", type=int, default=None,
                    help="spatial size of the CPU baseline (default: the workload's own)")
    ap.add_argument("--no-reference-cuda", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-volumes", type=int, default=64)
    ap.add_argument("--batch-steps", type=int, default=3)
    ap.add_argument("--no-svf", action="store_true")
    ap.add_argument("--no-fused", action="store_true", help="skip the fused pull_push leg")
    ap.add_argument("--only-resize", action="store_true", help="run the resize leg alone")
    ap.add_argument("--only-svf", action="store_true", help="run the config-5 leg alone")
    ap.add_argument("--only-regulariser", action="store_true", help="run the regulariser leg alone")
    ap.add_argument("--no-regulariser", action="store_true", help="skip the regulariser leg")
    ap.add_argument("--no-resize", action="store_true")
    ap.add_argument("--svf-steps", type=int, default=5)
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
        line = run_all(args, rank, world, device)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
