"""Side-by-side timing of the reference's own CUDA push/pull kernels
(nitorch's CUDA backend compiled for sm_100a by oracle/build_ref_cuda.py)
and this library's, on the same B200, the same inputs and the same chain --
a measurement script, not a test (pytest does not collect it).

    python tests/perf_reference_cuda.py [--size 192] [--steps 5] [--warmup 3] [--svf]

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


def make_pull(mod):
    """Autograd wrapper of a backend's native grid_pull, as nitorch/_C/grid.py
    (GridPull, 192-230) wraps the reference's: the backward asks for the
    gradients of the inputs that require them."""
    class Pull(torch.autograd.Function):
        @staticmethod
        def forward(ctx, inp, grid, bound, order, ex):
            ctx.opt = (bound, order, ex)
            ctx.save_for_backward(inp, grid)
            return mod.grid_pull(inp, grid, bound, order, ex)

        @staticmethod
        def backward(ctx, g):
            inp, grid = ctx.saved_tensors
            grads = list(mod.grid_pull_backward(g.contiguous(), inp, grid, *ctx.opt))
            gi = grads.pop(0) if ctx.needs_input_grad[0] else None
            gg = grads.pop(0) if ctx.needs_input_grad[1] else None
            return gi, gg, None, None, None
    return Pull.apply


def svf_iteration(mod, v, mov, fix, idg):
    """Config-5 iteration through one backend's native pull: exp(v) by 8
    squarings u <- u + pull(u, id + u) (linear, dft, extrapolate; the
    reference's exp_forward, nitorch/spatial/_svf.py:85-94), pull of the
    moving image (cubic, dct2), MSE, backward."""
    pull = make_pull(mod)
    lin, dft = [mod.InterpolationType.linear], [mod.BoundType.dft]
    cub, dct2 = [mod.InterpolationType.cubic], [mod.BoundType.dct2]
    vr = v.detach().requires_grad_(True)
    u = vr / 256.0
    for _ in range(8):
        u = u + pull(u.movedim(-1, 1).contiguous(), idg + u, dft, lin, 1).movedim(1, -1)
    w = pull(mov, idg + u, dct2, cub, 0)
    loss = ((w - fix) ** 2).mean()
    loss.backward()
    return loss.detach(), vr.grad


def time_svf(mod, v, mov, fix, idg, steps, warmup):
    for _ in range(warmup):
        svf_iteration(mod, v, mov, fix, idg)
    torch.cuda.synchronize()
    ts = []
    out = None
    for _ in range(steps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        out = svf_iteration(mod, v, mov, fix, idg)
        e.record()
        torch.cuda.synchronize()
        ts.append(s.elapsed_time(e))
    return out, float(np.median(ts))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=192)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--svf", action="store_true", help="also time a config-5 registration iteration")
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
    if args.svf:
        v5, mov, fix = workloads.config5()
        v5, mov, fix = v5.float().to(dev), mov.float().to(dev), fix.float().to(dev)
        shape = v5.shape[1:-1]
        idg = torch.stack(torch.meshgrid(*[torch.arange(n, dtype=torch.float32, device=dev) for n in shape],
                                         indexing="ij"), -1)[None]
        sv = {"workload": "cfg5 iteration: exp(v) 8 squarings (linear, dft) -> pull moving (cubic, dct2) -> "
                          "MSE -> backward, 1x160x192x160, both backends through the same autograd wiring"}
        outs5 = {}
        for name, mod in (("reference_cuda", ref), ("b200", spatial)):
            out, ms = time_svf(mod, v5, mov, fix, idg, max(2, args.steps // 2), 2)
            outs5[name] = out
            sv[name] = {"ms_per_iteration": round(ms, 3)}
        sv["speedup"] = round(sv["reference_cuda"]["ms_per_iteration"] / sv["b200"]["ms_per_iteration"], 2)
        ga, gb = outs5["b200"][1].double(), outs5["reference_cuda"][1].double()
        sv["grad_max_rel_diff"] = float((ga - gb).abs().max() / gb.abs().max().clamp_min(1e-30))
        res["svf"] = sv
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
