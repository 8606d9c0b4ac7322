"""Many volumes of uneven shapes in a few launches per mode.

nitorch's backend processes one tensor per call; training and registration
loops over many subjects then pay a launch (and a Python round trip) per
volume and per op.  Here a batch of 3-D volumes -- any shapes, any channel
count, isotropic orders 0-3, float32 or bfloat16 images -- goes through one
launch per (order, channel block) group and mode (pull, push, their
backward passes, or the fused pull-push and its backward), driven by a host
plan (``pp_batch_plan`` / ``pp_batch_run`` in ``include/nitorch_b200.h``)
whose per-volume arguments travel as kernel parameters.

`PullPushBatch` is the pull -> push -> <z, w> -> backward step of the
batched benchmark configuration, on static buffers ("arenas"), so the whole
step -- per-volume sample ordering, the batched launches and the loss -- can
be captured once in a CUDA graph and replayed.  Three forms: "fused" (the
fused normal operator, two batched passes per step), "chain" (the four
separate passes of the two-call chain, batched) and "percall" (every volume
through the single-volume entry points and their kernels -- brick order,
brick kernels -- from one host loop, captured in the same graph).
`Autotuner` picks the form, the launch shape and the sample order per
(orders, dtype, channel mix, batch size) key by timing them, and caches the
choice on disk.

`plan_shards` partitions a batch over ranks (longest processing time first
on points x channels); the volumes are independent, so multi-GPU runs need
no collective on the data path.
"""
import ctypes
import gc
import json
import os
import threading
import time

import torch

from . import _lib
from .enums import BoundType


def _entry(src=None, trgt=None, grid=None, out=None, gg=None, opt=None):
    e = _lib.PPBatchEntry()
    for name, t in (("src", src), ("trgt", trgt), ("grid", grid), ("out", out), ("gg", gg)):
        if t is not None:
            setattr(e, name, _lib.desc(t))
    e.opt = opt
    return e


class BatchPlan:
    """A plan of one batched mode over fixed tensors.  The tensors (and the
    sample orders named in the options) must stay alive and in place while
    the plan is used; `run` only enqueues work (graph-capturable)."""

    def __init__(self, mode, entries, ctas=0, device=None):
        L = _lib.load()
        n = len(entries)
        arr = (_lib.PPBatchEntry * n)(*entries)
        nbytes = L.pp_batch_plan_bytes(n)
        self.device = torch.device(device or "cuda")
        self.buf = ctypes.create_string_buffer(nbytes)
        self.mode = mode
        # interleaved accumulators of the vectorised scatters (device scratch)
        sbytes = L.pp_batch_scratch_bytes(arr, n, mode)
        self.scratch = torch.empty(sbytes, dtype=torch.uint8, device=self.device) if sbytes else None
        sptr = ctypes.c_void_p(self.scratch.data_ptr()) if sbytes else None
        _lib.check(L.pp_batch_plan(arr, n, mode, int(ctas), ctypes.cast(self.buf, ctypes.c_void_p), nbytes,
                                   sptr, sbytes))

    def run(self):
        L = _lib.load()
        stream = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        _lib.check(L.pp_batch_run(ctypes.cast(self.buf, ctypes.c_void_p), stream))


def _arena(sizes, dtype, device):
    """One flat buffer and per-volume views of the given shapes."""
    total = sum(int(torch.Size(s).numel()) for s in sizes)
    flat = torch.empty(total, dtype=dtype, device=device)
    views, off = [], 0
    for s in sizes:
        n = int(torch.Size(s).numel())
        views.append(flat[off:off + n].view(s))
        off += n
    return flat, views


class PullPushBatch:
    """Batched step: for every volume i,
        y_i = pull(x_i, g_i);  z_i = push(y_i, g_i);  loss = sum_i <z_i, w_i>
    and the gradients d loss / d x_i (float32) and d loss / d g_i.

    shapes: list of 3-D spatial shapes; channels: list of C; orders: list of
    isotropic orders (0-3).  Images are `dtype` (float32 or bfloat16); grids,
    scatter outputs and gradients float32.  Inputs live in the arenas
    `x`, `grid`, `w` (write them in place, e.g. `batch.x[i].copy_(...)`).
    With `fused` (default) y_i is never stored: one pass computes z_i and one
    pass the gradients; otherwise `y`, `dy` and the two grid-gradient terms
    are kept in their own arenas.
    """

    FORMS = ("fused", "chain", "percall")

    def __init__(self, shapes, channels, orders, bound="dct2", extrapolate=False,
                 dtype=torch.float32, device=None, sorted_order=True, ctas=0, fused=True, form=None,
                 deterministic=False):
        self.device = torch.device(device or "cuda")
        # scatters in int64 fixed point: bit-identical results from run to run
        self.flags = _lib.PP_DETERMINISTIC if deterministic else 0
        self.n = len(shapes)
        self.shapes = [tuple(int(v) for v in s) for s in shapes]
        self.channels = [int(c) for c in channels]
        self.orders = [int(o) for o in orders]
        self.dtype = dtype
        self.sorted_order = bool(sorted_order)
        self.ctas = int(ctas)
        self.form = form or ("fused" if fused else "chain")
        if self.form not in self.FORMS:
            raise ValueError(f"unknown batch form {self.form}")
        self.fused = self.form == "fused"
        self.bound = int(BoundType[bound] if isinstance(bound, str) else bound)
        self.extrapolate = int(extrapolate)
        if self.form == "percall":
            self._init_percall()
            return
        img = [(1, c, *s) for c, s in zip(self.channels, self.shapes)]
        grd = [(1, *s, 3) for s in self.shapes]
        dev = self.device
        self.x_flat, self.x = _arena(img, dtype, dev)
        self.grid_flat, self.grid = _arena(grd, torch.float32, dev)
        self.w_flat, self.w = _arena(img, dtype, dev)
        self.z_flat, self.z = _arena(img, torch.float32, dev)
        self.dx_flat, self.dx = _arena(img, torch.float32, dev)
        if not self.fused:
            self.y_flat, self.y = _arena(img, dtype, dev)
            self.dy_flat, self.dy = _arena(img, dtype, dev)
            self.dg1_flat, self.dg1 = _arena(grd, torch.float32, dev)
            self.dg2_flat, self.dg2 = _arena(grd, torch.float32, dev)
        self.dgrid_flat, self.dgrid = _arena(grd, torch.float32, dev)
        self.loss = torch.zeros((), dtype=torch.float32, device=dev)
        self.perm_flat, self.perm = _arena([(int(torch.Size(s).numel()),) for s in self.shapes], torch.int32, dev)
        L = _lib.load()
        ws = 0
        for g, s in zip(self.grid, self.shapes):
            src = (ctypes.c_int64 * 3)(*s)
            ws = max(ws, L.pp_sample_order_workspace_bytes(ctypes.byref(_lib.desc(g)), src))
        self.sort_ws = torch.empty(max(ws, 256), dtype=torch.uint8, device=dev)
        self._build_plans()
        self.graph = None
        self.graph_launches = 0

    # -- the per-call form ------------------------------------------------------
    def _init_percall(self):
        """Static buffers of the per-call form: every volume goes through the
        single-volume entry points (pp_brick_order, pp_grid_pull,
        pp_grid_push, pp_grid_push_backward, pp_grid_pull_backward) -- the
        kernels of the per-call API -- enqueued from one host loop, so that a
        CUDA graph holds the whole step.  Pulled / pushed values and the image
        gradient keep the image dtype, as the per-call API returns them."""
        img = [(1, c, *s) for c, s in zip(self.channels, self.shapes)]
        grd = [(1, *s, 3) for s in self.shapes]
        dev, dt = self.device, self.dtype
        self.x_flat, self.x = _arena(img, dt, dev)
        self.grid_flat, self.grid = _arena(grd, torch.float32, dev)
        self.w_flat, self.w = _arena(img, dt, dev)
        self.y_flat, self.y = _arena(img, dt, dev)
        self.z_flat, self.z = _arena(img, dt, dev)
        self.dy_flat, self.dy = _arena(img, dt, dev)
        self.dx_flat, self.dx = _arena(img, dt, dev)
        self.dg1_flat, self.dg1 = _arena(grd, torch.float32, dev)
        self.dg2_flat, self.dg2 = _arena(grd, torch.float32, dev)
        self.dgrid_flat, self.dgrid = _arena(grd, torch.float32, dev)
        self.loss = torch.zeros((), dtype=torch.float32, device=dev)
        L = _lib.load()
        npts = [int(torch.Size(s).numel()) for s in self.shapes]
        self.perm_flat, self.perm = _arena([(n,) for n in npts], torch.int32, dev)
        nb, ws, pws = [], 256, 256
        for g, s, z, dx in zip(self.grid, self.shapes, self.z, self.dx):
            src = (ctypes.c_int64 * 3)(*s)
            nb.append(int(L.pp_brick_count(ctypes.byref(_lib.desc(g)), src)) + 1)
            ws = max(ws, L.pp_brick_order_workspace_bytes(ctypes.byref(_lib.desc(g)), src))
            pws = max(pws, L.pp_push_workspace_bytes(ctypes.byref(_lib.desc(z)), self.flags),
                      L.pp_push_workspace_bytes(ctypes.byref(_lib.desc(dx)), self.flags))
        self.starts_flat, self.starts = _arena([(n,) for n in nb], torch.int32, dev)
        self.recs_flat, self.recs = _arena([(n, 4) for n in npts], torch.float32, dev)
        self.sort_ws = torch.empty(ws, dtype=torch.uint8, device=dev)
        self.push_ws = torch.empty(pws, dtype=torch.uint8, device=dev)
        self.plans = {}
        self.graph = None
        self.graph_launches = 0

    def _step_percall(self):
        L = _lib.load()
        B = _lib
        stream = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        ws, nws = ctypes.c_void_p(self.push_ws.data_ptr()), self.push_ws.numel()
        ref = lambda t: ctypes.byref(B.desc(t))  # noqa: E731
        opts = []
        for i in range(self.n):
            if self.sorted_order:
                src = (ctypes.c_int64 * 3)(*self.shapes[i])
                B.check(L.pp_brick_order(ref(self.grid[i]), src, ctypes.c_void_p(self.perm[i].data_ptr()),
                                         ctypes.c_void_p(self.starts[i].data_ptr()),
                                         ctypes.c_void_p(self.recs[i].data_ptr()),
                                         ctypes.c_void_p(self.sort_ws.data_ptr()), self.sort_ws.numel(), stream))
                opts.append(B.options([self.bound], [self.orders[i]], self.extrapolate, self.flags,
                                      self.perm[i].data_ptr(), self.starts[i].data_ptr(),
                                      self.recs[i].data_ptr()))
            else:
                opts.append(B.options([self.bound], [self.orders[i]], self.extrapolate, self.flags))
        for i in range(self.n):
            o = ctypes.byref(opts[i])
            B.check(L.pp_grid_pull(ref(self.x[i]), ref(self.grid[i]), ref(self.y[i]), o, stream))
            B.check(L.pp_grid_push(ref(self.y[i]), ref(self.grid[i]), ref(self.z[i]), o, stream, ws, nws))
        self._loss()
        for i in range(self.n):
            o = ctypes.byref(opts[i])
            B.check(L.pp_grid_push_backward(ref(self.w[i]), ref(self.y[i]), ref(self.grid[i]), ref(self.dy[i]),
                                            ref(self.dg1[i]), o, stream))
            B.check(L.pp_grid_pull_backward(ref(self.dy[i]), ref(self.x[i]), ref(self.grid[i]), ref(self.dx[i]),
                                            ref(self.dg2[i]), o, stream, ws, nws))
        torch.add(self.dg1_flat, self.dg2_flat, out=self.dgrid_flat)
        return self.loss

    # -- plans ---------------------------------------------------------------
    def _opt(self, i):
        perm = self.perm[i].data_ptr() if self.sorted_order else None
        return _lib.options([self.bound], [self.orders[i]], self.extrapolate, self.flags, perm)

    def _build_plans(self):
        B = _lib
        if self.fused:
            ents = {"pp": [], "pp_bwd": []}
            for i in range(self.n):
                o = self._opt(i)
                ents["pp"].append(_entry(src=self.x[i], grid=self.grid[i], out=self.z[i], opt=o))
                ents["pp_bwd"].append(_entry(src=self.x[i], trgt=self.w[i], grid=self.grid[i], out=self.dx[i],
                                             gg=self.dgrid[i], opt=o))
            modes = {"pp": B.PP_BATCH_PULL_PUSH, "pp_bwd": B.PP_BATCH_PULL_PUSH_BACKWARD}
        else:
            ents = {m: [] for m in ("pull", "push", "push_bwd", "pull_bwd")}
            for i in range(self.n):
                o = self._opt(i)
                ents["pull"].append(_entry(src=self.x[i], grid=self.grid[i], out=self.y[i], opt=o))
                ents["push"].append(_entry(trgt=self.y[i], grid=self.grid[i], out=self.z[i], opt=o))
                ents["push_bwd"].append(_entry(src=self.w[i], trgt=self.y[i], grid=self.grid[i], out=self.dy[i],
                                               gg=self.dg1[i], opt=o))
                ents["pull_bwd"].append(_entry(src=self.x[i], trgt=self.dy[i], grid=self.grid[i], out=self.dx[i],
                                               gg=self.dg2[i], opt=o))
            modes = {"pull": B.PP_BATCH_PULL, "push": B.PP_BATCH_PUSH,
                     "push_bwd": B.PP_BATCH_PUSH_BACKWARD, "pull_bwd": B.PP_BATCH_PULL_BACKWARD}
        self.plans = {k: BatchPlan(modes[k], ents[k], ctas=self.ctas, device=self.device) for k in ents}

    # -- the step --------------------------------------------------------------
    def _sort(self):
        L = _lib.load()
        stream = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        for i in range(self.n):
            src = (ctypes.c_int64 * 3)(*self.shapes[i])
            _lib.check(L.pp_sample_order(ctypes.byref(_lib.desc(self.grid[i])), src,
                                         ctypes.c_void_p(self.perm[i].data_ptr()),
                                         ctypes.c_void_p(self.sort_ws.data_ptr()), self.sort_ws.numel(), stream))

    def _loss(self):
        if self.dtype == torch.float32:
            torch.dot(self.z_flat, self.w_flat, out=self.loss)
        else:
            self.loss.copy_((self.z_flat.float() * self.w_flat.float()).sum())

    def step_eager(self):
        """One step without the graph; returns the loss tensor (device)."""
        if self.form == "percall":
            return self._step_percall()
        if self.sorted_order:
            self._sort()
        if self.fused:
            self.plans["pp"].run()
            self._loss()
            self.plans["pp_bwd"].run()
            return self.loss
        self.plans["pull"].run()
        self.plans["push"].run()
        self._loss()
        self.plans["push_bwd"].run()
        self.plans["pull_bwd"].run()
        torch.add(self.dg1_flat, self.dg2_flat, out=self.dgrid_flat)
        return self.loss

    def capture(self):
        """Capture one step in a CUDA graph (after a warm-up step)."""
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.step_eager()
        torch.cuda.current_stream(self.device).wait_stream(s)
        self.graph = torch.cuda.CUDAGraph()
        l0 = _lib.kernel_launches()
        with torch.cuda.graph(self.graph):
            self.step_eager()
        # the library's kernels inside the graph: what each replay launches
        self.graph_launches = _lib.kernel_launches() - l0
        return self

    def step(self):
        if self.graph is None:
            return self.step_eager()
        self.graph.replay()
        return self.loss

    def release(self):
        """Drop the graph and the buffers (the object is unusable after)."""
        self.graph = None
        self.plans = {}
        for k in list(vars(self)):
            if isinstance(getattr(self, k), (torch.Tensor, list)):
                setattr(self, k, None)

    def points(self):
        return sum(int(torch.Size(s).numel()) for s in self.shapes)


# ---------------------------------------------------------------------------
# autotuner
# ---------------------------------------------------------------------------
class Autotuner:
    """Chooses the launch shape (persistent CTAs per SM, or one CTA per work
    item) and the sample order of a batch by timing candidate
    configurations of the captured step, and caches the winner on disk (JSON
    at $PP_AUTOTUNE_CACHE, default ~/.cache/nitorch_b200/autotune.json),
    keyed by GPU, dtype, the set of orders, the channel mix, the batch size
    and the step form (fused or chain)."""

    # (form, persistent CTAs per SM (0 = one CTA per work item), sample order):
    # the per-volume entry points in one graph, and the batched kernels
    CANDIDATES = ([("percall", 0, True), ("percall", 0, False)] +
                  [(form, ctas_per_sm, srt) for form in ("chain", "fused") for srt in (True, False)
                   for ctas_per_sm in (0, 4)])

    _lock = threading.Lock()  # one tuning / cache write at a time per process

    def __init__(self, path=None):
        self.path = path or os.environ.get("PP_AUTOTUNE_CACHE") or os.path.join(
            os.path.expanduser("~"), ".cache", "nitorch_b200", "autotune.json")
        try:
            with open(self.path) as f:
                self.cache = json.load(f)
        except (OSError, ValueError):
            self.cache = {}

    @staticmethod
    def key(shapes, channels, orders, dtype, device):
        name = torch.cuda.get_device_name(device)
        nb = 1 << max(0, (len(shapes) - 1).bit_length())
        cmix = ",".join(str(c) for c in sorted(set(channels)))
        omix = ",".join(str(o) for o in sorted(set(orders)))
        return f"{name}|{dtype}|o{omix}|c{cmix}|n{nb}"

    def choose(self, shapes, channels, orders, dtype=torch.float32, device=None, bound="dct2",
               extrapolate=False, reps=3, init=None):
        """Returns (form, ctas, sorted_order, timings).  `init(batch)` fills
        the input arenas of a candidate batch before it is timed."""
        with Autotuner._lock:
            return self._choose(shapes, channels, orders, dtype, device, bound, extrapolate, reps, init)

    def _choose(self, shapes, channels, orders, dtype, device, bound, extrapolate, reps, init):
        device = torch.device(device or "cuda")
        k = self.key(shapes, channels, orders, dtype, device)
        if k in self.cache and "form" in self.cache[k]:
            c = self.cache[k]
            return c["form"], c["ctas"], c["sorted"], c.get("ms", {})
        sms = torch.cuda.get_device_properties(device).multi_processor_count
        timings = {}
        best = None
        for form, per_sm, srt in self.CANDIDATES:
            b = PullPushBatch(shapes, channels, orders, bound, extrapolate, dtype, device, srt, per_sm * sms,
                              form=form)
            if init is not None:
                init(b)
            b.capture()
            b.step()
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            for _ in range(reps):
                b.step()
            torch.cuda.synchronize(device)
            ms = (time.perf_counter() - t0) * 1e3 / reps
            timings[f"{form}:{per_sm}x{'sorted' if srt else 'natural'}"] = round(ms, 3)
            if best is None or ms < best[0]:
                best = (ms, form, per_sm * sms, srt)
            b.release()
            del b
            gc.collect()
            torch.cuda.empty_cache()
        self.cache[k] = {"form": best[1], "ctas": best[2], "sorted": best[3], "ms": timings}
        try:
            # write-then-rename: a concurrent reader never sees a partial file
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            tmp = f"{self.path}.{os.getpid()}.tmp"
            with open(tmp, "w") as f:
                json.dump(self.cache, f, indent=1)
            os.replace(tmp, self.path)
        except OSError:
            pass
        return best[1], best[2], best[3], timings


# ---------------------------------------------------------------------------
# multi-GPU sharding
# ---------------------------------------------------------------------------
def plan_shards(costs, world):
    """Longest-processing-time-first partition of independent volumes over
    `world` ranks.  costs: per-volume work (points x channels).  Returns a
    list of index lists, one per rank, and their loads."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    shards = [[] for _ in range(world)]
    loads = [0] * world
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        shards[r].append(i)
        loads[r] += costs[i]
    for s in shards:
        s.sort()
    return shards, loads
