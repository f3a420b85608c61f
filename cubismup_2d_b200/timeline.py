"""In-graph kernel timeline of one step (the trace build).

    python -m cubismup_2d_b200.build --trace
    python -m cubismup_2d_b200.timeline [swimmer|cylinder] [--steps N] [--noflush] [--fp32] [--operators]

Runs the workload on the trace build (libcup2d_trace.so, compiled with
-DCUP2D_TRACE): thread 0 of every CTA of every kernel stamps %globaltimer at
entry and exit, so each kernel's first start and last end inside one
graph-replayed step can be read back.  Prints, per kernel, the median over
the timed steps of its start, end and duration relative to the step's first
kernel, with the L2 flushed before every step as in bench.py unless
--noflush is given; --fp32 runs the FP32 Poisson transforms (CUP2D_PREC_FP32).
--operators runs the reference's loop through the ABI instead of graph
steps (calcMaxTimestep with its dt read back, the four operators, the step
end, the shape state read back; no L2 flush, as in bench.py's e2e) and
reports the host's wall-clock time per step beside the kernels' spans.
"""
import argparse
import ctypes
import os
import sys
import time

import numpy as np

from . import abi, build
from .synthetic import FORCED_CYLINDER_RE100, SWIMMER_1024x512, noise_field

# the order of TraceId in csrc/internal.cuh
KERNELS = ["step_begin/max_u", "set_dt", "end_step", "advdiff", "rhs_div", "pcorr", "fade_sums",
           "obj_begin", "disk_place", "raster_disk", "chi", "moments", "udef_grid",
           "rhs_obst", "rhs_corr", "momenta", "collide", "penalize", "forces", "fish_midline",
           "fish_frame", "fish_raster", "rows_r2c", "cols", "rows_c2r", "dct_rows_fwd", "dct_cols",
           "dct_rows_inv", "fish_tile_search", "max_next"]
TRACE_ITEMS = 4096
WORKLOADS = {"swimmer": SWIMMER_1024x512, "cylinder": FORCED_CYLINDER_RE100}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", nargs="?", default="swimmer", choices=sorted(WORKLOADS))
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--noflush", action="store_true")
    ap.add_argument("--fp32", action="store_true")
    ap.add_argument("--operators", action="store_true")
    a = ap.parse_args(argv)
    if not os.path.exists(build.TRACE_LIB):
        build.build(trace=True)
    abi.LIB_PATH = build.TRACE_LIB
    import torch
    sim = abi.Simulation(WORKLOADS[a.workload] + (" -precision fp32" if a.fp32 else ""))
    sim.init()
    ctx = sim.ctx
    for comp, f in enumerate(("u", "v")):
        ctx.set(f, ctx.get(f) + noise_field(0, comp, ctx.ny, ctx.nx))
    L = abi.lib()
    L.cup2d_trace.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_int]
    n = len(KERNELS)
    buf = (ctypes.c_ulonglong * (2 * n + 8 * TRACE_ITEMS))()

    calls = {}

    def operator_step():
        # host time of each call (µs), from the step's start
        t = [time.perf_counter()]
        dt = sim.calcMaxTimestep()
        t.append(time.perf_counter())
        for op in sim.pipeline:
            op(dt)
            t.append(time.perf_counter())
        ctx.end_step()
        t.append(time.perf_counter())
        st = ctx.shape(0)
        t.append(time.perf_counter())
        names = ["calcMaxTimestep"] + [op.getName() for op in sim.pipeline] + ["end_step", "shape"]
        for i, n in enumerate(names):
            calls.setdefault(n, []).append(((t[i] - t[0]) * 1e6, (t[i + 1] - t[0]) * 1e6))
        return st

    if a.operators:
        for _ in range(a.warmup):
            operator_step()
    else:
        ctx.advance(a.warmup)
    ctx.sync()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{sim.cfg.device}")
    spans, steps = {}, []
    for _ in range(a.steps):
        if a.operators:
            L.cup2d_trace(ctx.h_, None, 1)
            t0h = time.perf_counter()
            operator_step()
            steps.append((time.perf_counter() - t0h) * 1e6)
        else:
            if not a.noflush:
                flush.fill_(1.0)
            torch.cuda.synchronize()
            L.cup2d_trace(ctx.h_, None, 1)
            steps.append(ctx.time_step() * 1e3)
        L.cup2d_trace(ctx.h_, buf, 0)
        t = np.array(buf[:2 * n], dtype=np.uint64).reshape(n, 2)
        used = t[:, 1] > 0
        t0 = t[used, 0].min()
        for i in np.nonzero(used)[0]:
            spans.setdefault(KERNELS[i], []).append(((t[i, 0] - t0) / 1e3, (t[i, 1] - t0) / 1e3))
    if a.operators:
        print(f"operator step (host wall clock): median {np.median(steps):.1f} us over {a.steps} steps")
        print(f"{'host call':18s} {'start':>8s} {'end':>8s} {'dur':>7s}  (us, from the step's first call)")
        for n, v in calls.items():
            v = np.array(v[-a.steps:])
            print(f"{n:18s} {np.median(v[:, 0]):8.1f} {np.median(v[:, 1]):8.1f} {np.median(v[:, 1] - v[:, 0]):7.1f}")
    else:
        print(f"step (CUDA events): median {np.median(steps):.1f} us over {a.steps} steps"
              + (" (no L2 flush)" if a.noflush else " (L2 flushed before each step)"))
    rows = sorted((np.median(np.array(v)[:, 0]), np.median(np.array(v)[:, 1]), k) for k, v in spans.items())
    print(f"{'kernel':18s} {'start':>8s} {'end':>8s} {'dur':>7s}  (us)")
    for s0, e0, k in rows:
        print(f"{k:18s} {s0:8.1f} {e0:8.1f} {e0 - s0:7.1f}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
