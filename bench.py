"""Benchmark of the B200 CubismUP_2D timestep pipeline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload swimmer|cylinder|tandem|ensemble] [--members M]

Workload (default): the self-propelled swimmer on a 1024x512 grid (32x16
blocks of 32x32), StefanFish L=0.2, T=1 at (0.4, 0.25), nu = 2e-5
(Re = (L/T) L / nu = 2000), free-space FFT Poisson, fp64 fields, from rest
plus seeded 1e-6 uniform noise on u, v.  A step is one pass of
Simulation::simulate's loop: calcMaxTimestep, PutObjectsOnGrid, advDiff,
PressureSingle, ComputeForces.  The metric is cell-steps per second
(Nx*Ny per completed step), reported in Gcell-steps/s.

Timing: W warm-up steps, then K steps each bracketed by CUDA events on the
library's stream; between timed steps the L2 is flushed by writing a 256 MB
buffer (the working set, ~45 MB, would otherwise stay L2-resident).  Under
torchrun each rank advances its own independent replica (the path does not
shard: "replicas only") and rank 0 reports the max time over ranks.

--impl reference times the reference's own C++ operators (compiled from its
sources by oracle/Makefile into oracle/_ref) on the host cores, same workload
and metric, rank 0 only.

--workload ensemble: M (default 64) independent members drawn from a seed
(cubismup_2d_b200.synthetic.ensemble_configs: 256x128, 512x256 or 1024x512
grids; a forced cylinder or a StefanFish; Re log-uniform in [100, 1000])
advanced together, one graph launch per ensemble step (cup2d_ensemble_*);
the metric is the aggregate cell-steps/s, reported beside the same members
advanced one after another on their own graphs.  The members' fields
(~2 GB at M = 64) exceed the L2, so no flush is needed between steps.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "swimmer": ("swimmer_1024x512_fp64",
                "-bpdx 32 -bpdy 16 -extent 1 -CFL 0.1 -nu 2e-5 -lambda 1e4 -poissonType freespace "
                "-muteAll 1 -shapes 'stefanfish L=0.2 T=1 xpos=0.4 ypos=0.25'"),
    "cylinder": ("forced_cylinder_re100_512x256_fp64",
                 "-bpdx 16 -bpdy 8 -extent 1 -CFL 0.1 -nu 1.5e-4 -lambda 1e4 -poissonType freespace "
                 "-muteAll 1 -shapes 'disk radius=0.0375 xpos=0.2 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'"),
    # the swimmer with the carangiform curvature envelope of the benchmark
    # configurations, 0.82 (s/L + 0.0025) / 1.0025 (no reference counterpart)
    "swimmer_envelope": ("envelope_swimmer_1024x512_fp64",
                         "-bpdx 32 -bpdy 16 -extent 1 -CFL 0.1 -nu 2e-5 -lambda 1e4 -poissonType freespace "
                         "-muteAll 1 -shapes 'envelopefish L=0.2 T=1 xpos=0.4 ypos=0.25'"),
    # the large single-GPU case: 4096x2048 on a 2x1 domain, two swimmers
    # L = 0.1 in tandem 0.15 apart, a quarter period out of phase (phi = 0.5,
    # the reference multiplies phi by pi), Re = 5000 on L (graph steps)
    "tandem": ("tandem_swimmers_4096x2048_fp64",
               "-bpdx 128 -bpdy 64 -extent 2 -CFL 0.1 -nu 2e-6 -lambda 1e4 -poissonType freespace "
               "-muteAll 1 -shapes 'stefanfish L=0.1 T=1 xpos=0.6 ypos=0.5, "
               "stefanfish L=0.1 T=1 xpos=0.75 ypos=0.5 phi=0.5'"),
    # ... with the freely falling cylinder of that case (R = 0.03, density
    # ratio 1.01, gravity 1 in -y): a body of rhoS != 1 runs the reference's
    # variable-density branch, which needs -iterativePenalization 1
    # (advDiffGrav + PressureVarRho_approx, Simulation.cpp:183-192); its
    # convergence is decided on the host each iteration, so operator steps
    "tandem_falling": ("tandem_swimmers_falling_cylinder_4096x2048_fp64",
                       "-bpdx 128 -bpdy 64 -extent 2 -CFL 0.1 -nu 2e-6 -lambda 1e4 -poissonType freespace "
                       "-muteAll 1 -iterativePenalization 1 -gravity '0 -1' "
                       "-shapes 'stefanfish L=0.1 T=1 xpos=0.6 ypos=0.5, "
                       "stefanfish L=0.1 T=1 xpos=0.75 ypos=0.5 phi=0.5, "
                       "disk radius=0.03 xpos=1.4 ypos=0.7 rhoS=1.01'"),
}

ENSEMBLE_NAME = "ensemble{}_seed0_fp64"

# fp64 bytes per cell that each dense kernel must move (reads + writes once)
ALGO_BYTES_PER_CELL = {
    "advdiff": 40,        # read u, v; write u, v and the RHS divergence (one kernel)
    "rhs_div": 24,        # read u, v; write rhs
    "pcorr": 40,          # read p, u, v; write u, v
    "fft_rows_fwd": 24,   # read rhs (8); write half spectrum (16)
    "fft_cols": 40,       # read spectrum (16) + G^ (8); write spectrum (16)
    "fft_rows_inv": 24,   # read spectrum (16); write p (8)
    "max_u": 16,          # read u, v
}


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
# dense kernels on the swimmer workload, from one ncu capture of
# `python bench.py --steps 4 --warmup 3 --no-cpu-baseline`.  Writes stay in the 126 MB L2
# within a launch, so the captured figure is the reads.
TRAFFIC_BYTES = {
    ("swimmer", "fft_cols"): 12672768,
    ("swimmer", "fft_rows_fwd"): 4269312,
    ("swimmer", "advdiff"): 8416768,
    ("swimmer", "rhs_div"): 8396032,
    ("swimmer", "pcorr"): 12591360,
}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples the SM clock, its maximum and the clock-event reasons during
    the timed region: through NVML (read-only queries, every 5 ms, plus one
    sample at each end, so that short regions are covered), else through
    `nvidia-smi -lms 200`."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index, self.rows, self.proc, self.nvml = index, [], None, None
        self.stop = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:                                   # the device torch calls `index`
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
        masks = [getattr(pynvml, "nvmlClocksEventReason" + n, 0) for n in
                 ("HwSlowdown", "HwThermalSlowdown", "SwThermalSlowdown", "SwPowerCap")]
        return pynvml, h, masks

    def _nvml_sample(self):
        pynvml, h, masks = self.nvml
        sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
        mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        try:
            r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
        except Exception:
            r = pynvml.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        self.rows.append([str(sm), str(mx), ""] + ["Active" if (m and r & m) else "Not Active" for m in masks])

    def _nvml_loop(self):
        while not self.stop.wait(0.005):
            try:
                self._nvml_sample()
            except Exception:
                return

    def __enter__(self):
        try:
            self.nvml = self._nvml_handle()
            self._nvml_sample()
            self.t = threading.Thread(target=self._nvml_loop, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.nvml:
            self.stop.set()
            self.t.join(timeout=5)
            try:
                self._nvml_sample()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        reasons = sorted({self.NAMES[k] for r in self.rows for k in range(4) if r[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(self.rows),
                "source": "nvml" if self.nvml else "nvidia-smi"}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


class stdout_to_stderr:
    """Sends file descriptor 1 to stderr while the compiled reference runs:
    it prints its set-up messages with printf, and stdout carries only the
    one JSON line."""

    def __enter__(self):
        import ctypes
        self._libc = ctypes.CDLL(None)
        sys.stdout.flush()
        self._libc.fflush(None)
        self._saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        self._libc.fflush(None)
        os.dup2(self._saved, 1)
        os.close(self._saved)
        return False


def run_reference(args, world, rank, pg):
    """The reference's own operators (oracle/_ref) on the host cores.  For
    the ensemble: its first four members one after another, the steps split
    among them."""
    if rank != 0:
        return None
    from oracle.refsim import RefSim
    from cubismup_2d_b200.synthetic import noise_field
    if args.workload == "ensemble":
        from cubismup_2d_b200.synthetic import ensemble_configs
        name = ENSEMBLE_NAME.format(args.members)
        cfgs = ensemble_configs(n=args.members, seed=0)[:4]
        steps = max(1, args.steps // len(cfgs))
        warm = min(args.warmup, 1)
        sample = (f"members 0-{len(cfgs) - 1} of the ensemble one after another, {steps} timed steps "
                  f"each after {warm} warm-up step(s); ")
    else:
        name, argline = WORKLOADS[args.workload]
        cfgs, steps, warm = [argline], args.steps, args.warmup
        sample = f"{steps} timed steps after {warm} warm-up steps; "
    cores = os.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    el, cell_steps, prof = 0.0, 0, {}
    with stdout_to_stderr():
        for i, argline in enumerate(cfgs):
            r = RefSim(argline)
            for comp, fname in enumerate(("u", "v")):
                r.set(fname, r.get(fname) + noise_field(i, comp, r.ny, r.nx))
            for _ in range(warm):
                r.step()
            r.profile_reset()
            t0 = time.perf_counter()
            for _ in range(steps):
                r.step()
            el += time.perf_counter() - t0
            cell_steps += r.nx * r.ny * steps
            for k, v in r.profile().items():
                prof[k] = prof.get(k, 0.0) + v
            del r
    val = cell_steps / el / 1e9
    nsteps = steps * len(cfgs)
    line = {
        "impl": "reference", "metric": "cell-steps/s", "value": val, "unit": "Gcell-steps/s",
        "n_gpus": world, "steps": nsteps, "warmup": warm, "ms_per_step": el / nsteps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": name,
                   ("cells_per_member_step" if args.workload == "ensemble" else "cells"): cell_steps // nsteps},
        "cpu_baseline": {"value": val, "unit": "Gcell-steps/s", "cores": cores, "kind": "reference",
                         "sample": sample + "reference operators compiled from its sources with OpenMP; "
                                            "FFT = project FFTW-API stand-in (FFTW absent)"},
        "e2e": {"value": val, "unit": "Gcell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "stage_seconds": {k: round(v, 4) for k, v in prof.items()},
    }
    return line


def cpu_baseline_sample(argline, nsteps=3):
    from oracle.refsim import RefSim
    from cubismup_2d_b200.synthetic import noise_field
    with stdout_to_stderr():
        r = RefSim(argline)
        for comp, fname in enumerate(("u", "v")):
            r.set(fname, r.get(fname) + noise_field(0, comp, r.ny, r.nx))
        r.step()
        t0 = time.perf_counter()
        for _ in range(nsteps):
            r.step()
        el = time.perf_counter() - t0
    return r.nx * r.ny * nsteps / el / 1e9, os.cpu_count(), nsteps


def make_sim(argline, local, rank):
    from cubismup_2d_b200 import Simulation
    from cubismup_2d_b200.synthetic import noise_field
    sim = Simulation(argline)
    sim.cfg.device = local
    sim.init()
    ctx = sim.ctx
    for comp, fname in enumerate(("u", "v")):
        ctx.set(fname, ctx.get(fname) + noise_field(rank, comp, ctx.ny, ctx.nx))
    return sim


def timed_steps(ctx, steps, flush, pg):
    """K graph steps, each between CUDA events on the library's stream, the
    L2 flushed before each; returns (total ms, kernel launches)."""
    import torch
    launches0 = ctx.kernel_launches()
    step_ms = []
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    for _ in range(steps):
        flush.fill_(1.0)                     # evict L2 between timed steps
        torch.cuda.synchronize()
        step_ms.append(ctx.time_step())
    torch.cuda.synchronize()
    return float(np.sum(step_ms)), ctx.kernel_launches() - launches0


DENSE_KERNELS = ("fft_cols", "advdiff", "pcorr", "fft_rows_fwd", "fft_rows_inv", "rhs_div", "max_u")


def dense_roofline(ctx, peak, peak_kind, workload, reps=30):
    """Every dense kernel timed live (CUDA events around each launch on the
    library's stream, the L2 flushed before every launch, so that inputs
    come from HBM); the slowest one is the roofline's kernel."""
    cells = ctx.nx * ctx.ny
    kt = {k: ctx.time_kernel(k, reps, flush_l2=True) for k in DENSE_KERNELS}
    dom = max(kt, key=kt.get)
    achieved = ALGO_BYTES_PER_CELL[dom] * cells / (kt[dom] * 1e-3) / 1e9
    per = {k: {"ms": round(v, 5), "GB/s": round(ALGO_BYTES_PER_CELL[k] * cells / (v * 1e-3) / 1e9, 1),
               "frac": round(ALGO_BYTES_PER_CELL[k] * cells / (v * 1e-3) / 1e9 / peak, 4)}
           for k, v in kt.items()}
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
            "unit": "GB/s", "frac": achieved / peak, "traffic": TRAFFIC_BYTES.get((workload, dom)),
            "algorithmic_bytes_per_launch": ALGO_BYTES_PER_CELL[dom] * cells,
            "timing": "CUDA events around each launch, L2 flushed before each by reading a 256 MB buffer (clean lines: no write-back charged to the launch)",
            "kernels": per}


def div_2h(u, v, h):
    """The divergence of PressureSingle's RHS (PressureSingle.cpp:112-128):
    central differences over 2h, zero-gradient ghosts at the domain edge."""
    ue = np.concatenate([u[:, 1:], u[:, -1:]], axis=1)
    uw = np.concatenate([u[:, :1], u[:, :-1]], axis=1)
    vn = np.concatenate([v[1:, :], v[-1:, :]], axis=0)
    vs = np.concatenate([v[:1, :], v[:-1, :]], axis=0)
    return (ue - uw + vn - vs) / (2 * h)


def fp32_error_report(argline, local, rank, nsteps, sample=50):
    """The FP32-transform path against the FP64 path over nsteps graph steps
    from the same state: the body's speed (time-averaged over the run and
    worst sample), its force (worst sample, against the largest force), the
    fields at the end, and the divergence difference against the FP64 path's
    own divergence (the discretisation floor: the reference's projection is
    not discretely divergence-free)."""
    a = make_sim(argline, local, rank)
    b = make_sim(argline + " -precision fp32", local, rank)
    spd_a, spd_b, fx_a, fx_b = [], [], [], []
    done = 0
    while done < nsteps:
        n = min(sample, nsteps - done)
        a.ctx.advance(n)
        b.ctx.advance(n)
        done += n
        sa, sb = a.ctx.shape(0), b.ctx.shape(0)
        spd_a.append(np.hypot(sa["u"], sa["v"]))
        spd_b.append(np.hypot(sb["u"], sb["v"]))
        fx_a.append(sa["forcex"])
        fx_b.append(sb["forcex"])
    a.ctx.sync()
    b.ctx.sync()
    spd_a, spd_b, fx_a, fx_b = map(np.array, (spd_a, spd_b, fx_a, fx_b))
    fields = {}
    for f in ("u", "v", "pres"):
        fa, fb = a.ctx.get(f), b.ctx.get(f)
        fields[f] = float(np.max(np.abs(fb - fa)) / max(np.max(np.abs(fa)), 1e-300))
    h = a.ctx.h
    da = div_2h(a.ctx.get("u"), a.ctx.get("v"), h)
    db = div_2h(b.ctx.get("u"), b.ctx.get("v"), h)
    fscale = max(np.max(np.abs(fx_a)), 1e-300)
    return {"steps": nsteps, "sample_every": sample,
            "speed_mean_rel_err": float(abs(spd_b.mean() - spd_a.mean()) / max(spd_a.mean(), 1e-300)),
            "speed_max_rel_err": float(np.max(np.abs(spd_b - spd_a)) / max(np.max(spd_a), 1e-300)),
            "force_x_max_rel_err": float(np.max(np.abs(fx_b - fx_a)) / fscale),
            "fields_rel_err_end": fields,
            "div_delta_inf": float(np.max(np.abs(db - da))),
            "div_fp64_inf": float(np.max(np.abs(da))),
            "against": "this library's FP64 path (itself parity-tested against the reference)"}


def cufft_comparison(ctx, flush, reps=20):
    """The free-space solve's convolution done by cuFFT (through torch.fft,
    a comparison only, never on the product path): a double-precision 2D
    real-to-complex FFT of the zero-padded 2Ny x 2Nx RHS, times the real
    kernel, and the complex-to-real inverse, timed with CUDA events with the
    L2 flushed before each solve; beside the sum of this library's three
    transform passes timed the same way."""
    import torch
    nx, ny = ctx.nx, ctx.ny
    dev = flush.device
    x = torch.zeros(2 * ny, 2 * nx, dtype=torch.float64, device=dev)
    x[:ny, :nx] = torch.rand(ny, nx, dtype=torch.float64, device=dev)
    g = torch.rand(2 * ny, nx + 1, dtype=torch.float64, device=dev)
    for _ in range(3):
        y = torch.fft.irfft2(torch.fft.rfft2(x) * g, s=x.shape)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    for _ in range(reps):
        flush.fill_(1.0)
        e0.record()
        y = torch.fft.irfft2(torch.fft.rfft2(x) * g, s=x.shape)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    del y
    ours = sum(ctx.time_kernel(k, reps, flush_l2=True) for k in ("fft_rows_fwd", "fft_cols", "fft_rows_inv"))
    cu = float(np.mean(ms))
    return {"cufft_ms": round(cu, 5), "ours_ms": round(ours, 5), "ours_speedup": round(cu / ours, 3),
            "transform": f"D2Z/Z2D {2 * ny}x{2 * nx} (zero-padded free-space convolution), FP64",
            "note": "cuFFT via torch.fft, comparison only; ours = the three hand-written passes "
                    "(fade, zero halves skipped, kernel multiply fused)"}


LARGE_CASE = "tandem"


def operator_steps(sim, steps, pg):
    """Steps through the operator path (calcMaxTimestep, the four operators,
    end_step), as Simulation::advance calls them; the iterated operators read
    each iteration's change back, so the host waits on the device inside
    every step anyway.  Returns (host ms of the K steps after a device
    synchronisation on both sides, iterations per step)."""
    import torch
    its = []
    if pg is not None:
        pg.barrier()
    sim.ctx.sync()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        dt = sim.calcMaxTimestep()
        for op in sim.pipeline:
            op(dt)
        sim.ctx.end_step()
        its.append(sim.ctx.iteration_stats()[0])
    sim.ctx.sync()
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) * 1e3, its


def falling_measurement(local, rank, pg, warmup=3, steps=6):
    """The large case with its falling cylinder (variable density)."""
    name, argline = WORKLOADS["tandem_falling"]
    sim = make_sim(argline, local, rank)
    cells = sim.ctx.nx * sim.ctx.ny
    _, its_w = operator_steps(sim, warmup, pg)
    ms, its = operator_steps(sim, steps, pg)
    ms = max_over_ranks(pg, ms)
    out = {"workload": name, "value": cells * steps / (ms / 1e3) / 1e9, "unit": "Gcell-steps/s",
           "ms_per_step": ms / steps, "steps": steps, "warmup": warmup,
           "iterations_per_step": its, "iterations_warmup": its_w,
           "pipeline": [op.name for op in sim.pipeline],
           "timing": "host clock around K operator steps, device synchronised on both sides "
                     "(the iterated operator synchronises every iteration)",
           "disk_v_after": sim.ctx.shape(2)["v"]}
    del sim
    return out


def adjoint_measurement(local, rank, pg, warm=50, nsteps=200, every=20):
    """The discrete adjoint on the forced cylinder (512x256): the gradient of
    the time-averaged drag force over 200 steps (checkpoints every 20) with
    respect to the initial velocity and the body's velocity; its cost against
    the same 200 steps as graph steps and as operator steps, and the body
    velocity gradient against a central difference of the forward."""
    name, argline = WORKLOADS["cylinder"]
    sim = make_sim(argline, local, rank)
    ctx = sim.ctx
    ctx.advance(warm)
    ctx.sync()
    blob = ctx.checkpoint()
    obj = dict(box=None, w_force=(1.0, 0.0))
    ctx.adjoint(nsteps, every=every, **obj)             # warm-up (allocations, first launches)
    ctx.restore(blob)
    J, gu, gv, gb, dts, ms = ctx.adjoint(nsteps, every=every, **obj)
    ctx.restore(blob)
    graph_ms = ctx.time_step(nsteps)
    eps, ub, Js = 1e-6, ctx.shape(0)["u"], []
    for sgn in (1, -1):
        ctx.restore(blob)
        ctx.set_shape(0, {"u": ub + sgn * eps})
        Js.append(ctx.adjoint(nsteps, dt=dts, gradient=False, **obj)[0])
    fd = (Js[0] - Js[1]) / (2 * eps)
    bwd = max_over_ranks(pg, ms[1])
    out = {"workload": name, "steps": nsteps, "checkpoint_every": every, "warm_steps_before": warm,
           "objective": "time-averaged forcex (ComputeForces) over the steps",
           "J": J, "forward_graph_ms": graph_ms, "forward_operator_ms_with_checkpoints": ms[0],
           "backward_ms": bwd, "adjoint_over_forward": bwd / graph_ms,
           "adjoint_over_forward_operator": bwd / ms[0],
           "fd_check": {"parameter": "body velocity u", "adjoint": float(gb[0]), "central_difference": fd,
                        "eps": eps, "rel_err": abs(gb[0] - fd) / max(abs(fd), 1e-300)},
           "timing": "CUDA events on the context's stream; backward = the recomputation from the "
                     f"checkpoints plus the transposed steps; forward = the same {nsteps} steps as graph steps"}
    del sim
    return out


def gait_measurement(local, rank, pg, warm=1500, nsteps=200, every=20):
    """The gait gradient of the benchmark's adjoint case on a held swimmer:
    the carangiform envelope swimmer (L = 0.2, 512x256, Re = 1000 on L and
    the 0.2 stream it is held in, past its first period), its curvature
    amplitude's eight Fourier coefficients drawn from a seeded N(1, 0.05),
    objective the time-averaged forcex plus 0.1 mean |torque| over 200
    steps (checkpoints every 20); its cost against the same steps as graph
    steps, and the gradient against central differences of the whole
    simulation."""
    argline = ("-bpdx 16 -bpdy 8 -extent 1 -CFL 0.1 -nu 4e-5 -lambda 1e4 -poissonType freespace -muteAll 1 "
               "-shapes 'envelopefish L=0.2 T=1 xpos=0.4 ypos=0.25 bFixed=1 bForced=1 xvel=0.2'")
    sim = make_sim(argline, local, rank)
    ctx = sim.ctx
    ctx.set_fish_gait(0, np.random.default_rng(2024).normal(1.0, 0.05, 8))
    ctx.advance(warm)
    ctx.sync()
    blob = ctx.checkpoint()
    obj = dict(box=None, w_force=(1.0, 0.0), w_torque=0.1)
    eps = 1e-7                      # the placement's and the whole simulation's difference step
    J, gu, gv, gb, dts, ms, gg = ctx.adjoint(nsteps, every=every, gait=True, gait_step=eps, **obj)
    ctx.restore(blob)
    graph_ms = ctx.time_step(nsteps)
    theta = ctx.fish_gait(0)

    def central(n, q, dt):
        Js = []
        for sgn in (1, -1):
            ctx.restore(blob)
            th = theta.copy()
            th[q] += sgn * eps
            ctx.set_fish_gait(0, th)
            Js.append(ctx.adjoint(n, dt=dt, gradient=False, **obj)[0])
            ctx.set_fish_gait(0, theta)
        return (Js[0] - Js[1]) / (2 * eps)

    fd = central(nsteps, 0, dts)
    # a short horizon (fewer raster switches within the step)
    ctx.restore(blob)
    short = 16
    _, _, _, _, dts16, _, gg16 = ctx.adjoint(short, every=short, gait=True, gait_step=eps, **obj)
    fd16 = [central(short, q, dts16) for q in range(8)]
    ctx.restore(blob)
    out = {"workload": "tethered_envelope_swimmer_512x256_re1000_fp64", "steps": nsteps,
           "checkpoint_every": every, "warm_graph_steps_before": warm,
           "objective": "time-averaged forcex + 0.1 mean |torque| (ComputeForces) over the steps",
           "parameters": "the 8 Fourier coefficients of the curvature amplitude, seeded N(1, 0.05)",
           "theta": [float(x) for x in theta],
           "J": J, "grad_gait": [float(x) for x in gg],
           "forward_graph_ms": graph_ms, "backward_ms": ms[1], "gait_replay_ms": ms[2],
           "adjoint_over_forward": ms[1] / graph_ms,
           "gradient_over_forward": (ms[1] + ms[2]) / graph_ms,
           "fd_check": {"parameter": "f_0", "adjoint": float(gg[0]), "central_difference": fd,
                        "eps": eps, "rel_err": abs(gg[0] - fd) / max(abs(fd), 1e-300)},
           "fd_check_16_steps": {"adjoint": [float(x) for x in gg16], "central_difference": fd16,
                                 "max_rel_err": max(abs(a - b) / max(abs(b), 1e-300) for a, b in zip(gg16, fd16))},
           "method": "flow: discrete adjoint with checkpointed recomputation; the body geometry's "
                     "dependence on the gait: central differences of the placement alone (16 replays)"}
    del sim
    return out


def run_ours(args, world, rank, local, pg):
    import torch
    name, argline = WORKLOADS[args.workload]
    torch.cuda.set_device(local)
    sim = make_sim(argline, local, rank)
    ctx = sim.ctx
    cells = ctx.nx * ctx.ny
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    # warm-up (also captures the step graph)
    ctx.advance(max(args.warmup, 3))
    ctx.sync()

    with ClockSampler(local) as clk:
        total_ms, launches = timed_steps(ctx, args.steps, flush, pg)
    total_ms = max_over_ranks(pg, total_ms)
    value = world * cells * args.steps / (total_ms / 1e3) / 1e9

    # the same workload with the FP32 Poisson transforms (CUP2D_PREC_FP32):
    # pressure after one step from the same state against FP64, then timed
    fp32 = None
    if not args.no_fp32:
        a = make_sim(argline, local, rank)
        b = make_sim(argline + " -precision fp32", local, rank)
        a.ctx.advance(1); b.ctx.advance(1)
        pa, pb = a.ctx.get("pres"), b.ctx.get("pres")
        perr = float(np.max(np.abs(pb - pa)) / max(np.max(np.abs(pa)), 1e-300))
        del a
        b.ctx.advance(max(args.warmup, 3))
        b.ctx.sync()
        ms32, _ = timed_steps(b.ctx, args.steps, flush, pg)
        ms32 = max_over_ranks(pg, ms32)
        fp32 = {"value": world * cells * args.steps / (ms32 / 1e3) / 1e9, "unit": "Gcell-steps/s",
                "ms_per_step": ms32 / args.steps, "speedup_vs_fp64": total_ms / ms32,
                "pres_rel_err_1step": perr,
                "transform_ms": {k: round(b.ctx.time_kernel(k, 20, flush_l2=True), 5)
                                 for k in ("fft_rows_fwd", "fft_cols", "fft_rows_inv")},
                "note": "FP32 free-space Poisson transforms; fields, stencils, obstacle sums and "
                        "forces FP64; Cd within 1e-4 of FP64 is checked by tests/test_gpu_fp32.py"}
        del b

    if fp32 is not None and args.fp32_report_steps > 0:
        fp32["error_report"] = fp32_error_report(argline, local, rank, args.fp32_report_steps)

    # e2e: the reference's own loop through the C ABI with host transfers per
    # step: dt read back (calcMaxTimestep prints it), dt passed to the four
    # operators, shape state (forces) read back for the force log.
    ne = max(20, args.steps // 5)
    from cubismup_2d_b200.abi import ShapeState
    st0 = ShapeState()                     # the forces, read each step into one struct
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(ne):
        dt = sim.calcMaxTimestep()
        for op in sim.pipeline:
            op(dt)
        ctx.end_step()
        ctx.shape_state(0, st0)
    ctx.sync()
    e2e_s = max_over_ranks(pg, time.perf_counter() - t0)
    e2e = world * cells * ne / e2e_s / 1e9

    # roofline of the dominant dense kernel, timed live with CUDA events
    peak, peak_kind = measured_peaks()
    roof = dense_roofline(ctx, peak, peak_kind, args.workload)
    cufft = None if args.no_cufft else cufft_comparison(ctx, flush)
    ctx.sync()
    # the same at the large case's size (4096x2048), where the working set
    # exceeds the L2 by itself
    roof_large = None
    if not args.no_large and args.workload != LARGE_CASE:
        lname, largs = WORKLOADS[LARGE_CASE]
        big = make_sim(largs, local, rank)
        big32 = None if args.no_fp32 else make_sim(largs + " -precision fp32", local, rank)
        big.ctx.advance(1)
        step_large = {}
        if big32 is not None:
            big32.ctx.advance(1)
            pa, pb = big.ctx.get("pres"), big32.ctx.get("pres")
            step_large["pres_rel_err_1step_fp32"] = float(np.max(np.abs(pb - pa)) / max(np.max(np.abs(pa)), 1e-300))
            del pa, pb
        big.ctx.advance(3)
        big.ctx.sync()
        roof_large = dense_roofline(big.ctx, peak, peak_kind, LARGE_CASE)
        roof_large["workload"] = lname
        # the whole graph step at this size, FP64 and with the FP32 Poisson
        # transforms, timed as the headline's steps (L2 flushed before each)
        nl = 30
        ms64, _ = timed_steps(big.ctx, nl, flush, pg)
        step_large["fp64_ms_per_step"] = max_over_ranks(pg, ms64) / nl
        if big32 is not None:
            big32.ctx.advance(3)
            big32.ctx.sync()
            ms32, _ = timed_steps(big32.ctx, nl, flush, pg)
            step_large["fp32_transforms_ms_per_step"] = max_over_ranks(pg, ms32) / nl
            step_large["fp32_transforms_speedup"] = ms64 / ms32
            step_large["fp32_transform_ms"] = {k: round(big32.ctx.time_kernel(k, 20, flush_l2=True), 5)
                                               for k in ("fft_rows_fwd", "fft_cols", "fft_rows_inv")}
            del big32
        step_large["steps"] = nl
        roof_large["step"] = step_large
        if not args.no_cufft:
            roof_large["cufft"] = cufft_comparison(big.ctx, flush)
        del big
    falling = None
    if not args.no_large and not args.no_falling:
        falling = falling_measurement(local, rank, pg)
    adjoint = None if args.no_adjoint else adjoint_measurement(local, rank, pg)
    if adjoint is not None:
        adjoint["gait"] = gait_measurement(local, rank, pg)

    line = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            try:
                v, cores, n = cpu_baseline_sample(argline, nsteps=args.cpu_steps)
                cpu = {"value": v, "unit": "Gcell-steps/s", "cores": cores, "kind": "reference",
                       "sample": f"{n} steps of the same workload after 1 warm-up step; reference "
                                 "operators compiled from its sources (OpenMP, all host cores); "
                                 "FFT = project FFTW-API stand-in (FFTW absent)"}
            except Exception as e:  # noqa: BLE001
                cpu = {"value": None, "unit": "Gcell-steps/s", "cores": os.cpu_count(), "kind": "reference",
                       "sample": f"unavailable: {e}"}
        line = {
            "metric": "cell-steps/s", "value": value, "unit": "Gcell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": name, "cells": cells},
            "timing": {"parallelism": f"replicas{world}",
                       "l2": "flushed between timed steps (256 MB write)"},
            "clocks": clk.summary(),
            "e2e": {"value": e2e, "unit": "Gcell-steps/s", "h2d_bytes_per_step": 8,
                    "d2h_bytes_per_step": 8 + 42 * 8, "steps": ne},
            "gpu_launches": launches,
            "roofline": roof,
            "roofline_large": roof_large,
            "poisson_vs_cufft": cufft,
            "fp32": fp32,
            "falling_cylinder_large": falling,
            "adjoint": adjoint,
            "cpu_baseline": cpu,
        }
    return line


def run_ensemble(args, world, rank, local, pg):
    """The batched ensemble: M members, one graph launch per ensemble step."""
    import torch
    from cubismup_2d_b200 import Ensemble
    from cubismup_2d_b200.synthetic import ensemble_configs
    torch.cuda.set_device(local)
    cfgs = ensemble_configs(n=args.members, seed=0)
    sims = [make_sim(a, local, 1000 * rank + i) for i, a in enumerate(cfgs)]
    sizes = [s.ctx.nx * s.ctx.ny for s in sims]
    cells = int(sum(sizes))
    ens = Ensemble(sims)
    ens.advance(max(args.warmup, 3))
    ens.sync()
    launches0 = sum(s.ctx.kernel_launches() for s in sims)
    with ClockSampler(local) as clk:
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()
        total_ms = ens.advance_timed(args.steps)
    launches = sum(s.ctx.kernel_launches() for s in sims) - launches0
    total_ms = max_over_ranks(pg, total_ms)
    value = world * cells * args.steps / (total_ms / 1e3) / 1e9

    # the same members one after another, each on its own step graph
    for s in sims:
        s.ctx.advance(3)
    ens.sync()
    seq_ms = max_over_ranks(pg, float(sum(s.ctx.time_step(args.steps) for s in sims)))
    seq_value = world * cells * args.steps / (seq_ms / 1e3) / 1e9

    # e2e: an ensemble step, then every member's shape states read back
    ne = max(10, args.steps // 10)
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(ne):
        ens.advance(1)
        _ = ens.shape_states()
    ens.sync()
    e2e_s = max_over_ranks(pg, time.perf_counter() - t0)
    e2e = world * cells * ne / e2e_s / 1e9

    # FP32 Poisson transforms on the same members
    fp32 = None
    if not args.no_fp32:
        del ens
        sims32 = [make_sim(a + " -precision fp32", local, 1000 * rank + i) for i, a in enumerate(cfgs)]
        ens32 = Ensemble(sims32)
        ens32.advance(max(args.warmup, 3))
        ens32.sync()
        ms32 = max_over_ranks(pg, ens32.advance_timed(args.steps))
        fp32 = {"value": world * cells * args.steps / (ms32 / 1e3) / 1e9, "unit": "Gcell-steps/s",
                "ms_per_step": ms32 / args.steps, "speedup_vs_fp64": total_ms / ms32,
                "note": "FP32 free-space Poisson transforms; fields, stencils, obstacle sums and forces FP64"}
        del ens32, sims32

    # roofline: the dominant dense kernel of the largest member
    peak, peak_kind = measured_peaks()
    big = sims[int(np.argmax(sizes))]
    roof = dense_roofline(big.ctx, peak, peak_kind, "ensemble")
    roof["member"] = f"{big.ctx.nx}x{big.ctx.ny}"

    line = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            try:
                v, cores, n = cpu_baseline_sample(cfgs[0], nsteps=args.cpu_steps)
                cpu = {"value": v, "unit": "Gcell-steps/s", "cores": cores, "kind": "reference",
                       "sample": f"{n} steps of member 0 ({sims[0].ctx.nx}x{sims[0].ctx.ny}) after 1 "
                                 "warm-up step; reference operators compiled from its sources (OpenMP, "
                                 "all host cores); FFT = project FFTW-API stand-in (FFTW absent)"}
            except Exception as e:  # noqa: BLE001
                cpu = {"value": None, "unit": "Gcell-steps/s", "cores": os.cpu_count(), "kind": "reference",
                       "sample": f"unavailable: {e}"}
        grids = {}
        for s in sims:
            key = f"{s.ctx.nx}x{s.ctx.ny}"
            grids[key] = grids.get(key, 0) + 1
        line = {
            "metric": "cell-steps/s", "value": value, "unit": "Gcell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": ENSEMBLE_NAME.format(args.members), "members": args.members,
                       "cells": cells, "grids": grids,
                       "shapes": {"disk": sum("disk" in a for a in cfgs),
                                  "stefanfish": sum("stefanfish" in a for a in cfgs)}},
            "timing": {"parallelism": f"replicas{world}",
                       "l2": "not flushed: the members' fields (~2 GB at 64 members) exceed the L2"},
            "clocks": clk.summary(),
            "sequential": {"value": seq_value, "unit": "Gcell-steps/s", "ms_per_step": seq_ms / args.steps,
                           "speedup_of_ensemble": seq_ms / total_ms,
                           "note": "the same members one after another, each on its own step graph"},
            "e2e": {"value": e2e, "unit": "Gcell-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": len(sims) * 42 * 8, "steps": ne},
            "gpu_launches": launches,
            "roofline": roof,
            "fp32": fp32,
            "cpu_baseline": cpu,
        }
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    # (tandem_falling is measured beside the headline: its steps are not graph steps)
    ap.add_argument("--workload", default="swimmer",
                    choices=sorted(k for k in WORKLOADS if k != "tandem_falling") + ["ensemble"])
    ap.add_argument("--members", type=int, default=64, help="ensemble members (--workload ensemble)")
    ap.add_argument("--cpu-steps", type=int, default=6)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp32", action="store_true", help="skip the FP32-Poisson measurement")
    ap.add_argument("--no-large", action="store_true", help="skip the 4096x2048 kernel roofline")
    ap.add_argument("--fp32-report-steps", type=int, default=2000,
                    help="steps of the FP32-against-FP64 error report (0: skip)")
    ap.add_argument("--no-cufft", action="store_true", help="skip the cuFFT comparison")
    ap.add_argument("--no-falling", action="store_true",
                    help="skip the 4096x2048 case with the falling cylinder (variable density)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint measurement")
    ap.add_argument("--adjoint-only", type=int, default=0, metavar="N",
                    help="run only the adjoint measurement, over N steps in one checkpoint segment")
    args = ap.parse_args()
    world, rank, local, pg = dist_setup()
    if args.adjoint_only > 0:
        import torch
        torch.cuda.set_device(local)
        out = adjoint_measurement(local, rank, pg, nsteps=args.adjoint_only, every=args.adjoint_only)
        if rank == 0:
            print(json.dumps(out))
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()
        return
    if args.impl == "reference":
        # a step of the reference at 1024x512 takes ~0.1 s on 16 host cores:
        # bound the sample to 20 timed steps (same warm-up as our arm)
        args.steps = min(args.steps, 20)
        line = run_reference(args, world, rank, pg)
    elif args.workload == "ensemble":
        line = run_ensemble(args, world, rank, local, pg)
    else:
        line = run_ours(args, world, rank, local, pg)
    if rank == 0 and line is not None:
        print(json.dumps(line))
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
