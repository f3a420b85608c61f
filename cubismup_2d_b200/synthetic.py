"""Seeded synthetic inputs shared by tests and bench.py.

The benchmark configurations start "from rest plus seeded 1e-6 uniform
noise on u, v" (the reference's own IC noise is commented out,
Helpers.cpp:52-54, 75-79).  The noise is a counter-based hash
(SplitMix64 finaliser) of (seed, component, global cell index), so any
grid size, any device and the CPU oracle see identical values.
"""
import numpy as np

M64 = (1 << 64) - 1


def _splitmix64(x):
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(M64)
    z = x
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9) & np.uint64(M64)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB) & np.uint64(M64)
    return z ^ (z >> np.uint64(31))


def noise_field(seed, component, ny, nx, amp=1e-6):
    """(ny, nx) array uniform in [-amp, amp), row-major global cell index."""
    with np.errstate(over="ignore"):
        idx = np.arange(ny * nx, dtype=np.uint64)
        key = (np.uint64(seed) * np.uint64(0x100000001B3) + np.uint64(component + 1)) & np.uint64(M64)
        z = _splitmix64(idx ^ (key << np.uint64(32)) ^ key)
    u01 = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return (amp * (2.0 * u01 - 1.0)).reshape(ny, nx)


# Workloads of the benchmark configurations, as reference command lines.
FORCED_CYLINDER_RE100 = (
    "-bpdx 16 -bpdy 8 -extent 1 -CFL 0.1 -nu 1.5e-4 -lambda 1e4 -poissonType freespace "
    "-nsteps 1000 -shapes 'disk radius=0.0375 xpos=0.2 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'")
SWIMMER_1024x512 = (
    "-bpdx 32 -bpdy 16 -extent 1 -CFL 0.1 -nu 2e-5 -lambda 1e4 -poissonType freespace "
    "-nsteps 2000 -shapes 'stefanfish L=0.2 T=1 xpos=0.4 ypos=0.25'")

# Grids of the ensemble members (blocks of 32x32 cells): 256x128, 512x256,
# 768x384 and 1024x512.
ENSEMBLE_GRIDS = [(8, 4), (16, 8), (24, 12), (32, 16)]


def fish_length_ok(L, h):
    """Whether FishData's arclength grid exists for a fish of length L on
    spacing h (FishLibrary.cpp:14-38: the refined end spacing dSref must be
    positive, the assertion at line 21); the reference aborts otherwise."""
    ds_mid_tgt, ds_refine_tgt = h / np.sqrt(2.0), 0.125 * h
    n_mid = int(np.ceil(L * 0.8 / ds_mid_tgt / 8)) * 8
    ds_mid = L * 0.8 / n_mid
    n_end = int(np.ceil(0.1 * L * 2 / (ds_mid + ds_refine_tgt) / 4)) * 4
    return 0.1 * L * 2 / n_end - ds_mid > 0


def ensemble_configs(n=64, seed=0):
    """Reference command lines of n independent members drawn from a seed:
    the grid from ENSEMBLE_GRIDS; a forced cylinder (radius in [0.02, 0.05],
    u = 0.2, nu = U 2R / Re) or a StefanFish (L in [0.15, 0.25], redrawn
    until the fish's arclength grid exists at the member's spacing, T = 1,
    nu = (L/T) L / Re); Re log-uniform in [100, 1000]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        bx, by = ENSEMBLE_GRIDS[rng.integers(len(ENSEMBLE_GRIDS))]
        re = float(np.exp(rng.uniform(np.log(100.0), np.log(1000.0))))
        grid = (f"-bpdx {bx} -bpdy {by} -extent 1 -CFL 0.1 -lambda 1e4 -poissonType freespace -nsteps 500 "
                "-muteAll 1")
        if rng.uniform() < 0.5:
            r = float(rng.uniform(0.02, 0.05))
            nu = 0.2 * 2 * r / re
            out.append(f"{grid} -nu {nu:.17g} -shapes 'disk radius={r:.17g} xpos=0.2 ypos=0.25 "
                       "bForced=1 bFixed=1 xvel=0.2'")
        else:
            L = float(rng.uniform(0.15, 0.25))
            while not fish_length_ok(L, 1.0 / (32 * max(bx, by))):
                L = float(rng.uniform(0.15, 0.25))
            nu = L * L / re
            out.append(f"{grid} -nu {nu:.17g} -shapes 'stefanfish L={L:.17g} T=1 xpos=0.4 ypos=0.25'")
    return out
