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
