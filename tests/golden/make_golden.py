"""Generate the golden fixtures of tests/golden/ from the reference's own code.

    python tests/golden/make_golden.py

Each fixture is the output of oracle/_ref/libcup2d_ref.so -- the reference's
sources compiled unmodified by oracle/Makefile against the project's
stand-ins for Cubism, FFTW and GSL -- on a small configuration started from
rest plus the seeded noise of cubismup_2d_b200.synthetic.noise_field: the
chi field after Simulation::init (Simulation.cpp:171-241), then, after
NSTEPS passes of Simulation::simulate's loop body (calcMaxTimestep +
advance, Simulation.cpp:243-305), the velocity, pressure and chi fields
(disk cases), the time steps taken and every scalar of the first shape
(Shape.h:22-62).  The reference ships no tests or golden data of its own,
so these are the known answers the numpy restatement (oracle/cup2d_oracle.py)
and the CUDA pipeline are checked against.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cubismup_2d_b200.synthetic import noise_field  # noqa: E402
from oracle import refsim  # noqa: E402

NOISE_SEED = 11
COMMON = "-extent 1 -CFL 0.1 -muteAll 1 "
CASES = {
    # name: (arguments, steps, store velocity/pressure fields)
    "disk_forced_freespace": (
        "-bpdx 2 -bpdy 1 " + COMMON + "-nu 1e-3 -lambda 1e4 -poissonType freespace "
        "-shapes 'disk radius=0.1 xpos=0.3 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'", 4, True),
    "disk_free_periodic": (
        "-bpdx 2 -bpdy 1 " + COMMON + "-nu 1e-3 -poissonType periodic "
        "-shapes 'disk radius=0.08 xpos=0.4 ypos=0.22 xvel=0.1 yvel=0.05'", 4, True),
    "disk_free_cosine": (
        "-bpdx 2 -bpdy 1 " + COMMON + "-nu 1e-3 -poissonType cosine "
        "-shapes 'disk radius=0.08 xpos=0.4 ypos=0.22 xvel=0.1 yvel=0.05'", 4, True),
    "stefanfish": (
        "-bpdx 8 -bpdy 4 " + COMMON + "-nu 1e-4 -poissonType freespace "
        "-shapes 'stefanfish L=0.18 T=1 xpos=0.4 ypos=0.25'", 3, False),
    "carlingfish": (
        "-bpdx 8 -bpdy 4 " + COMMON + "-nu 1e-4 -poissonType freespace "
        "-shapes 'carlingfish L=0.18 T=1 xpos=0.4 ypos=0.25 angle=10'", 3, False),
}


def run_case(args, nsteps, fields):
    r = refsim.RefSim(args)
    out = {"args": np.array(args), "noise_seed": np.array(NOISE_SEED), "nsteps": np.array(nsteps)}
    for comp, name in enumerate(("u", "v")):
        r.set(name, r.get(name) + noise_field(NOISE_SEED, comp, r.ny, r.nx))
    out["init_chi"] = r.get("chi")
    dts = [r.step() for _ in range(nsteps)]
    out["dt"] = np.array(dts)
    out["time"] = np.array(r.time)
    if fields:
        for name in ("u", "v", "pres", "chi"):
            out["final_" + name] = r.get(name)
    sh = r.shape(0)
    out["shape_keys"] = np.array(list(sh.keys()))
    out["shape_values"] = np.array(list(sh.values()))
    r.close()
    return out


def main():
    if not refsim.available():
        refsim.build()
    for name, (args, nsteps, fields) in CASES.items():
        data = run_case(args, nsteps, fields)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **data)
        print(f"{name}: {os.path.getsize(path) / 1024:.1f} KB")


if __name__ == "__main__":
    main()
