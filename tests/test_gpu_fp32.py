"""The FP32 Poisson transforms (CUP2D_PREC_FP32) against the FP64 pipeline.

Only the free-space / periodic FFT passes change arithmetic; fields, stencils,
obstacle sums and forces stay FP64.  The bar is the one the benchmark names
for the reduced-precision pipeline: drag coefficient within 1e-4 relative of
the FP64 path, here on the forced cylinder at Re = 100 after 200 steps.
Pressure after one step is checked at the FP32 rounding level of the
transforms (1e-5 relative to max |p|).
"""
import numpy as np
import pytest

from cubismup_2d_b200 import Simulation
from cubismup_2d_b200.synthetic import FORCED_CYLINDER_RE100, SWIMMER_1024x512, noise_field

pytestmark = pytest.mark.gpu

PERIODIC_DISK = ("-bpdx 8 -bpdy 8 -extent 1 -CFL 0.1 -nu 1e-3 -lambda 1e4 -poissonType periodic "
                 "-shapes 'disk radius=0.1 xpos=0.5 ypos=0.5 bForced=1 xvel=0.1'")


def _pair(argline, seed=5):
    sims = []
    for prec in ("fp64", "fp32"):
        s = Simulation(argline + f" -precision {prec}")
        s.init()
        for comp, f in enumerate(("u", "v")):
            s.ctx.set(f, s.ctx.get(f) + noise_field(seed, comp, s.ctx.ny, s.ctx.nx))
        sims.append(s)
    return sims


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("argline", [SWIMMER_1024x512, PERIODIC_DISK], ids=["freespace_swimmer", "periodic_disk"])
def test_fp32_pressure_one_step(argline):
    s64, s32 = _pair(argline)
    for s in (s64, s32):
        s.ctx.advance(1)
        s.ctx.sync()
    assert _rel(s32.ctx.get("pres"), s64.ctx.get("pres")) < 1e-5
    for f in ("u", "v"):
        assert _rel(s32.ctx.get(f), s64.ctx.get(f)) < 1e-5


def test_fp32_cylinder_cd_200_steps():
    s64, s32 = _pair(FORCED_CYLINDER_RE100, seed=3)
    U, D = 0.2, 2 * 0.0375
    for s in (s64, s32):
        s.ctx.advance(200)
        s.ctx.sync()
    a, b = s32.ctx.shape(0), s64.ctx.shape(0)
    cd32, cd64 = 2 * a["forcex"] / (U * U * D), 2 * b["forcex"] / (U * U * D)
    assert abs(cd32 - cd64) <= 1e-4 * abs(cd64), (cd32, cd64)


def test_fp32_cosine_not_available():
    with pytest.raises(Exception):
        s = Simulation("-bpdx 4 -bpdy 4 -poissonType cosine -precision fp32 -shapes 'disk radius=0.1 xpos=0.5 ypos=0.5'")
        s.init()
