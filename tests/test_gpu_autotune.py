"""The transform autotuner (cup2d_config.autotune): the row passes' variants
are timed on the grid at set-up and the faster kept; every context of the
grid then takes the same variants (bitwise-equal runs), and the solution
differs from the built-in choice by rounding only."""
import numpy as np
import pytest

from cubismup_2d_b200 import Simulation
from cubismup_2d_b200.synthetic import noise_field

pytestmark = pytest.mark.gpu

ARGS = ("-bpdx 32 -bpdy 16 -extent 1 -CFL 0.1 -nu 2e-5 -poissonType freespace -muteAll 1 "
        "-shapes 'stefanfish L=0.2 T=1 xpos=0.4 ypos=0.25'")


def _run(args, steps=3):
    s = Simulation(args)
    s.init()
    for comp, f in enumerate(("u", "v")):
        s.ctx.set(f, s.ctx.get(f) + noise_field(1, comp, s.ctx.ny, s.ctx.nx))
    s.ctx.advance(steps)
    s.ctx.sync()
    return s


def test_tuned_contexts_agree_and_match_the_built_in_choice():
    a = _run(ARGS + " -autotune 1")
    b = _run(ARGS + " -autotune 1")
    c = _run(ARGS)
    ta, tb, tc = a.ctx.tuning(), b.ctx.tuning(), c.ctx.tuning()
    assert ta["tuned"] and tb["tuned"] and not tc["tuned"]
    assert ta["fft_rows_fwd_e"] in (8, 16) and ta["fft_rows_inv_e"] in (8, 16)
    assert all(t > 0 for t in ta["us"])
    # the second context of the grid reuses the first one's choice
    assert (ta["fft_rows_fwd_e"], ta["fft_rows_inv_e"]) == (tb["fft_rows_fwd_e"], tb["fft_rows_inv_e"])
    for f in ("u", "v", "pres"):
        assert np.array_equal(a.ctx.get(f), b.ctx.get(f)), f
        ref = c.ctx.get(f)
        assert np.max(np.abs(a.ctx.get(f) - ref)) <= 1e-10 * np.max(np.abs(ref)), f
    # the choice follows the measured times
    us = ta["us"]
    assert ta["fft_rows_fwd_e"] == (16 if us[1] < us[0] else 8)
    assert ta["fft_rows_inv_e"] == (16 if us[3] < us[2] else 8)
