"""The iterated penalization (-iterativePenalization 1: PressureIterator_unif
in place of PressureSingle, Simulation.cpp:213-216) against the reference's
own operator on the same inputs, step by step through the operator path."""
import numpy as np
import pytest

from cubismup_2d_b200 import Cup2DError, Simulation
from cubismup_2d_b200.synthetic import noise_field

pytestmark = pytest.mark.gpu

ITER = "-extent 1 -CFL 0.1 -poissonType freespace -muteAll 1 -iterativePenalization 1 "
FORCED = ("-bpdx 4 -bpdy 2 -nu 1e-3 -lambda 1e4 " + ITER +
          "-shapes 'disk radius=0.1 xpos=0.3 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'")
FREE = ("-bpdx 4 -bpdy 2 -nu 1e-3 " + ITER +
        "-shapes 'disk radius=0.08 xpos=0.4 ypos=0.22 xvel=0.1 yvel=0.05'")
FISH = ("-bpdx 8 -bpdy 4 -nu 1e-4 " + ITER +
        "-shapes 'stefanfish L=0.18 T=1 xpos=0.4 ypos=0.25'")


def _pair(refsim, args, seed=5):
    r = refsim.RefSim(args)
    s = Simulation(args)
    s.init()
    for comp, name in enumerate(("u", "v")):
        a = r.get(name) + noise_field(seed, comp, r.ny, r.nx)
        r.set(name, a)
        s.ctx.set(name, a)
    return r, s


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("args", [FORCED, FREE, FISH], ids=["forced_disk", "free_disk", "fish"])
def test_iterated_steps_match_reference(ref, args):
    r, s = _pair(ref, args)
    for _ in range(3):
        r.step()
        s.advance(s.calcMaxTimestep())
        # the same number of iterations, step by step (oldNsteps of the
        # reference's operator)
        assert s.ctx.iteration_stats()[0] == r.iterations()
    s.ctx.sync()
    errs = {f: _rel(s.ctx.get(f), r.get(f)) for f in ("u", "v", "pres", "chi")}
    assert all(e <= 1e-9 for e in errs.values()), errs
    a, b = s.ctx.shape(0), r.shape(0)
    for key in ("u", "v", "omega", "center_x", "center_y", "penalM", "penalJ", "fluidMomX",
                "fluidMomY", "forcex", "forcey"):
        scale = max(abs(b[key]), 1e-12)
        assert abs(a[key] - b[key]) <= 1e-8 * scale, (key, a[key], b[key])
    n, rel = s.ctx.iteration_stats()
    assert 1 <= n <= 102 and rel >= 0


def test_iterated_graph_path_refused():
    s = Simulation(FORCED)
    s.init()
    with pytest.raises(Cup2DError):
        s.ctx.advance(1)


def test_iterated_checkpoint_carries_the_adaptive_state():
    a = Simulation(FISH)
    a.init()
    for comp, name in enumerate(("u", "v")):
        a.ctx.set(name, a.ctx.get(name) + noise_field(2, comp, a.ctx.ny, a.ctx.nx))
    for _ in range(2):
        a.advance(a.calcMaxTimestep())
    blob = a.ctx.checkpoint()
    b = Simulation(FISH)
    b.init()
    b.ctx.restore(blob)
    for s in (a, b):
        for _ in range(2):
            s.advance(s.calcMaxTimestep())
        s.ctx.sync()
    for f in ("u", "v", "pres"):
        assert np.array_equal(a.ctx.get(f), b.ctx.get(f)), f
    assert a.ctx.iteration_stats() == b.ctx.iteration_stats()
