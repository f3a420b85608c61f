"""The lambda-implicit penalization (PressureSingle as compiled without
EXPL_INTEGRATE_MOM, PressureSingle.cpp:20: momenta with F = h^2 rho X/(1+X),
X = chi lambda dt, and alpha = 1/(1 + lambda dt chi), the forms of
UpdateObjects.cpp:128-210) against the reference's own code composed the
same way (oracle harness option -implicitPenalization 1), step by step,
through the operator path and the graph path."""
import numpy as np
import pytest

from cubismup_2d_b200 import Simulation
from cubismup_2d_b200.synthetic import noise_field

pytestmark = pytest.mark.gpu

IMPL = "-extent 1 -CFL 0.1 -poissonType freespace -muteAll 1 -implicitPenalization 1 "
FORCED = ("-bpdx 4 -bpdy 2 -nu 1e-3 -lambda 1e4 " + IMPL +
          "-shapes 'disk radius=0.1 xpos=0.3 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'")
FREE = ("-bpdx 4 -bpdy 2 -nu 1e-3 -lambda 1e3 " + IMPL +
        "-shapes 'disk radius=0.08 xpos=0.4 ypos=0.22 xvel=0.1 yvel=0.05'")
FISH = ("-bpdx 8 -bpdy 4 -nu 1e-4 -dlm 1 " + IMPL +
        "-shapes 'stefanfish L=0.18 T=1 xpos=0.4 ypos=0.25'")


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _pair(ref, args, seed=3):
    r = ref.RefSim(args)
    s = Simulation(args)
    s.init()
    for comp, name in enumerate(("u", "v")):
        a = r.get(name) + noise_field(seed, comp, r.ny, r.nx)
        r.set(name, a)
        s.ctx.set(name, a)
    return r, s


@pytest.mark.parametrize("args", [FORCED, FREE, FISH], ids=["forced_disk", "free_disk", "fish_dlm"])
def test_steps_match_reference(ref, args):
    r, s = _pair(ref, args)
    for _ in range(4):
        r.step()
        s.advance(s.calcMaxTimestep())
    s.ctx.sync()
    errs = {f: _rel(s.ctx.get(f), r.get(f)) for f in ("u", "v", "pres", "chi")}
    assert all(e <= 1e-9 for e in errs.values()), errs
    a, b = s.ctx.shape(0), r.shape(0)
    for key in ("u", "v", "omega", "center_x", "center_y", "penalM", "penalJ", "fluidMomX",
                "fluidMomY", "forcex", "forcey"):
        scale = max(abs(b[key]), 1e-12)
        assert abs(a[key] - b[key]) <= 1e-8 * scale, (key, a[key], b[key])


def test_graph_steps_equal_operator_steps():
    a = Simulation(FORCED)
    b = Simulation(FORCED)
    for s in (a, b):
        s.init()
    for _ in range(3):
        a.advance(a.calcMaxTimestep())
    b.ctx.advance(3)
    for s in (a, b):
        s.ctx.sync()
    for f in ("u", "v", "pres"):
        assert np.array_equal(a.ctx.get(f), b.ctx.get(f)), f


def test_differs_from_the_explicit_forms():
    a = Simulation(FORCED)
    b = Simulation(FORCED.replace("-implicitPenalization 1", ""))
    for s in (a, b):
        s.init()
        s.ctx.advance(2)
        s.ctx.sync()
    assert not np.array_equal(a.ctx.get("u"), b.ctx.get("u"))
