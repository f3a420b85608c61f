"""The discrete adjoint (cup2d_adjoint_run; no counterpart in the reference):
the objective against the plain forward steps, the gradient with respect to
the initial velocity against central finite differences of the FP64 forward
along localized directions (in the wake, at the body, at the domain edge
where the fades and the outflow correction act), independence of the
checkpoint interval, the final state, and the configurations it refuses."""
import numpy as np
import pytest

from cubismup_2d_b200 import Cup2DError, Simulation
from cubismup_2d_b200.abi import ENOTSUP

pytestmark = pytest.mark.gpu

BASE = "-extent 1 -CFL 0.1 -nu 1e-3 -lambda 1e4 -muteAll 1 "
FORCED = (BASE + "-bpdx 8 -bpdy 4 -poissonType freespace "
          "-shapes 'disk radius=0.06 xpos=0.3 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'")
BOX = (0.36, 0.62, 0.14, 0.36)
NSTEPS = 16


def _developed(args=FORCED, warm=40):
    s = Simulation(args)
    s.init()
    for _ in range(warm):
        s.advance(s.calcMaxTimestep())
    s.ctx.sync()
    return s


def _bump(s, cx, cy, sig, au, av):
    n = s.ctx
    x = (np.arange(n.nx) + 0.5) * n.h
    y = (np.arange(n.ny) + 0.5) * n.h
    X, Y = np.meshgrid(x, y)
    g = np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / sig ** 2)
    return au * g, av * g


def _objective(s, dts):
    """J of the plain operator path: (1/N) sum_n (h^2/2) sum_box |u^n|^2."""
    n = s.ctx
    i0, i1 = int(np.floor(BOX[0] / n.h)), int(np.ceil(BOX[1] / n.h))
    j0, j1 = int(np.floor(BOX[2] / n.h)), int(np.ceil(BOX[3] / n.h))
    J = 0.0
    for dt in dts:
        s.advance(dt)
        u, v = n.get("u")[j0:j1, i0:i1], n.get("v")[j0:j1, i0:i1]
        J += 0.5 * n.h ** 2 * float(np.sum(u * u + v * v))
    return J / len(dts)


def test_objective_and_final_state_match_plain_steps():
    s = _developed()
    blob = s.ctx.checkpoint()
    J, gu, gv, dts, ms = s.ctx.adjoint(NSTEPS, BOX, every=5)
    assert np.all(dts > 0) and ms[0] > 0 and ms[1] > 0
    assert np.all(np.isfinite(gu)) and np.all(np.isfinite(gv)) and np.any(gu != 0)
    ua, va = s.ctx.get("u"), s.ctx.get("v")
    s.ctx.restore(blob)
    Jp = _objective(s, dts)
    assert abs(J - Jp) <= 1e-13 * abs(Jp), (J, Jp)
    # the context ends in the forward's final state
    assert np.array_equal(ua, s.ctx.get("u")) and np.array_equal(va, s.ctx.get("v"))


@pytest.mark.parametrize("where", ["wake", "body", "edge", "inflow"])
def test_gradient_matches_finite_differences(where):
    s = _developed()
    blob = s.ctx.checkpoint()
    J, gu, gv, dts, _ = s.ctx.adjoint(NSTEPS, BOX, every=5)
    s.ctx.restore(blob)
    u0, v0 = s.ctx.get("u"), s.ctx.get("v")
    cx, cy, sig = {"wake": (0.45, 0.27, 0.04), "body": (0.3, 0.31, 0.03),
                   "edge": (0.97, 0.22, 0.05), "inflow": (0.05, 0.3, 0.05)}[where]
    du, dv = _bump(s, cx, cy, sig, 0.7, -0.4)
    ad = float(np.sum(gu * du) + np.sum(gv * dv))
    # central differences at 1e-6: the fade's and the obstacle terms' sign
    # tests make the forward piecewise smooth, and a larger step crosses
    # their switches (1e-4 does, at the edge and the inflow)
    eps = 1e-6
    Js = []
    for sgn in (1, -1):
        s.ctx.restore(blob)
        s.ctx.set("u", u0 + sgn * eps * du)
        s.ctx.set("v", v0 + sgn * eps * dv)
        Js.append(s.ctx.adjoint(NSTEPS, BOX, dt=dts, gradient=False)[0])
    fd = (Js[0] - Js[1]) / (2 * eps)
    assert abs(fd) > 1e-8 * abs(J), (where, fd, J)
    assert abs(ad - fd) <= 2e-6 * abs(fd), (where, ad, fd)


def test_checkpoint_interval_does_not_change_the_gradient():
    s = _developed()
    blob = s.ctx.checkpoint()
    ref = s.ctx.adjoint(NSTEPS, BOX, every=NSTEPS)
    scale = max(np.max(np.abs(ref[1])), np.max(np.abs(ref[2])))
    for every in (1, 3):
        s.ctx.restore(blob)
        J, gu, gv, dts, _ = s.ctx.adjoint(NSTEPS, BOX, every=every, dt=ref[3])
        assert abs(J - ref[0]) <= 1e-13 * abs(ref[0])
        assert np.max(np.abs(gu - ref[1])) <= 1e-12 * scale
        assert np.max(np.abs(gv - ref[2])) <= 1e-12 * scale


@pytest.mark.parametrize("args", [
    FORCED.replace("freespace", "cosine"),
    BASE + "-bpdx 8 -bpdy 4 -poissonType freespace -shapes 'disk radius=0.06 xpos=0.3 ypos=0.25 xvel=0.2'",
    BASE + "-bpdx 8 -bpdy 4 -poissonType freespace -shapes 'stefanfish L=0.18 T=1 xpos=0.4 ypos=0.25'",
    FORCED + " -iterativePenalization 1",
], ids=["cosine_solver", "free_disk", "swimmer", "iterated"])
def test_uncovered_configurations_refused(args):
    s = Simulation(args)
    s.init()
    with pytest.raises(Cup2DError) as e:
        s.ctx.adjoint(4, BOX)
    assert e.value.code == ENOTSUP
