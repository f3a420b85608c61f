"""RL actuation of StefanFish against the reference's own StefanFish::act,
getLearnTPeriod and state (StefanFish.cpp:373-577, the 16-value state with
the head sensors StefanFish.h:12 compiles in), and the leader-follower
driver (main_RL_leadFollow.cpp:79-177) against the same loop written over
the reference.  Kinematic state entries are compared to 1e-9 of their
scale; the shear sensors, velocity differences over one cell divided by h,
to 1e-6."""
import numpy as np
import pytest

from cubismup_2d_b200 import Simulation
from cubismup_2d_b200.rl import LeadFollow, is_terminal
from cubismup_2d_b200.synthetic import noise_field

pytestmark = pytest.mark.gpu

PAIR = ("-bpdx 8 -bpdy 4 -extent 1 -CFL 0.1 -nu 1e-4 -poissonType freespace -muteAll 1 "
        "-shapes 'stefanfish L=0.18 T=1 xpos=0.3 ypos=0.25, stefanfish L=0.18 T=1 xpos=0.55 ypos=0.25'")


def _state_close(a, b, label):
    kin_scale = np.maximum(np.abs(b[:10]), 1e-3)
    assert np.all(np.abs(a[:10] - b[:10]) <= 1e-9 * kin_scale), (label, a[:10], b[:10])
    sens_scale = max(np.max(np.abs(b[10:])), 1e-3)
    assert np.all(np.abs(a[10:] - b[10:]) <= 1e-6 * sens_scale), (label, a[10:], b[10:])


def test_actions_and_state_match_reference(ref):
    r = ref.RefSim(PAIR)
    s = Simulation(PAIR)
    s.init()
    for comp, f in enumerate(("u", "v")):
        a = r.get(f) + noise_field(8, comp, r.ny, r.nx)
        r.set(f, a)
        s.ctx.set(f, a)
    _state_close(s.ctx.fish_state(1, 0), r.fish_state(1, 0), "initial state")
    t = 0.0
    for action, nsteps in (([0.5, 0.1], 25), ([-0.3], 15), ([0.2, -0.2], 20)):
        r.fish_act(1, t, action)
        s.ctx.fish_act(1, t, action)
        assert s.ctx.fish_period(1) == r.fish_period(1)
        for _ in range(nsteps):
            dt_r = r.step()
            dt_s = s.calcMaxTimestep()
            s.advance(dt_s)
            assert abs(dt_s - dt_r) <= 1e-12 * dt_r
            t += dt_r
        _state_close(s.ctx.fish_state(1, 0), r.fish_state(1, 0), f"after {action}")
        for f in ("u", "v", "pres", "chi"):
            a, b = s.ctx.get(f), r.get(f)
            assert np.max(np.abs(a - b)) <= 1e-8 * np.max(np.abs(b)), (action, f)
    # graph steps after an action form the same midlines as operator steps
    g = Simulation(PAIR)
    g.init()
    o = Simulation(PAIR)
    o.init()
    for sim in (g, o):
        sim.ctx.fish_act(1, 0.0, [0.7, 0.15])
    g.ctx.advance(6)
    for _ in range(6):
        o.advance(o.calcMaxTimestep())
    g.ctx.sync()
    for f in ("u", "v", "chi"):
        assert np.array_equal(g.ctx.get(f), o.ctx.get(f)), f


def test_lead_follow_driver_matches_the_reference_loop(ref):
    """Two actions of the driver (fixed initial condition: the evaluation
    branch of resetIC) against the same loop over the reference."""
    env = LeadFollow(PAIR, training=False)
    st = env.reset()
    r = ref.RefSim(PAIR)
    L = 0.18
    p = r.shape(0)
    C = (p["center_x"] + 1.25 * L, p["center_y"])
    r.set_shape_pose(0, (p["com_x"], p["center_y"]), (p["center_x"], p["center_y"]), p["orientation"])
    a = r.shape(1)
    r.set_shape_pose(1, C, (a["center_x"], a["center_y"]), 0.0)
    _state_close(st, r.fish_state(1, 0), "reset")
    t = tn = 0.0
    for action in ([0.4, 0.05], [-0.2, 0.0]):
        state, reward, done, info = env.step(action)
        r.fish_act(1, tn, action)
        tn = tn + r.fish_period(1) / 2
        while t < tn:
            t += r.step()
            if is_terminal(r.shape(1), r.shape(0), L):
                break
        _state_close(state, r.fish_state(1, 0), f"after {action}")
        rb = r.shape(1)["EffPDefBnd"]
        assert abs(reward - rb) <= 1e-8 * max(abs(rb), 1.0), (reward, rb)
        assert not done and info["reason"] == "running"


PID = ("-bpdx 8 -bpdy 4 -extent 1 -CFL 0.1 -nu 1e-4 -poissonType freespace -muteAll 1 "
       "-shapes 'stefanfish L=0.18 T=1 xpos=0.4 ypos=0.25 angle=4 {}=1'")


@pytest.mark.parametrize("flag", ["pid", "pidpos"])
def test_pid_controllers_match_reference(ref, flag):
    """StefanFish::create's controllers (StefanFish.cpp:264-364): -pid
    corrects the heading, -pidpos the position (also through the tail
    period).  30 operator steps against the reference, then graph steps
    bitwise equal to operator steps (the midline is formed inside the
    step, after the controller)."""
    args = PID.format(flag)
    r = ref.RefSim(args)
    s = Simulation(args)
    s.init()
    for comp, f in enumerate(("u", "v")):
        a = r.get(f) + noise_field(12, comp, r.ny, r.nx)
        r.set(f, a)
        s.ctx.set(f, a)
    for _ in range(30):
        dt_r = r.step()
        dt_s = s.calcMaxTimestep()
        s.advance(dt_s)
        assert abs(dt_s - dt_r) <= 1e-12 * dt_r
    a, b = s.ctx.shape(0), r.shape(0)
    for key in ("com_x", "com_y", "orientation"):
        assert abs(a[key] - b[key]) <= 1e-10, (key, a[key], b[key])
    for f in ("u", "v", "pres", "chi"):
        x, y = s.ctx.get(f), r.get(f)
        assert np.max(np.abs(x - y)) <= 1e-8 * np.max(np.abs(y)), f
    assert s.ctx.fish_period(0) == pytest.approx(r.fish_period(0), rel=1e-12, abs=0)
    _state_close(s.ctx.fish_state(0, 0), r.fish_state(0, 0), flag)
    g = Simulation(args); g.init()
    o = Simulation(args); o.init()
    g.ctx.advance(8)
    for _ in range(8):
        o.advance(o.calcMaxTimestep())
    g.ctx.sync()
    for f in ("u", "v", "chi"):
        assert np.array_equal(g.ctx.get(f), o.ctx.get(f)), f
    assert g.ctx.shape(0) == o.ctx.shape(0)
