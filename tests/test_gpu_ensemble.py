"""The batched ensemble (cup2d_ensemble_*): members of uneven grids and shapes
advanced by one graph end bitwise where their own graph steps leave them,
also when ensemble advances alternate with the members' own graph steps,
operator-by-operator steps and a re-initialisation."""
import numpy as np
import pytest

from cubismup_2d_b200 import Cup2DError, Ensemble, Simulation
from cubismup_2d_b200.abi import Context, parse_args
from cubismup_2d_b200.synthetic import ensemble_configs, noise_field

pytestmark = pytest.mark.gpu

MEMBERS = [
    ("-bpdx 4 -bpdy 2 -extent 1 -CFL 0.1 -nu 1e-3 -lambda 1e4 -poissonType freespace "
     "-shapes 'disk radius=0.1 xpos=0.3 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'"),
    ("-bpdx 8 -bpdy 4 -extent 1 -CFL 0.1 -nu 1e-4 -poissonType freespace "
     "-shapes 'stefanfish L=0.18 T=1 xpos=0.4 ypos=0.25'"),
    ("-bpdx 16 -bpdy 8 -extent 1 -CFL 0.1 -nu 2e-4 -lambda 1e4 -poissonType freespace "
     "-shapes 'disk radius=0.04 xpos=0.2 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'"),
    ("-bpdx 8 -bpdy 4 -extent 1 -CFL 0.1 -nu 1e-4 -poissonType periodic "
     "-shapes 'carlingfish L=0.18 T=1 xpos=0.4 ypos=0.25 angle=10'"),
    # 768x384: free space padded to 2048x1024
    ("-bpdx 24 -bpdy 12 -extent 1 -CFL 0.1 -nu 1e-4 -lambda 1e4 -poissonType freespace "
     "-shapes 'disk radius=0.03 xpos=0.2 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'"),
]


def _member(argline, seed):
    s = Simulation(argline)
    s.init()
    for comp, f in enumerate(("u", "v")):
        s.ctx.set(f, s.ctx.get(f) + noise_field(seed, comp, s.ctx.ny, s.ctx.nx))
    return s


def _operator_step(s):
    dt = s.calcMaxTimestep()
    for op in s.pipeline:
        op(dt)
    s.ctx.end_step()


def _same(a, b, label):
    a.ctx.sync(); b.ctx.sync()
    for f in ("u", "v", "pres", "chi"):
        assert np.array_equal(a.ctx.get(f), b.ctx.get(f)), (label, f)
    for k in range(a.ctx.nshapes):
        assert a.ctx.shape(k) == b.ctx.shape(k), (label, k)
    assert a.ctx.scalars() == b.ctx.scalars(), label


def test_ensemble_matches_members():
    alone = [_member(x, i) for i, x in enumerate(MEMBERS)]
    joint = [_member(x, i) for i, x in enumerate(MEMBERS)]
    ens = Ensemble(joint)
    ens.advance(3)
    ens.sync()
    for s in alone:
        s.ctx.advance(3)
    for i, (a, b) in enumerate(zip(alone, joint)):
        _same(a, b, f"member {i} after 3 ensemble steps")
    # members on their own in between: graph steps, then operator steps
    for s in alone + joint:
        s.ctx.advance(1)
        _operator_step(s)
    ens.advance(2)
    for s in alone:
        s.ctx.advance(2)
    for i, (a, b) in enumerate(zip(alone, joint)):
        _same(a, b, f"member {i} after mixed steps")
    # a member re-initialised (same context): the ensemble captures its step again
    alone[1].ctx.init(); joint[1].ctx.init()
    ens.advance(2)
    for s in alone:
        s.ctx.advance(2)
    for i, (a, b) in enumerate(zip(alone, joint)):
        _same(a, b, f"member {i} after a re-initialisation")


def test_ensemble_of_drawn_members_runs():
    """Eight members drawn as in the ensemble benchmark: the ensemble's steps
    equal each member's own."""
    cfgs = ensemble_configs(n=8, seed=3)
    alone = [_member(x, i) for i, x in enumerate(cfgs)]
    joint = [_member(x, i) for i, x in enumerate(cfgs)]
    ens = Ensemble(joint)
    ms = ens.advance_timed(4)
    assert ms > 0
    ens.sync()
    for s in alone:
        s.ctx.advance(4)
    for i, (a, b) in enumerate(zip(alone, joint)):
        _same(a, b, f"drawn member {i}")


def test_ensemble_rejects_bad_members():
    s = _member(MEMBERS[0], 0)
    with pytest.raises(Cup2DError):
        Ensemble([s, s])                       # the same context twice
    with pytest.raises(Cup2DError):
        Ensemble([])
    cfg, shapes = parse_args(MEMBERS[0])
    raw = Simulation(MEMBERS[0])
    raw.ctx = Context(cfg, shapes)             # created, not initialised
    with pytest.raises(Cup2DError):
        Ensemble([s, raw])
    ens = Ensemble([s])
    s.init()                                   # a new context replaces the member's
    with pytest.raises(Cup2DError):
        ens.advance(1)


TWO_DISKS = ("-bpdx 8 -bpdy 4 -extent 1 -CFL 0.1 -nu 1e-3 -poissonType freespace "
             "-shapes 'disk radius=0.06 xpos=0.4375 ypos=0.25 xvel=-0.3 bForced=1, "
             "disk radius=0.06 xpos=0.5625 ypos=0.26 xvel=0.3'")


def test_ensemble_shape_states_read_back():
    """One batched read-back of every member's shape states equals each
    member's own read-back: after ensemble steps (from mapped memory), and
    after a member's own graph or operator step (through the member)."""
    from cubismup_2d_b200.abi import SHAPE_STATE_FIELDS
    members = [_member(x, i) for i, x in enumerate(ensemble_configs(n=4, seed=4) + [TWO_DISKS])]
    ens = Ensemble(members)

    def own():
        return np.array([[s.ctx.shape(k)[f] for f in SHAPE_STATE_FIELDS]
                         for s in members for k in range(s.ctx.nshapes)])

    ens.advance(2)
    # the size query: no buffer, capacity 0
    import ctypes
    cnt = ctypes.c_int(-1)
    assert ens.L.cup2d_ensemble_get_shapes(ens.h_, None, 0, ctypes.byref(cnt)) == 0 and cnt.value == 6
    a = ens.shape_states()
    assert a.shape == (6, len(SHAPE_STATE_FIELDS))
    assert np.array_equal(a, own())
    members[1].ctx.advance(1)
    _operator_step(members[4])
    assert np.array_equal(ens.shape_states(), own())
    ens.advance(1)
    assert np.array_equal(ens.shape_states(), own())
    assert ens.shapes()[4][1]["forcex"] == members[4].ctx.shape(1)["forcex"]
