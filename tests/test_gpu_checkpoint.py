"""Checkpoint / restart (cup2d_checkpoint_*): continuing from a restored
checkpoint is bitwise the same as continuing the saved run, in a new
context or in the saved one rewound, from host or device buffers, after
graph steps or operator-by-operator steps; foreign or truncated checkpoints
are refused without changing the context."""
import numpy as np
import pytest

from cubismup_2d_b200 import Cup2DError, Ensemble, Simulation
from cubismup_2d_b200.synthetic import noise_field

pytestmark = pytest.mark.gpu

DISK = ("-bpdx 4 -bpdy 2 -extent 1 -CFL 0.1 -nu 1e-3 -lambda 1e4 -poissonType freespace "
        "-shapes 'disk radius=0.1 xpos=0.3 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'")
FISH = ("-bpdx 8 -bpdy 4 -extent 1 -CFL 0.1 -nu 1e-4 -poissonType freespace "
        "-shapes 'stefanfish L=0.18 T=1 xpos=0.4 ypos=0.25'")
TWO_DISKS = ("-bpdx 8 -bpdy 4 -extent 1 -CFL 0.1 -nu 1e-3 -poissonType freespace "
             "-shapes 'disk radius=0.06 xpos=0.4375 ypos=0.25 xvel=-0.3 bForced=1, "
             "disk radius=0.06 xpos=0.5625 ypos=0.26 xvel=0.3'")
TANDEM = ("-bpdx 16 -bpdy 8 -extent 1 -CFL 0.1 -nu 1e-4 -poissonType periodic "
          "-shapes 'stefanfish L=0.12 T=1 xpos=0.3 ypos=0.25, stefanfish L=0.12 T=1 xpos=0.45 ypos=0.25 phi=0.5'")


def _sim(args, seed=1):
    s = Simulation(args)
    s.init()
    for comp, f in enumerate(("u", "v")):
        s.ctx.set(f, s.ctx.get(f) + noise_field(seed, comp, s.ctx.ny, s.ctx.nx))
    return s


def _operator_step(s):
    dt = s.calcMaxTimestep()
    for op in s.pipeline:
        op(dt)
    s.ctx.end_step()
    return s.ctx.shape(0)


def _continue(s):
    _operator_step(s)
    _operator_step(s)
    s.ctx.advance(2)
    _operator_step(s)
    s.ctx.sync()


def _state(s):
    st = {f: s.ctx.get(f) for f in ("u", "v", "pres", "chi", "udef_x", "udef_y")}
    st["shapes"] = [s.ctx.shape(k) for k in range(s.ctx.nshapes)]
    st["scalars"] = s.ctx.scalars()
    return st


def _assert_same(a, b, label):
    for k in a:
        if isinstance(a[k], np.ndarray):
            assert np.array_equal(a[k], b[k]), (label, k)
        else:
            assert a[k] == b[k], (label, k)


@pytest.mark.parametrize("args", [DISK, FISH, TWO_DISKS, TANDEM], ids=["disk", "fish", "two_disks", "tandem"])
@pytest.mark.parametrize("last", ["graph", "operators"])
def test_restart_continues_bitwise(args, last):
    a = _sim(args)
    a.ctx.advance(2)
    _operator_step(a)
    if last == "graph":
        a.ctx.advance(1)
    else:
        _operator_step(a)
    blob = a.ctx.checkpoint()
    assert blob.nbytes == a.ctx.checkpoint_size()
    b = Simulation(args)
    b.init()
    b.ctx.restore(blob)
    _assert_same(_state(a), _state(b), "restored")
    _continue(a)
    _continue(b)
    ref = _state(a)
    _assert_same(ref, _state(b), "new context")
    # the saved context rewound to its checkpoint
    a.ctx.restore(blob)
    _continue(a)
    _assert_same(ref, _state(a), "rewound")


def test_restart_from_device_buffer_and_in_ensemble():
    torch = pytest.importorskip("torch")
    a = _sim(FISH)
    a.ctx.advance(3)
    dev = torch.empty(a.ctx.checkpoint_size(), dtype=torch.uint8, device="cuda")
    a.ctx.checkpoint(dev)
    host = a.ctx.checkpoint()
    assert np.array_equal(dev.cpu().numpy(), host)
    b = _sim(FISH, seed=9)
    c = _sim(DISK)
    ens = Ensemble([b, c])
    ens.advance(1)
    b.ctx.restore(dev)                         # a member rewound to another run's state
    ens.advance(3)
    ens.sync()
    a.ctx.advance(3)
    a.ctx.sync()
    _assert_same(_state(a), _state(b), "ensemble member")


def test_foreign_or_truncated_checkpoints_are_refused():
    a = _sim(DISK)
    a.ctx.advance(2)
    before = _state(a)
    fish = _sim(FISH)
    with pytest.raises(Cup2DError):
        a.ctx.restore(fish.ctx.checkpoint())
    other = _sim(DISK.replace("radius=0.1", "radius=0.09"))
    with pytest.raises(Cup2DError):
        a.ctx.restore(other.ctx.checkpoint())
    blob = a.ctx.checkpoint()
    with pytest.raises(Cup2DError):
        a.ctx.restore(blob[: blob.nbytes - 8])
    with pytest.raises(Cup2DError):
        a.ctx.restore(np.zeros(blob.nbytes, dtype=np.uint8))
    # a damaged payload (one byte of the last section, a field, flipped):
    # refused by the checksum, in host memory and in device memory
    bad = blob.copy()
    bad[-5] ^= 0x10
    with pytest.raises(Cup2DError) as e:
        a.ctx.restore(bad)
    assert "checksum" in str(e.value)
    import torch
    dbad = torch.from_numpy(bad).cuda()
    with pytest.raises(Cup2DError):
        a.ctx.restore(dbad)
    _assert_same(before, _state(a), "refused")
    a.ctx.restore(torch.from_numpy(blob).cuda())      # the intact blob, from device memory
    _assert_same(before, _state(a), "restored")
