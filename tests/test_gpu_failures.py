"""Failure detection without a GPU fault.

The reference aborts on a non-finite field (Checker, Helpers.cpp:178-288)
and exits when a body leaves the domain (PutObjectsOnGrid.cpp:214-218); its
obstacle blocks are allocated per step, so it has no capacity limit.  Here
the kernels raise status flags on the device, cup2d_sync reports each flag
once as CUP2D_ENAN / CUP2D_EDOMAIN / CUP2D_ECAPACITY, and the context stays
usable.  Every failure is made on the host: a NaN written into the velocity,
a body moved out of the domain through its state, and a tile capacity capped
by the fault-injection variable CUP2D_FAULT_TILE_CAPACITY.  None of these
makes a kernel read or write out of bounds (an empty or clipped tile range,
a capped tile list)."""
import numpy as np
import pytest

from cubismup_2d_b200 import Cup2DError, Simulation, abi

pytestmark = pytest.mark.gpu

DISK = ("-bpdx 4 -bpdy 2 -extent 1 -CFL 0.1 -nu 1e-3 -lambda 1e4 -poissonType freespace "
        "-muteAll 1 -shapes 'disk radius=0.1 xpos=0.3 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'")


def _expect(code, fn):
    with pytest.raises(Cup2DError) as e:
        fn()
    assert e.value.code == code, str(e.value)


def _steps(sim, n):
    for _ in range(n):
        sim.advance(sim.calcMaxTimestep())


def test_nan_in_the_velocity_is_reported_and_the_context_recovers():
    s = Simulation(DISK)
    s.init()
    _steps(s, 2)
    s.ctx.sync()
    good = s.ctx.get("u")
    bad = good.copy()
    bad[17, 33] = np.nan
    s.ctx.set("u", bad)
    s.calcMaxTimestep()                     # findMaxU scans every cell
    _expect(abi.ENAN, s.ctx.sync)
    s.ctx.sync()                            # reported once
    s.ctx.set("u", good)                    # the caller repairs the state
    _steps(s, 3)
    s.ctx.sync()
    assert np.all(np.isfinite(s.ctx.get("u")))
    # and the graph path detects it too
    s.ctx.set("u", bad)
    s.ctx.advance(1)
    _expect(abi.ENAN, s.ctx.sync)


def test_body_out_of_the_domain_is_reported_and_the_context_recovers():
    s = Simulation(DISK)
    s.init()
    _steps(s, 2)
    saved = s.ctx.shape(0)
    out = dict(saved)
    out["com_x"] = -0.1                     # the forced, fixed disk stays there
    out["center_x"] = -0.1
    s.ctx.set_shape(0, out)
    _steps(s, 1)
    _expect(abi.EDOMAIN, s.ctx.sync)
    s.ctx.sync()
    s.ctx.set_shape(0, saved)
    _steps(s, 2)
    s.ctx.sync()
    assert abs(s.ctx.shape(0)["center_x"] - saved["center_x"]) < 1e-12


def test_tile_capacity_overflow_is_reported(monkeypatch):
    # the disk (R = 0.1 at h = 1/128) touches 4 blocks; capacity 2 is too small
    monkeypatch.setenv("CUP2D_FAULT_TILE_CAPACITY", "2")
    s = Simulation(DISK)
    s.init()
    _expect(abi.ECAPACITY, s.ctx.sync)
    _steps(s, 1)
    _expect(abi.ECAPACITY, s.ctx.sync)
    # the device state stays consistent: fields read back, no CUDA error
    assert np.all(np.isfinite(s.ctx.get("chi")))
    monkeypatch.delenv("CUP2D_FAULT_TILE_CAPACITY")
    t = Simulation(DISK)
    t.init()
    _steps(t, 1)
    t.ctx.sync()


def test_bounded_tile_wait_runs_out_and_is_reported(monkeypatch):
    """advDiff's tile barrier made to expect more bytes than its TMA loads
    bring (CUP2D_FAULT_TMA_WAIT): the loads all land, the barrier's phase
    never completes, every CTA's wait gives up after its one-second limit
    and the step reports CUP2D_ETIMEOUT; the CUDA context stays usable."""
    monkeypatch.setenv("CUP2D_FAULT_TMA_WAIT", "1")
    s = Simulation(DISK)                    # 8 blocks: one wave of CTAs
    s.init()
    s.ctx.adv_diff(1e-3)
    _expect(abi.ETIMEOUT, s.ctx.sync)
    assert np.all(np.isfinite(s.ctx.get("chi")))
    monkeypatch.delenv("CUP2D_FAULT_TMA_WAIT")
    t = Simulation(DISK)
    t.init()
    _steps(t, 2)
    t.ctx.sync()
