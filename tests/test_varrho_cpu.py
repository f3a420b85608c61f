"""The variable-density branch on the CPU: the reference's own advDiffGrav
and PressureVarRho_approx run by the oracle driver (a heavy disk sinks, a
light one rises, gravity is honoured), and the host-side selection of the
pipeline (Simulation.cpp:183-220, SimulationData.cpp:122-130)."""
import numpy as np
import pytest

from cubismup_2d_b200.abi import parse_args, variable_density

ARGS = ("-bpdx 2 -bpdy 2 -extent 1 -CFL 0.1 -nu 1e-3 -muteAll 1 -iterativePenalization 1 "
        "-shapes 'disk radius=0.12 xpos=0.5 ypos=0.5 rhoS={}'")


@pytest.mark.parametrize("rho, sign", [(1.5, -1), (0.7, 1)])
def test_reference_body_moves_with_buoyancy(ref, rho, sign):
    r = ref.RefSim(ARGS.format(rho))
    assert r.variable_density()
    for _ in range(3):
        r.step()
        assert r.iterations() >= 1
    assert np.sign(r.shape(0)["v"]) == sign
    ir = r.get("invRho")
    assert np.isclose(ir.min(), min(1.0, 1 / rho)) and np.isclose(ir.max(), max(1.0, 1 / rho))


def test_reference_gravity_sets_the_direction(ref):
    r = ref.RefSim(ARGS.format(1.5))
    r.set_gravity(-9.8, 0.0)
    for _ in range(3):
        r.step()
    s = r.shape(0)
    assert s["u"] < 0 and abs(s["v"]) < abs(s["u"])


def test_pipeline_selection_and_gravity_parse():
    cfg, shapes = parse_args(ARGS.format(1.5))
    assert variable_density(shapes)
    assert tuple(cfg.gravity) == (0.0, -9.8)
    cfg, shapes = parse_args(ARGS.format(1.0) + " -gravity '1 2'")
    assert not variable_density(shapes)
    assert tuple(cfg.gravity) == (1.0, 2.0)


def test_reference_implicit_penalization_composes(ref):
    """The harness's PressureSingle without EXPL_INTEGRATE_MOM runs and
    differs from the shipped explicit forms."""
    base = ("-bpdx 2 -bpdy 2 -extent 1 -CFL 0.1 -nu 1e-3 -lambda 1e3 -muteAll 1 "
            "-shapes 'disk radius=0.12 xpos=0.5 ypos=0.5 bForced=1 xvel=0.1'")
    a, b = ref.RefSim(base + " -implicitPenalization 1"), ref.RefSim(base)
    for _ in range(3):
        a.step()
        b.step()
    assert np.all(np.isfinite(a.get("u")))
    assert not np.array_equal(a.get("u"), b.get("u"))


def test_reference_udef_clearing_depends_on_block_order(ref):
    """PressureVarRho_approx with a swimmer: the single-thread run is
    reproducible (the order the CUDA path follows)."""
    args = ("-bpdx 4 -bpdy 2 -extent 1 -CFL 0.1 -nu 1e-4 -muteAll 1 -iterativePenalization 1 "
            "-shapes 'stefanfish L=0.3 T=1 xpos=0.3 ypos=0.25, disk radius=0.05 xpos=0.75 ypos=0.3 rhoS=1.5'")
    old = ref.set_threads(1)
    try:
        runs = []
        for _ in range(2):
            r = ref.RefSim(args)
            r.step()
            runs.append(r.get("u"))
        assert np.array_equal(runs[0], runs[1])
    finally:
        ref.set_threads(old)
