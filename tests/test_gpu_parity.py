"""Parity of the CUDA pipeline with the reference's own operators.

Both sides start from identical state (same arguments, same seeded noise);
the oracle is the reference compiled from its sources (oracle/_ref).  Stage
tests feed both the same inputs and compare one Operator::operator()(dt);
step tests compare whole Simulation::advance passes.

Tolerances (fp64):
  - stencil stages with identical inputs: <= 4 ulp-scale (1e-15 relative);
  - anything downstream of a reduction or of the FFT: relative 1e-10 after a
    stage, 1e-8 after tens of steps (the FFT and the reduction orders differ
    from the reference's, so results agree to rounding, not bitwise);
  - force sums: relative 1e-8 of the largest component.
"""
import numpy as np
import pytest

from cubismup_2d_b200 import Simulation
from cubismup_2d_b200.synthetic import noise_field

pytestmark = pytest.mark.gpu

DISK = ("-bpdx 4 -bpdy 2 -extent 1 -CFL 0.1 -nu 1e-3 -lambda 1e4 -poissonType freespace "
        "-muteAll 1 -shapes 'disk radius=0.1 xpos=0.3 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'")
DISK_FREE = ("-bpdx 4 -bpdy 2 -extent 1 -CFL 0.1 -nu 1e-3 -poissonType freespace "
             "-muteAll 1 -shapes 'disk radius=0.08 xpos=0.4 ypos=0.22 xvel=0.1 yvel=0.05'")
FISH = ("-bpdx 8 -bpdy 4 -extent 1 -CFL 0.1 -nu 1e-4 -poissonType freespace "
        "-muteAll 1 -shapes 'stefanfish L=0.18 T=1 xpos=0.4 ypos=0.25'")
CARLING = ("-bpdx 8 -bpdy 4 -extent 1 -CFL 0.1 -nu 1e-4 -poissonType freespace "
           "-muteAll 1 -shapes 'carlingfish L=0.18 T=1 xpos=0.4 ypos=0.25 angle=10'")
# a forced disk in contact with a free one (collisions, several shapes)
TWO_DISKS = ("-bpdx 8 -bpdy 4 -extent 1 -CFL 0.1 -nu 1e-3 -poissonType freespace -muteAll 1 "
             "-shapes 'disk radius=0.06 xpos=0.4375 ypos=0.25 xvel=-0.3 bForced=1, "
             "disk radius=0.06 xpos=0.5625 ypos=0.26 xvel=0.3'")


def rel_err(a, b):
    scale = max(np.max(np.abs(b)), 1e-300)
    return float(np.max(np.abs(a - b)) / scale)


def make_pair(ref, args, noise_seed=None):
    r = ref.RefSim(args)
    s = Simulation(args)
    s.init()
    if noise_seed is not None:
        for comp, name in enumerate(("u", "v")):
            n = noise_field(noise_seed, comp, r.ny, r.nx)
            a = r.get(name) + n
            r.set(name, a)
            s.ctx.set(name, a)
    return r, s


def compare_fields(r, s, names, tol, label=""):
    errs = {}
    for n in names:
        errs[n] = rel_err(s.ctx.get(n), r.get(n))
    bad = {k: v for k, v in errs.items() if not v <= tol}
    assert not bad, f"{label} field mismatch (tol {tol}): {errs}"
    return errs


def compare_shape(r, s, keys, tol, k=0, label=""):
    a, b = s.ctx.shape(k), r.shape(k)
    errs = {}
    for key in keys:
        scale = max(abs(b[key]), 1e-30)
        errs[key] = abs(a[key] - b[key]) / scale
    bad = {k2: (a[k2], b[k2]) for k2, v in errs.items() if not v <= tol}
    assert not bad, f"{label} shape mismatch (tol {tol}): {bad}"


# Shape::computeForces (Shape.cpp:252-278) and the rigid-body state, grouped
# by the scale each is compared against
FORCE_KEYS = ["forcex", "forcey", "forcex_P", "forcey_P", "forcex_V", "forcey_V", "drag", "thrust"]
TORQUE_KEYS = ["torque", "torque_P", "torque_V"]
POWER_KEYS = ["Pout", "PoutBnd", "defPower", "defPowerBnd", "Pthrust", "Pdrag"]


def compare_shape_all(a, b, tol, label=""):
    """Every sum of cup2d_shape_state against the reference's: forces,
    torques and powers relative to the largest of their group, the
    perimeter and the circulation relative to themselves, the efficiencies
    (ratios of powers, Shape.cpp:274-277) absolutely."""
    errs = {}

    def group(keys):
        scale = max(max(abs(b[k]) for k in keys), 1e-30)
        for k in keys:
            errs[k] = abs(a[k] - b[k]) / scale
    group(FORCE_KEYS)
    group(TORQUE_KEYS)
    group(POWER_KEYS)
    for k in ("perimeter", "circulation"):
        errs[k] = abs(a[k] - b[k]) / max(abs(b[k]), 1e-30)
    for k in ("EffPDef", "EffPDefBnd"):
        errs[k] = abs(a[k] - b[k])
    bad = {k: (a[k], b[k], e) for k, e in errs.items() if not e <= tol}
    assert not bad, f"{label} force sums differ (tol {tol}): {bad}"


def test_init_disk(ref):
    r, s = make_pair(ref, DISK)
    assert (s.ctx.nx, s.ctx.ny) == (r.nx, r.ny)
    # Towers chi and the ApplyObjVel velocity come from identical arithmetic
    compare_fields(r, s, ["chi"], 0.0, "init")
    compare_fields(r, s, ["u", "v"], 1e-15, "init")
    compare_shape(r, s, ["center_x", "center_y", "com_x", "com_y", "M", "J", "u", "v"], 1e-12, label="init")


def test_advdiff_stage_bitwise(ref):
    r, s = make_pair(ref, DISK, noise_seed=7)
    dt = 1e-3
    r.run_op("advDiff", dt)
    s.ctx.adv_diff(dt)
    # outflow correction is a boundary reduction: allow its rounding
    compare_fields(r, s, ["u", "v"], 1e-14, "advDiff")


DISK_PERIODIC = DISK.replace("freespace", "periodic")
DISK_COSINE = DISK.replace("-poissonType freespace ", "")      # "" selects FFTW_dirichlet


@pytest.mark.parametrize("args", [DISK, DISK_PERIODIC, DISK_COSINE], ids=["freespace", "periodic", "cosine"])
def test_pressure_stage(ref, args):
    r, s = make_pair(ref, args, noise_seed=11)
    dt = 1e-3
    r.run_op("advDiff", dt); s.ctx.adv_diff(dt)
    r.run_op("PressureSingle", dt); s.ctx.pressure_single(dt)
    compare_fields(r, s, ["tmp"], 1e-12, "rhs")
    compare_fields(r, s, ["pres"], 1e-10, "pressure")
    compare_fields(r, s, ["u", "v"], 1e-10, "velocity")
    compare_shape(r, s, ["penalM", "penalJ", "fluidMomX", "fluidMomY"], 1e-10, label="momenta")


def test_pressure_stage_alone_and_rhs_bitwise(ref):
    """PressureSingle called without advDiff before it forms its divergence
    in k_rhs_div (PressureSingle.cpp:112-128): the stage matches the
    reference's, and in the blocks that neither the obstacle terms nor the
    fade reach (blocks 4-6 x 1-2 of 8 x 4, the disk in blocks 0-2) the RHS is
    (h/2dt)((u_E - u_W) + (v_N - v_S)) bit for bit."""
    args = ("-bpdx 8 -bpdy 4 -extent 1 -CFL 0.1 -nu 1e-3 -lambda 1e4 -poissonType freespace -muteAll 1 "
            "-shapes 'disk radius=0.05 xpos=0.2 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'")
    r, s = make_pair(ref, args, noise_seed=13)
    u, v = s.ctx.get("u"), s.ctx.get("v")
    dt = 1e-3
    r.run_op("PressureSingle", dt); s.ctx.pressure_single(dt)
    compare_fields(r, s, ["tmp"], 1e-12, "rhs")
    compare_fields(r, s, ["pres"], 1e-10, "pressure")
    compare_fields(r, s, ["u", "v"], 1e-10, "velocity")
    fac = 0.5 * s.ctx.h / dt
    b = fac * ((u[1:-1, 2:] - u[1:-1, :-2]) + (v[2:, 1:-1] - v[:-2, 1:-1]))
    rhs = s.ctx.get("tmp")[1:-1, 1:-1]
    rows, cols = slice(32 - 1, 96 - 1), slice(128 - 1, 224 - 1)   # blocks by 1-2, bx 4-6
    assert np.array_equal(rhs[rows, cols], b[rows, cols])


def test_forces_stage(ref):
    r, s = make_pair(ref, DISK, noise_seed=3)
    dt = 1e-3
    for name in ("advDiff", "PressureSingle", "ComputeForces"):
        r.run_op(name, dt)
    s.ctx.adv_diff(dt); s.ctx.pressure_single(dt); s.ctx.compute_forces(dt)
    a, b = s.ctx.shape(), r.shape()
    fscale = max(abs(b["forcex"]), abs(b["forcey"]), 1e-30)
    for key in ("forcex", "forcey", "forcex_P", "forcey_P", "forcex_V", "forcey_V"):
        assert abs(a[key] - b[key]) <= 1e-8 * fscale, (key, a[key], b[key])
    assert abs(a["perimeter"] - b["perimeter"]) <= 1e-12 * b["perimeter"]
    compare_shape_all(a, b, 1e-8, "forces stage")


@pytest.mark.parametrize("args", [FISH, CARLING, TWO_DISKS], ids=["stefanfish", "carlingfish", "two_disks"])
def test_all_force_sums_after_steps(ref, args):
    """All 17 additive sums of ComputeForces and the derived powers and
    efficiencies, for swimming bodies (deformation power, thrust) and for
    two shapes, after four steps of the operator loop."""
    r, s = make_pair(ref, args, noise_seed=13)
    for _ in range(4):
        r.step()
        s.advance(s.calcMaxTimestep())
    for k in range(r.nshapes()):
        compare_shape_all(s.ctx.shape(k), r.shape(k), 1e-7, f"shape {k}")


@pytest.mark.parametrize("args", [FISH, TWO_DISKS], ids=["stefanfish", "two_disks"])
def test_udef_grid_matches_reference(ref, args):
    """SimulationData::uDef as PutObjectsOnGrid leaves it
    (PutObjectsOnGrid.cpp:149-184): after operator steps, after a lone
    PutObjectsOnGrid, and after graph steps (which do not fill the grid:
    it is filled from the obstacle tiles when read)."""
    r, s = make_pair(ref, args, noise_seed=17)
    for _ in range(3):
        r.step()
        s.advance(s.calcMaxTimestep())
    scale = max(np.max(np.abs(r.get("udef_x"))), np.max(np.abs(r.get("udef_y"))), 1e-30)
    for f in ("udef_x", "udef_y"):
        assert np.max(np.abs(s.ctx.get(f) - r.get(f))) <= 1e-9 * scale, f
    dt = r.calc_dt()
    assert abs(s.calcMaxTimestep() - dt) <= 1e-12 * dt
    r.run_op("PutObjectsOnGrid", dt)
    s.ctx.put_objects(dt)
    for f in ("udef_x", "udef_y"):
        assert np.max(np.abs(s.ctx.get(f) - r.get(f))) <= 1e-9 * scale, f
    # graph steps against a context that ran the same steps operator by operator
    a = Simulation(args); a.init()
    b = Simulation(args); b.init()
    for _ in range(3):
        a.advance(a.calcMaxTimestep())
    b.ctx.advance(3)
    b.ctx.sync()
    for f in ("udef_x", "udef_y"):
        assert np.array_equal(a.ctx.get(f), b.ctx.get(f)), f


@pytest.mark.parametrize("args", [DISK, DISK_FREE, DISK_COSINE], ids=["forced_disk", "free_disk", "cosine"])
def test_steps_disk(ref, args):
    r, s = make_pair(ref, args, noise_seed=5)
    for it in range(12):
        dtr = r.step()
        dts = s.calcMaxTimestep()
        assert abs(dts - dtr) <= 1e-12 * dtr, (it, dts, dtr)
        s.advance(dts)
    compare_fields(r, s, ["u", "v", "pres", "chi"], 1e-8, "12 steps")
    compare_shape(r, s, ["com_x", "com_y", "u", "v", "omega", "forcex", "forcey"], 1e-7, label="12 steps")
    st = s.ctx.scalars()
    assert st["step"] == r.step_id and abs(st["time"] - r.time) <= 1e-12 * r.time


# two swimmers in tandem, half a period apart (the benchmark's tandem pair,
# at a resolution the reference's arc-length grid accepts for L = 0.12)
TANDEM = ("-bpdx 16 -bpdy 8 -extent 1 -CFL 0.1 -nu 1e-4 -poissonType freespace -muteAll 1 "
          "-shapes 'stefanfish L=0.12 T=1 xpos=0.3 ypos=0.25, stefanfish L=0.12 T=1 xpos=0.45 ypos=0.25 phi=0.5'")


@pytest.mark.parametrize("args", [FISH, CARLING, TANDEM], ids=["stefanfish", "carlingfish", "tandem"])
def test_fish_init_and_steps(ref, args):
    r, s = make_pair(ref, args, noise_seed=9)
    compare_fields(r, s, ["chi"], 1e-12, "fish init")
    compare_shape(r, s, ["com_x", "com_y", "M", "J", "d_gm_x", "d_gm_y"], 1e-10, label="fish init")
    for it in range(6):
        dtr = r.step()
        dts = s.calcMaxTimestep()
        assert abs(dts - dtr) <= 1e-12 * dtr, (it, dts, dtr)
        s.advance(dts)
    compare_fields(r, s, ["chi"], 1e-9, "fish steps")
    compare_fields(r, s, ["u", "v", "pres"], 1e-8, "fish steps")
    for k in range(args.count("fish ")):
        compare_shape(r, s, ["com_x", "com_y", "u", "v", "omega", "forcex", "forcey"], 1e-7, k=k,
                      label=f"fish steps, shape {k}")


def test_degenerate_fish_midline_is_rejected():
    # L = 0.2 at h = 1/256 gives dSref == 0 (FishLibrary.cpp:21 asserts dSref > 0;
    # a release build of the reference produces NaN): the context refuses it.
    from cubismup_2d_b200 import Cup2DError
    s = Simulation("-bpdx 8 -bpdy 4 -poissonType freespace -shapes 'stefanfish L=0.2 xpos=0.4 ypos=0.25'")
    with pytest.raises(Cup2DError) as e:
        s.init()
    assert "EINVAL" in str(e.value)


@pytest.mark.parametrize("args", [DISK, FISH, TWO_DISKS, TANDEM], ids=["disk", "fish", "two_disks", "tandem"])
def test_graph_replay_matches_eager(args):
    a = Simulation(args); a.init()
    b = Simulation(args); b.init()
    for comp, name in enumerate(("u", "v")):
        n = noise_field(1, comp, a.ctx.ny, a.ctx.nx)
        a.ctx.set(name, n); b.ctx.set(name, n)
    for _ in range(5):
        a.advance(a.calcMaxTimestep())
    b.ctx.advance(5)
    b.ctx.sync()
    for name in ("u", "v", "pres", "chi"):
        assert np.array_equal(a.ctx.get(name), b.ctx.get(name)), name
    for k in range(args.count("radius=") + args.count("L=")):
        assert a.ctx.shape(k) == b.ctx.shape(k), k


@pytest.mark.parametrize("args", [FISH, TANDEM], ids=["fish", "tandem"])
def test_operator_steps_then_graph_steps(args):
    """Operator-by-operator steps (which form the next midline ahead on a
    side stream) followed by graph steps: bitwise the same as operator steps
    throughout (the graph's first step takes or forms the current midline)."""
    a = Simulation(args); a.init()
    b = Simulation(args); b.init()
    for comp, name in enumerate(("u", "v")):
        n = noise_field(2, comp, a.ctx.ny, a.ctx.nx)
        a.ctx.set(name, n); b.ctx.set(name, n)
    for _ in range(6):
        a.advance(a.calcMaxTimestep())
    for _ in range(3):
        b.advance(b.calcMaxTimestep())
    b.ctx.advance(3)
    b.ctx.sync()
    for name in ("u", "v", "pres", "chi"):
        assert np.array_equal(a.ctx.get(name), b.ctx.get(name)), name
    for k in range(args.count("fish ")):
        assert a.ctx.shape(k) == b.ctx.shape(k), k


def _operator_step(sim, dt):
    for op in sim.pipeline:
        op(dt)
    sim.ctx.end_step()


@pytest.mark.parametrize("args", [DISK, FISH], ids=["disk", "fish"])
def test_operator_path_call_orders(args):
    """The operator path skips launches the device state makes redundant (the
    dt of calcMaxTimestep carried from the step end, sim.dt already set, the
    RHS divergence formed by advDiff, advDiff beside the obstacle chain).
    Calls in between that change or re-read the state must leave every
    result bitwise the same as the plain loop."""
    a = Simulation(args); a.init()
    b = Simulation(args); b.init()
    for comp, name in enumerate(("u", "v")):
        n = noise_field(4, comp, a.ctx.ny, a.ctx.nx)
        a.ctx.set(name, n); b.ctx.set(name, n)
    for _ in range(8):
        _operator_step(a, a.calcMaxTimestep())
        _ = a.ctx.shape(0)
    # 1: calcMaxTimestep twice, the state re-read between stages
    b.ctx.calc_dt(sync=False); b.calcMaxTimestep(); dt = b.calcMaxTimestep()
    b.pipeline[0](dt); _ = b.ctx.get("chi"); b.pipeline[1](dt); _ = b.ctx.get("tmp")
    b.pipeline[2](dt); b.pipeline[3](-1.0); b.ctx.end_step()
    # 2: a field written back between PutObjectsOnGrid and advDiff, and
    #    between advDiff and PressureSingle
    dt = b.calcMaxTimestep()
    b.pipeline[0](dt); b.ctx.set("u", b.ctx.get("u"))
    b.pipeline[1](dt); b.ctx.set("v", b.ctx.get("v"))
    b.pipeline[2](dt); b.pipeline[3](dt); b.ctx.end_step()
    # 3: the scalars written back (the carried dt is dropped), dt given to
    #    the first stage only
    st = b.ctx.scalars()
    b.ctx.set_scalars(st["time"], st["dt"], st["step"], st["uinfx"], st["uinfy"])
    dt = b.calcMaxTimestep()
    b.pipeline[0](dt)
    for op in b.pipeline[1:]:
        op(-1.0)
    b.ctx.end_step()
    # 4-5: graph steps, then 6-8: operator steps again
    b.ctx.advance(2)
    for _ in range(3):
        _operator_step(b, b.calcMaxTimestep())
    b.ctx.sync()
    for name in ("u", "v", "pres", "chi"):
        assert np.array_equal(a.ctx.get(name), b.ctx.get(name)), name
    assert a.ctx.shape(0) == b.ctx.shape(0)
    assert a.ctx.scalars() == b.ctx.scalars()


# ---- against the committed golden fixtures (no reference build needed) -------

GOLDEN_DIR = __import__("os").path.join(__import__("os").path.dirname(__import__("os").path.abspath(__file__)), "golden")


def _golden(name):
    z = np.load(__import__("os").path.join(GOLDEN_DIR, name + ".npz"))
    d = {k: z[k] for k in z.files}
    d["shape"] = dict(zip(d["shape_keys"].tolist(), d["shape_values"].tolist()))
    return d


@pytest.mark.parametrize("name", ["disk_forced_freespace", "disk_free_periodic", "disk_free_cosine",
                                  "stefanfish", "carlingfish"])
def test_steps_match_golden(name):
    """Same configuration, noise and step count as tests/golden/make_golden.py;
    the fixtures hold the reference's own outputs."""
    g = _golden(name)
    s = Simulation(str(g["args"]))
    s.init()
    seed = int(g["noise_seed"])
    for comp, f in enumerate(("u", "v")):
        s.ctx.set(f, s.ctx.get(f) + noise_field(seed, comp, s.ctx.ny, s.ctx.nx))
    chi0 = s.ctx.get("chi")
    if name.startswith("disk"):
        assert np.array_equal(chi0, g["init_chi"])               # Towers chi: same arithmetic
    else:
        assert rel_err(chi0, g["init_chi"]) < 1e-12              # the reference's own run-to-run level
    dts = []
    for _ in range(int(g["nsteps"])):
        dts.append(s.calcMaxTimestep())
        s.advance(dts[-1])
    assert rel_err(np.array(dts), g["dt"]) < 1e-12
    if "final_u" in g:
        assert rel_err(s.ctx.get("u"), g["final_u"]) < 1e-9
        assert rel_err(s.ctx.get("v"), g["final_v"]) < 1e-9
        assert rel_err(s.ctx.get("pres"), g["final_pres"]) < 1e-8
        assert rel_err(s.ctx.get("chi"), g["final_chi"]) < 1e-12
    a, b = s.ctx.shape(0), g["shape"]
    for key in ("com_x", "com_y", "u", "v", "omega", "orientation"):
        assert abs(a[key] - b[key]) <= 1e-9 * max(abs(b[key]), 1e-3), (key, a[key], b[key])
    fs = max(abs(b["forcex"]), abs(b["forcey"]))
    for key in ("forcex", "forcey", "torque"):
        assert abs(a[key] - b[key]) <= 1e-7 * fs, (key, a[key], b[key])


def test_two_disks_in_contact(ref):
    """Two shapes whose chi overlap from the first step: a forced disk pushes
    a free one (PressureSingle::preventCollidingObstacles, the per-shape RHS
    terms, penalization in shape order, both shapes' forces).  Six steps of
    the operator loop against the reference; small velocity components are
    compared against the scale of the forced speed."""
    r, s = make_pair(ref, TWO_DISKS, noise_seed=5)
    for _ in range(6):
        dt_r = r.step()
        dt_s = s.calcMaxTimestep()
        s.advance(dt_s)
        assert abs(dt_s - dt_r) <= 1e-12 * dt_r
    for k in range(2):
        a, b = s.ctx.shape(k), r.shape(k)
        for key in ("u", "v", "omega"):
            assert abs(a[key] - b[key]) <= 1e-9 * 0.3, (k, key, a[key], b[key])
        for key in ("center_x", "center_y", "com_x", "com_y"):
            assert abs(a[key] - b[key]) <= 1e-12, (k, key, a[key], b[key])
        for key in ("forcex", "forcey"):
            scale = max(abs(b["forcex"]), abs(b["forcey"]))
            assert abs(a[key] - b[key]) <= 1e-8 * scale, (k, key, a[key], b[key])
    assert s.ctx.shape(1)["u"] > 0.01               # the free disk was pushed
    compare_fields(r, s, ["u", "v", "pres"], 1e-8, "two disks, 6 steps")
    compare_fields(r, s, ["chi"], 1e-12, "two disks chi")
