"""The discrete adjoint (cup2d_adjoint_run; no counterpart in the reference).
Objectives: the time-averaged kinetic energy in a box behind a forced
cylinder, and its time-averaged force (ComputeForces' forcex / forcey).
Checked: the objective against the plain operator steps; the gradient with
respect to the initial velocity along localized directions (in the wake, at
the body, at the domain edge where the fades and the outflow correction
act) and with respect to the body's velocity, against central finite
differences of this FP64 forward and of the reference's own steps (the
compiled oracle); independence of the checkpoint interval; the final state;
the torch.autograd binding; the configurations it refuses."""
import numpy as np
import pytest

from cubismup_2d_b200 import Cup2DError, Simulation
from cubismup_2d_b200.abi import ENOTSUP

pytestmark = pytest.mark.gpu

BASE = "-extent 1 -CFL 0.1 -nu 1e-3 -lambda 1e4 -muteAll 1 "
FORCED = (BASE + "-bpdx 8 -bpdy 4 -poissonType freespace "
          "-shapes 'disk radius=0.06 xpos=0.3 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'")
# a free disk held on the grid (bFixed: the frame follows it), started at
# 0.2: its velocity comes from the momentum integrals every step
FREE = (BASE + "-bpdx 8 -bpdy 4 -poissonType freespace "
        "-shapes 'disk radius=0.06 xpos=0.3 ypos=0.25 bFixed=1 xvel=0.2'")
# a tethered swimmer: StefanFish held on the grid (forced, fixed) in a 0.2
# stream; its chi and udef move with its gait alone
TETHERED = (BASE.replace("-nu 1e-3", "-nu 1e-4") + "-bpdx 8 -bpdy 4 -poissonType freespace "
            "-shapes 'stefanfish L=0.18 T=1 xpos=0.35 ypos=0.25 bFixed=1 bForced=1 xvel=0.2'")
BOX = (0.36, 0.62, 0.14, 0.36)
NSTEPS = 16
BUMPS = {"wake": (0.45, 0.27, 0.04), "body": (0.3, 0.31, 0.03),
         "edge": (0.97, 0.22, 0.05), "inflow": (0.05, 0.3, 0.05)}
# central differences at 1e-6: the fade's and the obstacle terms' sign tests
# make the forward piecewise smooth, and a larger step crosses their
# switches (1e-4 does, at the edge and the inflow)
EPS = 1e-6
ENERGY = dict(box=BOX)
DRAG = dict(box=None, w_force=(1.0, 0.0))
BOTH = dict(box=BOX, w_energy=1.0, w_force=(1e-4, 2e-4))
ALL = dict(box=BOX, w_energy=1.0, w_force=(1e-4, 2e-4), w_body=(1e-3, 2e-3, 1e-4))
# the benchmark's adjoint objective on a held swimmer: its drag (the thrust
# it would swim with, negated) and 0.1 of its mean |torque|
THRUST_TORQUE = dict(box=None, w_force=(1.0, 0.0), w_torque=0.1)


def _developed(args=FORCED, warm=40):
    s = Simulation(args)
    s.init()
    for _ in range(warm):
        s.advance(s.calcMaxTimestep())
    s.ctx.sync()
    return s


def _developed_free():
    """The free disk in the developed flow of the forced one (its velocity,
    -0.2, and the fields after the forced warm-up): a free body's state at
    rest would leave the RHS near zero, where the obstacle terms' and the
    fade's sign tests switch under any finite difference."""
    f = _developed(FORCED)
    u, v, st = f.ctx.get("u"), f.ctx.get("v"), f.ctx.shape(0)
    s = Simulation(FREE)
    s.init()
    s.ctx.set("u", u)
    s.ctx.set("v", v)
    s.ctx.set_shape(0, {"u": st["u"], "v": st["v"], "omega": st["omega"]})
    s.ctx.sync()
    return s


def _bump(ctx, where, au=0.7, av=-0.4):
    cx, cy, sig = BUMPS[where]
    x = (np.arange(ctx.nx) + 0.5) * ctx.h
    y = (np.arange(ctx.ny) + 0.5) * ctx.h
    X, Y = np.meshgrid(x, y)
    g = np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / sig ** 2)
    return au * g, av * g


def _fd(ctx, blob, dts, obj, du=None, dv=None, dub=None):
    """Central difference of J along (du, dv) of the initial velocity and dub
    of the body velocity, the dt schedule frozen."""
    u0, v0 = ctx.get("u"), ctx.get("v")
    ub = ctx.shape(0)
    Js = []
    for sgn in (1, -1):
        ctx.restore(blob)
        if du is not None:
            ctx.set("u", u0 + sgn * EPS * du)
            ctx.set("v", v0 + sgn * EPS * dv)
        if dub is not None:
            dub3 = tuple(dub) + (0.0,) * (3 - len(dub))
            ctx.set_shape(0, {"u": ub["u"] + sgn * EPS * dub3[0], "v": ub["v"] + sgn * EPS * dub3[1],
                              "omega": ub["omega"] + sgn * EPS * dub3[2]})
        Js.append(ctx.adjoint(NSTEPS, dt=dts, gradient=False, **obj)[0])
    ctx.restore(blob)
    return (Js[0] - Js[1]) / (2 * EPS)


def _objective_plain(s, dts, obj):
    """J along the plain operator path."""
    n = s.ctx
    box = obj.get("box")
    wE = obj.get("w_energy", 1.0) if box is not None else 0.0
    wF = obj.get("w_force", (0.0, 0.0))
    J = 0.0
    for dt in dts:
        s.advance(dt)
        if wE:
            i0, i1 = int(np.floor(box[0] / n.h)), int(np.ceil(box[1] / n.h))
            j0, j1 = int(np.floor(box[2] / n.h)), int(np.ceil(box[3] / n.h))
            u, v = n.get("u")[j0:j1, i0:i1], n.get("v")[j0:j1, i0:i1]
            J += wE * 0.5 * n.h ** 2 * float(np.sum(u * u + v * v))
        st = n.shape(0)
        J += wF[0] * st["forcex"] + wF[1] * st["forcey"]
    return J / len(dts)


@pytest.mark.parametrize("obj", [ENERGY, DRAG, BOTH], ids=["energy", "drag", "both"])
def test_objective_and_final_state_match_plain_steps(obj):
    s = _developed()
    blob = s.ctx.checkpoint()
    J, gu, gv, gb, dts, ms = s.ctx.adjoint(NSTEPS, every=5, **obj)
    assert np.all(dts > 0) and ms[0] > 0 and ms[1] > 0
    assert np.all(np.isfinite(gu)) and np.all(np.isfinite(gv)) and np.any(gu != 0)
    assert np.all(np.isfinite(gb))
    ua, va = s.ctx.get("u"), s.ctx.get("v")
    s.ctx.restore(blob)
    Jp = _objective_plain(s, dts, obj)
    assert abs(J - Jp) <= 1e-12 * abs(Jp), (J, Jp)
    # the context ends in the forward's final state
    assert np.array_equal(ua, s.ctx.get("u")) and np.array_equal(va, s.ctx.get("v"))


@pytest.mark.parametrize("where", list(BUMPS))
def test_energy_gradient_matches_finite_differences(where):
    s = _developed()
    blob = s.ctx.checkpoint()
    J, gu, gv, gb, dts, _ = s.ctx.adjoint(NSTEPS, every=5, **ENERGY)
    s.ctx.restore(blob)
    du, dv = _bump(s.ctx, where)
    ad = float(np.sum(gu * du) + np.sum(gv * dv))
    fd = _fd(s.ctx, blob, dts, ENERGY, du, dv)
    assert abs(fd) > 1e-8 * abs(J), (where, fd, J)
    assert abs(ad - fd) <= 2e-6 * abs(fd), (where, ad, fd)


@pytest.mark.parametrize("where", ["body", "wake", "inflow"])
def test_drag_gradient_matches_finite_differences(where):
    s = _developed()
    blob = s.ctx.checkpoint()
    J, gu, gv, gb, dts, _ = s.ctx.adjoint(NSTEPS, every=5, **DRAG)
    s.ctx.restore(blob)
    du, dv = _bump(s.ctx, where)
    ad = float(np.sum(gu * du) + np.sum(gv * dv))
    fd = _fd(s.ctx, blob, dts, DRAG, du, dv)
    assert abs(ad - fd) <= 1e-5 * max(abs(fd), 1e-3 * abs(J)), (where, ad, fd)


@pytest.mark.parametrize("solver", ["cosine", "periodic"])
def test_other_solvers_gradient_matches_finite_differences(solver):
    """The cosine (the reference's default) and periodic solvers: their
    transforms with the fade off are the transposed solve too."""
    s = _developed(FORCED.replace("freespace", solver))
    blob = s.ctx.checkpoint()
    J, gu, gv, gb, dts, _ = s.ctx.adjoint(NSTEPS, every=5, **BOTH)
    s.ctx.restore(blob)
    for where in ("body", "edge"):
        du, dv = _bump(s.ctx, where)
        ad = float(np.sum(gu * du) + np.sum(gv * dv))
        fd = _fd(s.ctx, blob, dts, BOTH, du, dv)
        assert abs(ad - fd) <= 1e-5 * abs(fd), (solver, where, ad, fd)
    fd = _fd(s.ctx, blob, dts, BOTH, dub=(1.0, 0.0))
    assert abs(gb[0] - fd) <= 1e-5 * abs(fd), (solver, gb[0], fd)


@pytest.mark.parametrize("obj", [ENERGY, DRAG], ids=["energy", "drag"])
def test_body_velocity_gradient_matches_finite_differences(obj):
    s = _developed()
    blob = s.ctx.checkpoint()
    J, gu, gv, gb, dts, _ = s.ctx.adjoint(NSTEPS, every=5, **obj)
    s.ctx.restore(blob)
    # the y component is near zero (the flow is almost symmetric about the
    # cylinder's axis): the differences' rounding, about 1e-16 |J| / EPS,
    # bounds what they can resolve there
    floor = 1e-13 * abs(J) / EPS
    for comp in (0, 1, 2):
        d = [0.0, 0.0, 0.0]
        d[comp] = 1.0
        fd = _fd(s.ctx, blob, dts, obj, dub=d)
        assert abs(gb[comp] - fd) <= 1e-5 * abs(fd) + floor, (comp, gb[comp], fd)
    assert abs(gb[0]) > 1e3 * floor


@pytest.mark.parametrize("where", ["body", "wake", "edge"])
def test_free_body_gradient_matches_finite_differences(where):
    """A free disk: the momentum integrals, the 3x3 solve and the body
    velocity's role as the next step's lab velocity, transposed."""
    s = _developed_free()
    blob = s.ctx.checkpoint()
    J, gu, gv, gb, dts, _ = s.ctx.adjoint(NSTEPS, every=5, **ALL)
    s.ctx.restore(blob)
    du, dv = _bump(s.ctx, where)
    ad = float(np.sum(gu * du) + np.sum(gv * dv))
    fd = _fd(s.ctx, blob, dts, ALL, du, dv)
    assert abs(ad - fd) <= 1e-5 * abs(fd), (where, ad, fd)
    if where == "body":
        # the initial body velocity sets the first step's lab velocity only
        floor = 1e-13 * abs(J) / EPS
        for comp in (0, 1):
            d = [0.0, 0.0, 0.0]
            d[comp] = 1.0
            fd = _fd(s.ctx, blob, dts, ALL, dub=d)
            assert abs(gb[comp] - fd) <= 1e-5 * abs(fd) + floor, (comp, gb[comp], fd)
        assert gb[2] == 0.0


@pytest.mark.parametrize("obj", [ENERGY, DRAG], ids=["energy", "drag"])
def test_tethered_swimmer_gradient_matches_finite_differences(obj):
    """A deforming body: each transposed step uses the obstacle tiles its
    forward step placed (kept by the recomputation)."""
    s = _developed(TETHERED, warm=60)
    blob = s.ctx.checkpoint()
    J, gu, gv, gb, dts, _ = s.ctx.adjoint(NSTEPS, every=5, **obj)
    s.ctx.restore(blob)
    for where in ("body", "wake"):
        du, dv = _bump(s.ctx, where)
        ad = float(np.sum(gu * du) + np.sum(gv * dv))
        fd = _fd(s.ctx, blob, dts, obj, du, dv)
        assert abs(ad - fd) <= 1e-5 * abs(fd), (where, ad, fd)
    fd = _fd(s.ctx, blob, dts, obj, dub=(1.0, 0.0, 0.0))
    assert abs(gb[0] - fd) <= 1e-5 * abs(fd), (gb[0], fd)


def _fd_gait(ctx, blob, dts, obj, q, theta, eps=1e-6):
    Js = []
    for sgn in (1, -1):
        ctx.restore(blob)
        th = np.array(theta, dtype=np.float64)
        th[q] += sgn * eps
        ctx.set_fish_gait(0, th)
        Js.append(ctx.adjoint(NSTEPS, dt=dts, gradient=False, **obj)[0])
        ctx.set_fish_gait(0, theta)
    ctx.restore(blob)
    return (Js[0] - Js[1]) / (2 * eps)


@pytest.fixture(scope="module")
def swimming():
    """The tethered swimmer past its first period (the gait's ramp), by
    graph steps, and its checkpoint."""
    s = Simulation(TETHERED)
    s.init()
    s.ctx.advance(1200)
    s.ctx.sync()
    assert s.ctx.scalars()["time"] > 1.0
    return s, s.ctx.checkpoint()


@pytest.mark.parametrize("obj", [DRAG, ENERGY], ids=["drag", "energy"])
def test_gait_gradient_matches_finite_differences(swimming, obj):
    """dJ/d(amplitude, phase, the six curvature control scales) of a
    tethered StefanFish: the adjoint's per-step geometry sensitivities
    contracted with the placement's central differences, against central
    differences of the whole simulation (measured agreement 1e-8..1e-6)."""
    s, blob = swimming
    s.ctx.restore(blob)
    theta = s.ctx.fish_gait(0)
    assert np.array_equal(theta, [1, 0, 1, 1, 1, 1, 1, 1])
    # the placement's difference step equal to the whole simulation's (the
    # forward is piecewise smooth: both cross the same raster switches)
    J, gu, gv, gb, dts, ms, gg = s.ctx.adjoint(NSTEPS, every=5, gait=True, gait_step=1e-6, **obj)
    s.ctx.restore(blob)
    assert np.array_equal(s.ctx.fish_gait(0), theta)
    scale = np.max(np.abs(gg))
    assert scale > 0
    for q in range(8):
        fd = _fd_gait(s.ctx, blob, dts, obj, q, theta)
        assert abs(gg[q] - fd) <= 1e-5 * abs(fd) + 1e-7 * scale, (q, gg[q], fd)


def test_gait_gradient_matches_reference_finite_differences(ref):
    """The tethered swimmer from rest over 216 steps (its gait ramping up):
    the amplitude and phase components against central differences of the
    reference's own StefanFish (-amplitudeFactor, -phi) from the same
    state with the same dt schedule (measured agreement ~4e-6)."""
    from cubismup_2d_b200.synthetic import noise_field
    n = 216
    s = Simulation(TETHERED)
    s.init()
    r0 = ref.RefSim(TETHERED)
    ic = {}
    for comp, name in enumerate(("u", "v")):
        ic[name] = r0.get(name) + 0.05 * noise_field(3, comp, r0.ny, r0.nx)
        s.ctx.set(name, ic[name])
    r0.close()
    J, gu, gv, gb, dts, ms, gg = s.ctx.adjoint(n, every=24, gait=True, gait_step=1e-6, **DRAG)

    def ref_J(extra):
        r = ref.RefSim(TETHERED.replace("xvel=0.2'", "xvel=0.2 " + extra + "'"))
        r.set("u", ic["u"])
        r.set("v", ic["v"])
        Jr = 0.0
        for dt in dts:
            r.set_time(r.time, r.step_id, dt)
            r.advance()
            Jr += r.shape(0)["forcex"]
        r.close()
        return Jr / n

    assert abs(ref_J("") - J) <= 1e-12 * abs(J)
    for q, key, base in ((0, "amplitudeFactor", 1.0), (1, "phi", 0.0)):
        vp, vm = base + 1e-6, base - 1e-6
        fd = (ref_J(f"{key}={vp!r}") - ref_J(f"{key}={vm!r}")) / (vp - vm)
        assert abs(gg[q] - fd) <= 2e-5 * abs(fd), (key, gg[q], fd)


def test_envelope_swimmer_gait():
    """The envelope swimmer's gait: the eight Fourier coefficients of its
    curvature amplitude, from a seeded N(1, 0.05) draw (the benchmark's
    initialisation), the drag and |torque| objective."""
    args = TETHERED.replace("stefanfish", "envelopefish")
    s = Simulation(args)
    s.init()
    theta = np.random.default_rng(11).normal(1.0, 0.05, 8)
    s.ctx.set_fish_gait(0, theta)
    assert np.array_equal(s.ctx.fish_gait(0), theta)
    s.ctx.advance(1200)
    s.ctx.sync()
    blob = s.ctx.checkpoint()
    J, gu, gv, gb, dts, ms, gg = s.ctx.adjoint(NSTEPS, every=8, gait=True, gait_step=1e-6, **THRUST_TORQUE)
    s.ctx.restore(blob)
    scale = np.max(np.abs(gg))
    assert scale > 0
    for q in range(8):
        fd = _fd_gait(s.ctx, blob, dts, THRUST_TORQUE, q, theta)
        assert abs(gg[q] - fd) <= 1e-5 * abs(fd) + 1e-7 * scale, (q, gg[q], fd)


def test_torque_objective_gradient(swimming):
    """The |torque| term: the field gradient and the gait gradient (the
    torque's surface normals and its centre of mass) against central
    differences."""
    s, blob = swimming
    s.ctx.restore(blob)
    theta = s.ctx.fish_gait(0)
    J, gu, gv, gb, dts, ms, gg = s.ctx.adjoint(NSTEPS, every=8, gait=True, gait_step=1e-6, **THRUST_TORQUE)
    s.ctx.restore(blob)
    Jp = 0.0
    for dt in dts:
        s.advance(dt)
        st = s.ctx.shape(0)
        Jp += st["forcex"] + 0.1 * abs(st["torque"])
    assert abs(J - Jp / NSTEPS) <= 1e-12 * abs(J), (J, Jp / NSTEPS)
    s.ctx.restore(blob)
    for where in ("body", "wake"):
        du, dv = _bump(s.ctx, where)
        ad = float(np.sum(gu * du) + np.sum(gv * dv))
        fd = _fd(s.ctx, blob, dts, THRUST_TORQUE, du, dv)
        assert abs(ad - fd) <= 1e-5 * abs(fd), (where, ad, fd)
    scale = np.max(np.abs(gg))
    for q in range(8):
        fd = _fd_gait(s.ctx, blob, dts, THRUST_TORQUE, q, theta)
        assert abs(gg[q] - fd) <= 1e-5 * abs(fd) + 1e-7 * scale, (q, gg[q], fd)


def test_gait_descent_lowers_drag(swimming):
    """Steps against the gait gradient: a small one lowers the time-averaged
    drag by alpha |grad|^2 (first order); a larger one (a few 1e-3 in theta)
    still lowers it, though the raster's switches make the drag only
    piecewise smooth in the gait (measured: 0.67 of the first-order
    decrease)."""
    s, blob = swimming
    s.ctx.restore(blob)
    theta = s.ctx.fish_gait(0)
    J, gu, gv, gb, dts, ms, gg = s.ctx.adjoint(NSTEPS, every=8, gait=True, gait_step=1e-6, **DRAG)
    n2 = float(np.sum(gg * gg))
    for frac, check_first_order in ((1e-4, True), (3e-2, False)):
        alpha = frac * abs(J) / n2
        s.ctx.restore(blob)
        s.ctx.set_fish_gait(0, theta - alpha * gg)
        J2 = s.ctx.adjoint(NSTEPS, dt=dts, gradient=False, **DRAG)[0]
        s.ctx.set_fish_gait(0, theta)
        assert J2 < J, (frac, J, J2)
        if check_first_order:
            assert abs((J - J2) / (alpha * n2) - 1) < 1e-2, (J, J2, alpha * n2)
    s.ctx.restore(blob)


def test_gait_set_round_trip(swimming):
    s, blob = swimming
    s.ctx.restore(blob)
    th = np.array([1.1, 0.3, 1, 0.9, 1.2, 1, 1, 0.8])
    s.ctx.set_fish_gait(0, th)
    assert np.array_equal(s.ctx.fish_gait(0), th)
    # a checkpoint loads only into a context of its gait
    with pytest.raises(Cup2DError):
        s.ctx.restore(blob)
    s.ctx.set_fish_gait(0, [1, 0, 1, 1, 1, 1, 1, 1])
    s.ctx.restore(blob)


def test_free_body_objective_matches_plain_steps():
    s = _developed_free()
    blob = s.ctx.checkpoint()
    J, gu, gv, gb, dts, _ = s.ctx.adjoint(NSTEPS, every=5, **ALL)
    s.ctx.restore(blob)
    n = s.ctx
    Jp = 0.0
    i0, i1 = int(np.floor(BOX[0] / n.h)), int(np.ceil(BOX[1] / n.h))
    j0, j1 = int(np.floor(BOX[2] / n.h)), int(np.ceil(BOX[3] / n.h))
    for dt in dts:
        s.advance(dt)
        u, v = n.get("u")[j0:j1, i0:i1], n.get("v")[j0:j1, i0:i1]
        st = n.shape(0)
        Jp += (0.5 * n.h ** 2 * float(np.sum(u * u + v * v)) + 1e-4 * st["forcex"] + 2e-4 * st["forcey"]
               + 1e-3 * st["u"] + 2e-3 * st["v"] + 1e-4 * st["omega"])
    Jp /= len(dts)
    assert abs(J - Jp) <= 1e-12 * abs(Jp), (J, Jp)


@pytest.mark.parametrize("args", [FORCED, FREE], ids=["forced", "free"])
def test_gradient_matches_reference_finite_differences(ref, args):
    """Central differences of the reference's own steps (the compiled
    oracle), from the same state with the same dt schedule."""
    s = _developed() if args == FORCED else _developed_free()
    blob = s.ctx.checkpoint()
    J, gu, gv, gb, dts, _ = s.ctx.adjoint(NSTEPS, every=5, **BOTH)
    s.ctx.restore(blob)
    u0, v0 = s.ctx.get("u"), s.ctx.get("v")
    ub = s.ctx.shape(0)
    du, dv = _bump(s.ctx, "body")
    n = s.ctx
    i0, i1 = int(np.floor(BOX[0] / n.h)), int(np.ceil(BOX[1] / n.h))
    j0, j1 = int(np.floor(BOX[2] / n.h)), int(np.ceil(BOX[3] / n.h))

    def ref_J(eu, eb):
        r = ref.RefSim(args)
        r.set("u", u0 + eu * du)
        r.set("v", v0 + eu * dv)
        r.set_shape_velocity(0, ub["u"] + eb, ub["v"], ub["omega"])
        Jr = 0.0
        for dt in dts:
            r.set_time(r.time, r.step_id, dt)
            r.advance()
            u, v = r.get("u")[j0:j1, i0:i1], r.get("v")[j0:j1, i0:i1]
            st = r.shape(0)
            Jr += (0.5 * n.h ** 2 * float(np.sum(u * u + v * v)) + BOTH["w_force"][0] * st["forcex"]
                   + BOTH["w_force"][1] * st["forcey"])
        r.close()
        return Jr / len(dts)

    J0 = ref_J(0.0, 0.0)
    assert abs(J0 - J) <= 1e-9 * abs(J), (J0, J)
    fd_u = (ref_J(EPS, 0.0) - ref_J(-EPS, 0.0)) / (2 * EPS)
    ad_u = float(np.sum(gu * du) + np.sum(gv * dv))
    assert abs(ad_u - fd_u) <= 1e-5 * abs(fd_u), (ad_u, fd_u)
    fd_b = (ref_J(0.0, EPS) - ref_J(0.0, -EPS)) / (2 * EPS)
    # a free body's initial velocity sets only the first step's lab
    # velocity: a small derivative, resolved down to the differences of the
    # two codes' summation orders (about 1e-12 |J| per evaluation)
    assert abs(gb[0] - fd_b) <= 1e-5 * abs(fd_b) + 1e-12 * abs(J) / EPS, (gb[0], fd_b)


def test_benchmark_cylinder_gradient():
    """The benchmark's forced cylinder (512x256, Re=100): the drag's
    body-velocity gradient over 200 steps, checkpoints every 20, against a
    central difference, and its cost against the same steps as graph steps."""
    args = ("-bpdx 16 -bpdy 8 -extent 1 -CFL 0.1 -nu 1.5e-4 -lambda 1e4 -poissonType freespace -muteAll 1 "
            "-shapes 'disk radius=0.0375 xpos=0.2 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'")
    s = Simulation(args)
    s.init()
    s.ctx.advance(50)
    s.ctx.sync()
    blob = s.ctx.checkpoint()
    J, gu, gv, gb, dts, ms = s.ctx.adjoint(200, every=20, **DRAG)
    s.ctx.restore(blob)
    graph_ms = s.ctx.time_step(200)
    eps, ub = 1e-6, s.ctx.shape(0)["u"]
    Js = []
    for sgn in (1, -1):
        s.ctx.restore(blob)
        s.ctx.set_shape(0, {"u": ub + sgn * eps})
        Js.append(s.ctx.adjoint(200, dt=dts, gradient=False, **DRAG)[0])
    fd = (Js[0] - Js[1]) / (2 * eps)
    assert abs(gb[0] - fd) <= 1e-4 * abs(fd), (gb[0], fd)
    assert ms[1] < 6 * graph_ms, (ms, graph_ms)


def test_checkpoint_interval_does_not_change_the_gradient():
    s = _developed()
    blob = s.ctx.checkpoint()
    ref = s.ctx.adjoint(NSTEPS, every=NSTEPS, **BOTH)
    scale = max(np.max(np.abs(ref[1])), np.max(np.abs(ref[2])))
    for every in (1, 3):
        s.ctx.restore(blob)
        J, gu, gv, gb, dts, _ = s.ctx.adjoint(NSTEPS, every=every, dt=ref[4], **BOTH)
        assert abs(J - ref[0]) <= 1e-13 * abs(ref[0])
        assert np.max(np.abs(gu - ref[1])) <= 1e-12 * scale
        assert np.max(np.abs(gv - ref[2])) <= 1e-12 * scale
        assert np.allclose(gb, ref[3], rtol=1e-11, atol=0)


def test_autograd_binding():
    torch = pytest.importorskip("torch")
    from adjoint_binding import objective
    s = _developed()
    blob = s.ctx.checkpoint()
    J, gu, gv, gb, dts, _ = s.ctx.adjoint(NSTEPS, every=5, **BOTH)
    s.ctx.restore(blob)
    u0 = torch.from_numpy(s.ctx.get("u")).requires_grad_()
    v0 = torch.from_numpy(s.ctx.get("v")).requires_grad_()
    st = s.ctx.shape(0)
    ub = torch.tensor([st["u"], st["v"], st["omega"]], dtype=torch.float64, requires_grad=True)
    kw = dict(BOTH, dt=dts, every=5)
    Jt = objective(s.ctx, blob, NSTEPS, u0, v0, ub, **kw)
    Jt.backward()
    assert abs(Jt.item() - J) <= 1e-13 * abs(J)
    scale = np.max(np.abs(gu))
    assert np.max(np.abs(u0.grad.numpy() - gu)) <= 1e-12 * scale
    assert np.max(np.abs(v0.grad.numpy() - gv)) <= 1e-12 * scale
    assert np.allclose(ub.grad.numpy(), gb, rtol=1e-11, atol=0)
    # a small step against the gradient lowers the objective by about
    # alpha |grad|^2
    with torch.no_grad():
        n2 = float((u0.grad ** 2).sum() + (v0.grad ** 2).sum() + (ub.grad ** 2).sum())
        alpha = 1e-3 * abs(J) / n2
        J2 = objective(s.ctx, blob, NSTEPS, u0 - alpha * u0.grad, v0 - alpha * v0.grad, ub - alpha * ub.grad, **kw)
    assert J2.item() < J
    assert abs((J - J2.item()) / (alpha * n2) - 1) < 1e-2


@pytest.mark.parametrize("args", [
    FORCED + " -precision fp32",
    BASE + "-bpdx 8 -bpdy 4 -poissonType freespace -shapes 'disk radius=0.06 xpos=0.3 ypos=0.25 xvel=0.2'",
    BASE + "-bpdx 8 -bpdy 4 -poissonType freespace "
    "-shapes 'disk radius=0.06 xpos=0.3 ypos=0.25 bFixed=1 bForcedx=1 xvel=0.2'",
    BASE + "-bpdx 8 -bpdy 4 -poissonType freespace -shapes 'stefanfish L=0.18 T=1 xpos=0.4 ypos=0.25'",
    BASE + "-bpdx 8 -bpdy 4 -poissonType freespace "
    "-shapes 'stefanfish L=0.18 T=1 xpos=0.4 ypos=0.25 bFixed=1 bForced=1 pid=1'",
    FORCED + " -iterativePenalization 1",
    FORCED.replace("xvel=0.2", "xvel=0.2 tAccel=5"),
], ids=["fp32", "moving_disk", "half_forced", "free_swimmer", "pid_swimmer", "iterated", "accelerating"])
def test_uncovered_configurations_refused(args):
    s = Simulation(args)
    s.init()
    with pytest.raises(Cup2DError) as e:
        s.ctx.adjoint(4, BOX)
    assert e.value.code == ENOTSUP
