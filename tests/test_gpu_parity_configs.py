"""Parity at the sizes the benchmark workloads run: the Re = 100 forced
cylinder on 512x256 for its full 1000 steps, the self-propelled swimmer on
1024x512 (the default bench workload) and the two swimmers in tandem on
4096x2048 (the large single-GPU case without its falling cylinder), each
against the reference's own operators (oracle/_ref) from the same seeded
state.  The GPU side runs whole graph-replayed steps, as the bench does.

Tolerances: after a stage results agree to rounding (the FFT and the
reduction orders differ from the reference's); over many steps that
rounding grows with the flow's own sensitivity, so the long runs are held
to Cd/Cl within 1e-4 relative and fields within 1e-6 of their scale, the
shorter ones to 1e-8."""
import numpy as np
import pytest

from cubismup_2d_b200 import Simulation
from cubismup_2d_b200.synthetic import noise_field
from test_gpu_parity import compare_shape_all, make_pair, rel_err

pytestmark = pytest.mark.gpu

CYLINDER_RE100 = ("-bpdx 16 -bpdy 8 -extent 1 -CFL 0.1 -nu 1.5e-4 -lambda 1e4 -poissonType freespace "
                  "-muteAll 1 -shapes 'disk radius=0.0375 xpos=0.2 ypos=0.25 bForced=1 bFixed=1 xvel=0.2'")
SWIMMER_1024 = ("-bpdx 32 -bpdy 16 -extent 1 -CFL 0.1 -nu 2e-5 -lambda 1e4 -poissonType freespace "
                "-muteAll 1 -shapes 'stefanfish L=0.2 T=1 xpos=0.4 ypos=0.25'")
TANDEM_4096 = ("-bpdx 128 -bpdy 64 -extent 2 -CFL 0.1 -nu 2e-6 -lambda 1e4 -poissonType freespace "
               "-muteAll 1 -shapes 'stefanfish L=0.1 T=1 xpos=0.6 ypos=0.5, "
               "stefanfish L=0.1 T=1 xpos=0.75 ypos=0.5 phi=0.5'")


def _graph_steps_against_reference(r, s, nsteps, chunk):
    """nsteps reference steps beside the same number of graph steps, in
    chunks; the simulated time must agree after each chunk (the dt
    sequence, formed on the device, is the reference's)."""
    done = 0
    while done < nsteps:
        n = min(chunk, nsteps - done)
        for _ in range(n):
            r.step()
        s.ctx.advance(n)
        done += n
        st = s.ctx.scalars()
        assert st["step"] == r.step_id
        assert abs(st["time"] - r.time) <= 1e-11 * r.time, (done, st["time"], r.time)


def test_cylinder_re100_1000_steps(ref):
    """Config: the forced cylinder at Re = 100 (512x256), 1000 steps from
    rest plus seeded noise.  Cd = 2 Fx / (U^2 2R) and Cl = 2 Fy / (U^2 2R)
    within 1e-4 relative of the reference's (Cl against Cd's scale: it
    starts at rounding level), fields within 1e-6."""
    r, s = make_pair(ref, CYLINDER_RE100, noise_seed=3)
    U, D = 0.2, 2 * 0.0375
    _graph_steps_against_reference(r, s, 1000, 100)
    s.ctx.sync()
    a, b = s.ctx.shape(0), r.shape(0)
    cd_s, cd_r = 2 * a["forcex"] / (U * U * D), 2 * b["forcex"] / (U * U * D)
    cl_s, cl_r = 2 * a["forcey"] / (U * U * D), 2 * b["forcey"] / (U * U * D)
    assert abs(cd_s - cd_r) <= 1e-4 * abs(cd_r), (cd_s, cd_r)
    assert abs(cl_s - cl_r) <= 1e-4 * abs(cd_r), (cl_s, cl_r)
    for f in ("u", "v", "pres"):
        assert rel_err(s.ctx.get(f), r.get(f)) <= 1e-6, f


def test_swimmer_1024x512_50_steps(ref):
    """The bench's default workload: StefanFish L = 0.2 at Re = 2000 on
    1024x512, 50 graph steps against 50 reference steps: the body's
    position, velocity and every force sum, and the fields."""
    r, s = make_pair(ref, SWIMMER_1024, noise_seed=0)
    assert rel_err(s.ctx.get("chi"), r.get("chi")) <= 1e-12
    _graph_steps_against_reference(r, s, 50, 10)
    s.ctx.sync()
    a, b = s.ctx.shape(0), r.shape(0)
    for key in ("com_x", "com_y", "center_x", "center_y", "orientation"):
        assert abs(a[key] - b[key]) <= 1e-10, (key, a[key], b[key])
    vscale = max(abs(b["u"]), abs(b["v"]), 1e-6)
    for key in ("u", "v"):
        assert abs(a[key] - b[key]) <= 1e-7 * vscale, (key, a[key], b[key])
    assert abs(a["omega"] - b["omega"]) <= 1e-7 * max(abs(b["omega"]), 1e-3)
    compare_shape_all(a, b, 1e-7, "swimmer 1024x512, 50 steps")
    for f in ("u", "v", "pres"):
        assert rel_err(s.ctx.get(f), r.get(f)) <= 1e-8, f
    assert rel_err(s.ctx.get("chi"), r.get("chi")) <= 1e-9


def test_tandem_4096x2048_2_steps(ref):
    """The large case's two swimmers in tandem on 4096x2048 (8.4 M cells),
    placement and two steps against the reference."""
    r, s = make_pair(ref, TANDEM_4096, noise_seed=1)
    assert rel_err(s.ctx.get("chi"), r.get("chi")) <= 1e-12
    _graph_steps_against_reference(r, s, 2, 2)
    s.ctx.sync()
    for f in ("u", "v", "pres"):
        assert rel_err(s.ctx.get(f), r.get(f)) <= 1e-8, f
    assert rel_err(s.ctx.get("chi"), r.get("chi")) <= 1e-9
    for k in range(2):
        a, b = s.ctx.shape(k), r.shape(k)
        for key in ("com_x", "com_y", "orientation"):
            assert abs(a[key] - b[key]) <= 1e-10, (k, key, a[key], b[key])
        compare_shape_all(a, b, 1e-7, f"tandem shape {k}")


# grids whose block counts are not powers of two: the free-space solve pads
# to powers of two (the reference pads to 2N - 1 with FFTW's mixed-radix
# transforms); the convolution on the domain is the same
ODD_GRIDS = [
    ("-bpdx 3 -bpdy 2 -extent 1 -CFL 0.1 -nu 1e-3 -poissonType freespace -muteAll 1 "
     "-shapes 'disk radius=0.08 xpos=0.4 ypos=0.3 bForced=1 bFixed=1 xvel=0.2'"),
    ("-bpdx 24 -bpdy 12 -extent 1 -CFL 0.1 -nu 4e-5 -lambda 1e4 -poissonType freespace -muteAll 1 "
     "-shapes 'stefanfish L=0.2 T=1 xpos=0.4 ypos=0.25'"),
]


@pytest.mark.parametrize("args", ODD_GRIDS, ids=["96x64_disk", "768x384_swimmer"])
def test_free_space_on_grids_of_any_block_count(ref, args):
    r, s = make_pair(ref, args, noise_seed=6)
    dt = 1e-4
    r.run_op("advDiff", dt); s.ctx.adv_diff(dt)
    r.run_op("PressureSingle", dt); s.ctx.pressure_single(dt)
    assert rel_err(s.ctx.get("tmp"), r.get("tmp")) <= 1e-12
    assert rel_err(s.ctx.get("pres"), r.get("pres")) <= 1e-10
    assert rel_err(s.ctx.get("u"), r.get("u")) <= 1e-10
    r2, s2 = make_pair(ref, args, noise_seed=7)
    _graph_steps_against_reference(r2, s2, 6, 3)
    for f in ("u", "v", "pres"):
        assert rel_err(s2.ctx.get(f), r2.get(f)) <= 1e-8, f
    compare_shape_all(s2.ctx.shape(0), r2.shape(0), 1e-7, "odd grid")
