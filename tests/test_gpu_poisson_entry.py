"""The standalone Poisson entry (cup2d_poisson_solve: PoissonSolver::solve
(BSRC, BDST), PoissonSolver.h:35-40) against a solver made by the
reference's own factory, on the same seeded RHS: each solver type, a solve
into another field and one in place (solve(tmp, tmp), as
PressureVarRho_approx calls it)."""
import numpy as np
import pytest

from cubismup_2d_b200 import Cup2DError, Simulation
from cubismup_2d_b200.abi import EINVAL

pytestmark = pytest.mark.gpu

BASE = "-bpdx 4 -bpdy 2 -extent 1 -muteAll 1 -shapes 'disk radius=0.05' "


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _pair(ref, solver, seed):
    args = BASE + ("-poissonType " + solver if solver else "")
    r = ref.RefSim(args)
    s = Simulation(args)
    s.init()
    rhs = np.random.default_rng(seed).standard_normal((r.ny, r.nx))
    r.set("tmp", rhs)
    s.ctx.set("tmp", rhs)
    return r, s


@pytest.mark.parametrize("solver", ["freespace", "periodic", ""], ids=["freespace", "periodic", "cosine"])
def test_solve_into_pressure(ref, solver):
    r, s = _pair(ref, solver, 3)
    r.poisson_solve("tmp", "pres")
    s.ctx.poisson_solve("tmp", "pres")
    assert _rel(s.ctx.get("tmp"), r.get("tmp")) <= 1e-13      # faded in place
    assert _rel(s.ctx.get("pres"), r.get("pres")) <= 1e-10


def test_solve_in_place(ref):
    r, s = _pair(ref, "freespace", 4)
    r.poisson_solve("tmp", "tmp")
    s.ctx.poisson_solve("tmp", "tmp")
    assert _rel(s.ctx.get("tmp"), r.get("tmp")) <= 1e-10


def test_solve_refuses_unknown_fields():
    s = Simulation(BASE)
    s.init()
    with pytest.raises(Cup2DError) as e:
        s.ctx.poisson_solve("tmp", "invRho")                 # constant density: no such plane
    assert e.value.code == EINVAL
