"""Oracle test infrastructure: ctypes wrapper of oracle/_ref/libcup2d_ref.so.

The library is the reference's OWN operator sources (PutObjectsOnGrid.cpp,
advDiff.cpp, PressureSingle.cpp, PressureIterator_unif.cpp, advDiffGrav.cpp,
PressureIterator_approx.cpp, ComputeForces.cpp, Helpers.cpp, Shape.cpp,
Obstacles/*.cpp, Poisson/PoissonSolver.cpp, Poisson/FFTW_freespace.cpp,
SimulationData.cpp) compiled unmodified against the project-written shims in
oracle/shim, driven by oracle/ref_driver.cpp, which restates
Simulation.cpp:66-305: the constant-density branch and the variable-density
one with -iterativePenalization (advDiffGrav + PressureVarRho_approx).

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
use this module; the product never does.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libcup2d_ref.so")
# the reference's source tree: $CUP2D_REFERENCE_SOURCE, else a checkout named
# "reference" beside this repository
REFERENCE_SOURCE = os.environ.get(
    "CUP2D_REFERENCE_SOURCE",
    os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference", "source"))

# order of ref_get_shape's output; the product's cup2d_shape_state matches it
SHAPE_FIELDS = [
    "center_x", "center_y", "com_x", "com_y", "orientation", "u", "v", "omega",
    "M", "J", "d_gm_x", "d_gm_y", "lab_com_x", "lab_com_y",
    "penalM", "penalJ", "penalDX", "penalDY", "fluidMomX", "fluidMomY", "fluidAngMom",
    "perimeter", "forcex", "forcey", "forcex_P", "forcey_P", "forcex_V", "forcey_V",
    "torque", "torque_P", "torque_V", "drag", "thrust", "circulation",
    "Pout", "PoutBnd", "defPower", "defPowerBnd", "Pthrust", "Pdrag", "EffPDef", "EffPDefBnd",
]
FIELDS = {"u": 0, "v": 1, "chi": 2, "pres": 3, "tmp": 4, "udef_x": 5, "udef_y": 6,
          "invRho": 7, "tmpV_x": 8, "tmpV_y": 9}
OPS = {"PutObjectsOnGrid": 0, "advDiff": 1, "PressureSingle": 2, "ComputeForces": 3,
       "advDiffGrav": 1, "PressureVarRho_approx": 2}

_lib = None


def available():
    return os.path.exists(LIB_PATH) or os.path.isdir(REFERENCE_SOURCE)


def build(quiet=True):
    """Compile the reference through oracle/Makefile (needs the reference tree)."""
    if not os.path.isdir(REFERENCE_SOURCE):
        raise RuntimeError("reference sources not present; cannot build oracle/_ref")
    out = subprocess.run(["make", "-C", HERE, "-j8", "REF=" + REFERENCE_SOURCE],
                         capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle/_ref build failed:\n" + out.stdout[-4000:] + out.stderr[-4000:])


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    L = ctypes.CDLL(LIB_PATH)
    vp, d, i = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
    dp = ctypes.POINTER(ctypes.c_double)
    L.ref_create.restype = vp
    L.ref_create.argtypes = [ctypes.c_char_p]
    L.ref_last_error.restype = ctypes.c_char_p
    L.ref_destroy.argtypes = [vp]
    for name in ("ref_nx", "ref_ny", "ref_stepid", "ref_nshapes", "ref_advance", "ref_iterations",
                 "ref_variable_density"):
        getattr(L, name).argtypes = [vp]
        getattr(L, name).restype = i
    for name in ("ref_h", "ref_time", "ref_dt", "ref_lambda", "ref_calc_dt", "ref_max_u"):
        getattr(L, name).argtypes = [vp]
        getattr(L, name).restype = d
    L.ref_uinf.argtypes = [vp, dp]
    L.ref_set_uinf.argtypes = [vp, d, d]
    L.ref_set_gravity.argtypes = [vp, d, d]
    L.ref_set_threads.argtypes = [i]
    L.ref_set_threads.restype = i
    L.ref_poisson_solve.argtypes = [vp, i, i]
    L.ref_poisson_solve.restype = i
    L.ref_set_time.argtypes = [vp, d, i, d]
    L.ref_run_op.argtypes = [vp, i, d]
    L.ref_reset.argtypes = [vp]
    L.ref_get_field.argtypes = [vp, i, dp]
    L.ref_set_field.argtypes = [vp, i, dp]
    L.ref_get_shape.argtypes = [vp, i, dp]
    L.ref_get_obstacle.argtypes = [vp, i, dp]
    L.ref_get_obstacle.restype = ctypes.c_long
    L.ref_set_pose.argtypes = [vp, i, d, d, d, d, d]
    L.ref_set_shape_velocity.argtypes = [vp, i, d, d, d]
    L.ref_fish_act.argtypes = [vp, i, d, dp, i]
    L.ref_fish_act.restype = i
    L.ref_fish_period.argtypes = [vp, i]
    L.ref_fish_period.restype = d
    L.ref_fish_state.argtypes = [vp, i, i, dp]
    L.ref_fish_state.restype = i
    L.ref_profile.argtypes = [vp, ctypes.c_char_p, i, dp, i]
    L.ref_profile.restype = i
    L.ref_profile_reset.argtypes = [vp]
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def set_threads(n):
    """OpenMP threads of the reference's loops; returns the previous count."""
    return lib().ref_set_threads(n)


class RefSim:
    """One reference simulation (constant density pipeline), CLI-style args."""

    def __init__(self, args):
        self.L = lib()
        self.h_ = self.L.ref_create(args.encode())
        if not self.h_:
            raise RuntimeError("ref_create failed: " + self.L.ref_last_error().decode())
        self.nx = self.L.ref_nx(self.h_)
        self.ny = self.L.ref_ny(self.h_)
        self.h = self.L.ref_h(self.h_)

    def close(self):
        if self.h_:
            self.L.ref_destroy(self.h_)
            self.h_ = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # fields are (ny, nx) row-major arrays, x fastest
    def get(self, name):
        a = np.empty((self.ny, self.nx), dtype=np.float64)
        self.L.ref_get_field(self.h_, FIELDS[name], _dp(a))
        return a

    def set(self, name, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == (self.ny, self.nx)
        self.L.ref_set_field(self.h_, FIELDS[name], _dp(a))

    def shape(self, k=0):
        a = np.empty(len(SHAPE_FIELDS), dtype=np.float64)
        self.L.ref_get_shape(self.h_, k, _dp(a))
        return dict(zip(SHAPE_FIELDS, a.tolist()))

    def nshapes(self):
        return self.L.ref_nshapes(self.h_)

    def obstacle(self, k=0):
        """{block_index: dict(chi, dist, udef_x, udef_y, surface=array(n,5))}"""
        n = self.L.ref_get_obstacle(self.h_, k, None)
        a = np.empty(n, dtype=np.float64)
        self.L.ref_get_obstacle(self.h_, k, _dp(a))
        out, p, BS2 = {}, 0, 32 * 32
        while p < n:
            b = int(a[p]); p += 1
            rec = {}
            for key in ("chi", "dist", "udef_x", "udef_y"):
                rec[key] = a[p:p + BS2].reshape(32, 32).copy(); p += BS2
            ns = int(a[p]); p += 1
            rec["surface"] = a[p:p + 5 * ns].reshape(ns, 5).copy(); p += 5 * ns
            out[b] = rec
        return out

    @property
    def time(self):
        return self.L.ref_time(self.h_)

    @property
    def step_id(self):
        return self.L.ref_stepid(self.h_)

    @property
    def dt(self):
        return self.L.ref_dt(self.h_)

    @property
    def uinf(self):
        a = np.zeros(2)
        self.L.ref_uinf(self.h_, _dp(a))
        return a

    def set_uinf(self, ux, uy):
        self.L.ref_set_uinf(self.h_, ux, uy)

    def set_time(self, t, step, dt):
        self.L.ref_set_time(self.h_, t, step, dt)

    def calc_dt(self):
        return self.L.ref_calc_dt(self.h_)

    def max_u(self):
        return self.L.ref_max_u(self.h_)

    def advance(self):
        return self.L.ref_advance(self.h_)

    def step(self):
        """calcMaxTimestep + advance, as Simulation::simulate's loop body."""
        dt = self.calc_dt()
        self.advance()
        return dt

    def iterations(self):
        """Iterations of the last PressureIterator_unif or
        PressureVarRho_approx call (-1 without -iterativePenalization)."""
        return self.L.ref_iterations(self.h_)

    def variable_density(self):
        """SimulationData::bVariableDensity (a shape with rhoS != 1)."""
        return self.L.ref_variable_density(self.h_) == 1

    def poisson_solve(self, src="tmp", dst="pres"):
        """PoissonSolver::solve(src, dst) with a solver from makeSolver."""
        assert self.L.ref_poisson_solve(self.h_, FIELDS[src], FIELDS[dst]) == 0

    def set_gravity(self, gx, gy):
        """SimulationData::gravity, (0, -9.8) unless set."""
        self.L.ref_set_gravity(self.h_, gx, gy)

    def fish_act(self, k, t, action):
        """StefanFish::act(t, action) on shape k."""
        a = np.ascontiguousarray(action, dtype=np.float64)
        assert self.L.ref_fish_act(self.h_, k, t, _dp(a), len(a)) == 0

    def fish_period(self, k):
        return self.L.ref_fish_period(self.h_, k)

    def fish_state(self, k, other):
        """StefanFish::state(shapes[other]) of shape k."""
        out = np.zeros(32)
        n = self.L.ref_fish_state(self.h_, k, other, _dp(out))
        assert n > 0
        return out[:n]

    def set_shape_pose(self, k, com, center, orientation):
        """Shape::setCenterOfMass / center / setOrientation (as an RL driver's
        resetIC does, main_RL_leadFollow.cpp:27-41)."""
        self.L.ref_set_pose(self.h_, k, com[0], com[1], center[0], center[1], orientation)

    def set_shape_velocity(self, k, u, v, omega):
        """Shape::u, v, omega of shape k (a forced body keeps them)."""
        self.L.ref_set_shape_velocity(self.h_, k, u, v, omega)

    def run_op(self, name, dt):
        self.L.ref_run_op(self.h_, OPS[name], dt)

    def reset(self):
        self.L.ref_reset(self.h_)

    def profile(self):
        names = ctypes.create_string_buffer(4096)
        secs = np.zeros(64)
        n = self.L.ref_profile(self.h_, names, 4096, _dp(secs), 64)
        keys = names.value.decode().split(";")[:n]
        return dict(zip(keys, secs[:n].tolist()))

    def profile_reset(self):
        self.L.ref_profile_reset(self.h_)
