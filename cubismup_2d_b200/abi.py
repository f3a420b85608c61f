"""ctypes binding of libcup2d.so (include/cup2d.h) and a host-side mirror of
the reference's Simulation / Operator interface.

The reference drives its pipeline from C++ (Simulation.cpp:175-305); the
mirror below accepts the same command-line arguments (Simulation.cpp:66-104)
and shape descriptors (Simulation.cpp:106-173) and exposes the same calls:
``init()``, ``calcMaxTimestep()``, ``advance(dt)``, ``simulate()`` and the
four pipeline operators with ``operator()(dt)`` / ``getName()``.

There is no CPU fallback: if the CUDA library is missing or no GPU is
visible, creating a context raises.
"""
import ctypes
import os
import shlex

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcup2d.so")

OK, EINVAL, ECUDA, ENAN, EDOMAIN, ECAPACITY, ENOTSUP, ESTATE, ENOMEM, ETOOLARGE, ETIMEOUT = range(11)
ERRORS = {EINVAL: "EINVAL", ECUDA: "ECUDA", ENAN: "ENAN", EDOMAIN: "EDOMAIN",
          ECAPACITY: "ECAPACITY", ENOTSUP: "ENOTSUP", ESTATE: "ESTATE", ENOMEM: "ENOMEM",
          ETOOLARGE: "ETOOLARGE", ETIMEOUT: "ETIMEOUT"}
POISSON = {"freespace": 0, "periodic": 1, "": 2, "cosine": 2}
PREC_FP64, PREC_FP32 = 0, 1
FIELDS = {"u": 0, "v": 1, "chi": 2, "pres": 3, "tmp": 4, "udef_x": 5, "udef_y": 6, "sdf": 7, "invRho": 8}
SHAPE_KINDS = {"disk": 0, "stefanfish": 1, "carlingfish": 2, "envelopefish": 3}

# the exported entry points, in include/cup2d.h order
EXPORTS = [
    "cup2d_config_default", "cup2d_create", "cup2d_destroy", "cup2d_last_error",
    "cup2d_shape_params_default", "cup2d_add_shape", "cup2d_init", "cup2d_calc_dt",
    "cup2d_put_objects", "cup2d_adv_diff", "cup2d_pressure_single", "cup2d_compute_forces",
    "cup2d_end_step", "cup2d_iteration_stats", "cup2d_advance", "cup2d_sync",
    "cup2d_get_field", "cup2d_set_field",
    "cup2d_get_shape", "cup2d_set_shape", "cup2d_get_scalars", "cup2d_set_scalars",
    "cup2d_grid_size", "cup2d_kernel_launches", "cup2d_time_kernel", "cup2d_advance_timed",
    "cup2d_checkpoint_size", "cup2d_checkpoint_save", "cup2d_checkpoint_load", "cup2d_adjoint_run",
    "cup2d_ensemble_create", "cup2d_ensemble_advance", "cup2d_ensemble_advance_timed",
    "cup2d_ensemble_sync", "cup2d_ensemble_get_shapes", "cup2d_ensemble_last_error",
    "cup2d_ensemble_destroy",
    "cup2d_fish_gait_get", "cup2d_fish_gait_set", "cup2d_fish_act", "cup2d_fish_period", "cup2d_fish_state", "cup2d_dump", "cup2d_poisson_solve",
    "cup2d_tuning_get",
    "cup2d_adv_diff_noalloc",
]
KERNELS = {"advdiff": 0, "rhs_div": 1, "pcorr": 2, "fft_rows_fwd": 3, "fft_cols": 4,
           "fft_rows_inv": 5, "max_u": 6, "objects": 7, "outflow": 8}


class AdjointObjective(ctypes.Structure):
    _fields_ = [("box", ctypes.c_double * 4), ("w_energy", ctypes.c_double), ("w_force", ctypes.c_double * 2),
                ("w_body", ctypes.c_double * 3), ("w_torque", ctypes.c_double), ("gait_step", ctypes.c_double)]


class Config(ctypes.Structure):
    _fields_ = [("bpdx", ctypes.c_int), ("bpdy", ctypes.c_int), ("extent", ctypes.c_double),
                ("CFL", ctypes.c_double), ("lambda_", ctypes.c_double), ("dlm", ctypes.c_double),
                ("nu", ctypes.c_double), ("fadeLen", ctypes.c_double), ("nsteps", ctypes.c_int),
                ("tend", ctypes.c_double), ("poisson", ctypes.c_int), ("precision", ctypes.c_int),
                ("device", ctypes.c_int), ("iterative", ctypes.c_int),
                ("gravity", ctypes.c_double * 2), ("implicit_penalization", ctypes.c_int), ("autotune", ctypes.c_int)]


class ShapeParams(ctypes.Structure):
    _fields_ = [("xpos", ctypes.c_double), ("ypos", ctypes.c_double), ("angle", ctypes.c_double),
                ("rhoS", ctypes.c_double), ("bFixed", ctypes.c_int), ("bFixedx", ctypes.c_int),
                ("bFixedy", ctypes.c_int), ("bForced", ctypes.c_int), ("bForcedx", ctypes.c_int),
                ("bForcedy", ctypes.c_int), ("bBlockAng", ctypes.c_int), ("xvel", ctypes.c_double),
                ("yvel", ctypes.c_double), ("angvel", ctypes.c_double), ("timeForced", ctypes.c_double),
                ("radius", ctypes.c_double), ("tAccel", ctypes.c_double), ("L", ctypes.c_double),
                ("T", ctypes.c_double), ("phi", ctypes.c_double), ("amplitudeFactor", ctypes.c_double),
                ("pid", ctypes.c_int), ("pidpos", ctypes.c_int)]


SHAPE_STATE_FIELDS = [
    "center_x", "center_y", "com_x", "com_y", "orientation", "u", "v", "omega",
    "M", "J", "d_gm_x", "d_gm_y", "lab_com_x", "lab_com_y",
    "penalM", "penalJ", "penalDX", "penalDY", "fluidMomX", "fluidMomY", "fluidAngMom",
    "perimeter", "forcex", "forcey", "forcex_P", "forcey_P", "forcex_V", "forcey_V",
    "torque", "torque_P", "torque_V", "drag", "thrust", "circulation",
    "Pout", "PoutBnd", "defPower", "defPowerBnd", "Pthrust", "Pdrag", "EffPDef", "EffPDefBnd",
]


class Tuning(ctypes.Structure):
    _fields_ = [("fft_rows_fwd_e", ctypes.c_int), ("fft_rows_inv_e", ctypes.c_int), ("tuned", ctypes.c_int),
                ("us", ctypes.c_double * 4)]


class ShapeState(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in SHAPE_STATE_FIELDS]


_lib = None


def lib():
    """Load libcup2d.so (building it first if this tree has nvcc and no .so)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build
        _build.build()
    L = ctypes.CDLL(LIB_PATH)
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    L.cup2d_config_default.argtypes = [ctypes.POINTER(Config)]
    L.cup2d_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(vp)]
    L.cup2d_destroy.argtypes = [vp]
    L.cup2d_last_error.argtypes = [vp]
    L.cup2d_last_error.restype = ctypes.c_char_p
    L.cup2d_shape_params_default.argtypes = [ctypes.POINTER(ShapeParams)]
    L.cup2d_add_shape.argtypes = [vp, i, ctypes.POINTER(ShapeParams), ip]
    L.cup2d_init.argtypes = [vp]
    L.cup2d_calc_dt.argtypes = [vp, dp]
    for name in ("cup2d_put_objects", "cup2d_adv_diff", "cup2d_pressure_single", "cup2d_compute_forces"):
        getattr(L, name).argtypes = [vp, d]
    L.cup2d_end_step.argtypes = [vp]
    L.cup2d_iteration_stats.argtypes = [vp, ip, dp]
    L.cup2d_advance.argtypes = [vp, i]
    L.cup2d_sync.argtypes = [vp]
    L.cup2d_get_field.argtypes = [vp, i, dp]
    L.cup2d_set_field.argtypes = [vp, i, dp]
    L.cup2d_get_shape.argtypes = [vp, i, ctypes.POINTER(ShapeState)]
    L.cup2d_set_shape.argtypes = [vp, i, ctypes.POINTER(ShapeState)]
    L.cup2d_get_scalars.argtypes = [vp, dp, dp, ip, dp, dp]
    L.cup2d_set_scalars.argtypes = [vp, d, d, i, d, d]
    L.cup2d_grid_size.argtypes = [vp, ip, ip, dp]
    L.cup2d_kernel_launches.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.cup2d_time_kernel.argtypes = [vp, i, i, i, dp]
    L.cup2d_advance_timed.argtypes = [vp, i, dp]
    L.cup2d_checkpoint_size.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t)]
    L.cup2d_checkpoint_save.argtypes = [vp, vp, ctypes.c_size_t]
    L.cup2d_checkpoint_load.argtypes = [vp, vp, ctypes.c_size_t]
    L.cup2d_adjoint_run.argtypes = [vp, i, i, ctypes.POINTER(AdjointObjective), dp, dp, dp, dp, dp, dp, dp, dp]
    L.cup2d_fish_gait_get.argtypes = [vp, i, dp]
    L.cup2d_fish_gait_set.argtypes = [vp, i, dp]
    L.cup2d_ensemble_create.argtypes = [ctypes.POINTER(vp), i, ctypes.POINTER(vp)]
    L.cup2d_ensemble_advance.argtypes = [vp, i]
    L.cup2d_ensemble_advance_timed.argtypes = [vp, i, dp]
    L.cup2d_ensemble_sync.argtypes = [vp]
    L.cup2d_ensemble_get_shapes.argtypes = [vp, ctypes.POINTER(ShapeState), i, ip]
    L.cup2d_ensemble_last_error.argtypes = [vp]
    L.cup2d_ensemble_last_error.restype = ctypes.c_char_p
    L.cup2d_ensemble_destroy.argtypes = [vp]
    L.cup2d_adv_diff_noalloc.argtypes = [vp, vp, vp, vp, i, i, d, d, d, d, d, vp]
    L.cup2d_dump.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p]
    L.cup2d_poisson_solve.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.cup2d_tuning_get.argtypes = [vp, ctypes.POINTER(Tuning)]
    L.cup2d_fish_act.argtypes = [vp, i, d, dp, i]
    L.cup2d_fish_period.argtypes = [vp, i, dp]
    L.cup2d_fish_state.argtypes = [vp, i, i, dp, i]
    for name in EXPORTS:
        if name not in ("cup2d_last_error", "cup2d_ensemble_last_error"):
            getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


class Cup2DError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def _buffer(obj):
    """(pointer, bytes) of a contiguous numpy array or a device tensor."""
    if isinstance(obj, np.ndarray):
        if not obj.flags["C_CONTIGUOUS"]:
            raise ValueError("checkpoint buffers must be contiguous")
        return ctypes.c_void_p(obj.ctypes.data), obj.nbytes
    return ctypes.c_void_p(obj.data_ptr()), obj.numel() * obj.element_size()


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def parse_args(argline):
    """Simulation::parseRuntime / createShapes restated for the Python mirror.

    Returns (Config, [(kind, ShapeParams)]).  Keys are taken with or without
    their leading '-'; -bpdx/-bpdy are required (strict mode, Simulation.cpp:72-75).
    """
    toks = shlex.split(argline)
    args = {}
    k = 0
    while k < len(toks):
        t = toks[k]
        if t.startswith("-") and len(t) > 1 and not (t[1].isdigit() or t[1] == "."):
            vals = []
            k += 1
            while k < len(toks) and not (toks[k].startswith("-") and len(toks[k]) > 1 and
                                         not (toks[k][1].isdigit() or toks[k][1] == ".")):
                vals.append(toks[k]); k += 1
            args[t[1:]] = " ".join(vals)
        else:
            k += 1
    cfg = Config()
    lib().cup2d_config_default(ctypes.byref(cfg))
    if "bpdx" not in args or "bpdy" not in args:
        raise Cup2DError(EINVAL, "runtime arguments -bpdx and -bpdy are required")
    cfg.bpdx = int(args["bpdx"]); cfg.bpdy = int(args["bpdy"])
    cfg.extent = float(args.get("extent", 1))
    cfg.nsteps = int(args.get("nsteps", 0))
    cfg.tend = float(args.get("tend", 0))
    cfg.CFL = float(args.get("CFL", 0.1))
    cfg.lambda_ = float(args.get("lambda", 1e3 / cfg.CFL))
    cfg.dlm = float(args.get("dlm", 0))
    cfg.nu = float(args.get("nu", 1e-2))
    cfg.fadeLen = float(args.get("fadeLen", 0.01))
    ptype = args.get("poissonType", "")
    if ptype not in POISSON:
        raise Cup2DError(ENOTSUP, f"poissonType {ptype!r} is not available")
    cfg.poisson = POISSON[ptype]
    cfg.precision = {"fp64": PREC_FP64, "fp32": PREC_FP32}[args.get("precision", "fp64")]
    cfg.iterative = int(args.get("iterativePenalization", 0)) != 0     # Simulation.cpp:101
    # PressureSingle without EXPL_INTEGRATE_MOM (a compile-time switch there)
    cfg.implicit_penalization = int(args.get("implicitPenalization", 0)) != 0
    cfg.autotune = int(args.get("autotune", 0)) != 0       # time the transform variants at set-up
    if "gravity" in args:                  # the reference fixes it at (0, -9.8), SimulationData.h:57
        gx, gy = (float(x) for x in args["gravity"].split())
        cfg.gravity[0], cfg.gravity[1] = gx, gy
    shapes = []
    for lines in args.get("shapes", "").split("\n"):
        lines = lines.replace("_", " ")
        for line in lines.split(","):
            parts = line.split()
            if not parts or parts[0].startswith("#"):
                continue
            name = parts[0]
            if name not in SHAPE_KINDS:
                raise Cup2DError(ENOTSUP, f"shape {name!r} is not available")
            kv = {}
            for p in parts[1:]:
                if "=" in p:
                    key, val = p.split("=", 1)
                    kv[key.strip().lstrip("-")] = val.strip()
            sp = ShapeParams()
            lib().cup2d_shape_params_default(ctypes.byref(sp))
            fl = {"xpos": "xpos", "ypos": "ypos", "angle": "angle", "rhoS": "rhoS", "xvel": "xvel",
                  "yvel": "yvel", "angvel": "angvel", "timeForced": "timeForced", "radius": "radius",
                  "tAccel": "tAccel", "L": "L", "T": "T", "phi": "phi",
                  "amplitudeFactor": "amplitudeFactor"}
            for key, field in fl.items():
                if key in kv:
                    setattr(sp, field, float(kv[key]))
            for key in ("bFixed", "bFixedx", "bFixedy", "bForced", "bForcedx", "bForcedy", "bBlockAng"):
                if key in kv:
                    v = kv[key]
                    setattr(sp, key, 1 if v in ("1", "true", "True") else (0 if v in ("0", "false", "False") else int(v) != 0))
            for key in ("pid", "pidpos"):                  # StefanFish.cpp:209-211
                if key in kv:
                    setattr(sp, key, int(kv[key]) != 0)
            shapes.append((SHAPE_KINDS[name], sp))
    return cfg, shapes


class Context:
    """One device context: grid, shapes and Poisson solver (SimulationData)."""

    def __init__(self, cfg, shapes):
        self.L = lib()
        h = ctypes.c_void_p()
        rc = self.L.cup2d_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != OK:
            raise Cup2DError(rc, "cup2d_create: " + self.L.cup2d_last_error(None).decode())
        self.h_ = h
        self.cfg = cfg
        for kind, sp in shapes:
            sid = ctypes.c_int()
            self._ck(self.L.cup2d_add_shape(self.h_, kind, ctypes.byref(sp), ctypes.byref(sid)))
        nx, ny, hh = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self.L.cup2d_grid_size(self.h_, ctypes.byref(nx), ctypes.byref(ny), ctypes.byref(hh))
        self.nx, self.ny, self.h = nx.value, ny.value, hh.value
        self.nshapes = len(shapes)

    def _ck(self, rc):
        if rc != OK:
            raise Cup2DError(rc, self.L.cup2d_last_error(self.h_).decode())

    def close(self):
        if getattr(self, "h_", None):
            self.L.cup2d_destroy(self.h_)
            self.h_ = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self):
        self._ck(self.L.cup2d_init(self.h_))

    def calc_dt(self, sync=True):
        if sync:
            dt = ctypes.c_double()
            self._ck(self.L.cup2d_calc_dt(self.h_, ctypes.byref(dt)))
            return dt.value
        self._ck(self.L.cup2d_calc_dt(self.h_, None))

    def put_objects(self, dt=-1.0):
        self._ck(self.L.cup2d_put_objects(self.h_, dt))

    def adv_diff(self, dt=-1.0):
        self._ck(self.L.cup2d_adv_diff(self.h_, dt))

    def pressure_single(self, dt=-1.0):
        self._ck(self.L.cup2d_pressure_single(self.h_, dt))

    def compute_forces(self, dt=-1.0):
        self._ck(self.L.cup2d_compute_forces(self.h_, dt))

    def tuning(self):
        """The transform variants in use (values per thread of the forward and
        inverse row passes) and, with -autotune 1, the times measured (us)."""
        t = Tuning()
        self._ck(self.L.cup2d_tuning_get(self.h_, ctypes.byref(t)))
        return {"fft_rows_fwd_e": t.fft_rows_fwd_e, "fft_rows_inv_e": t.fft_rows_inv_e,
                "tuned": bool(t.tuned), "us": list(t.us)}

    def poisson_solve(self, src="tmp", dst="pres"):
        """PoissonSolver::solve(BSRC, BDST): the context's solver on field
        src into field dst (src is faded in place, as cub2rhs does)."""
        self._ck(self.L.cup2d_poisson_solve(self.h_, FIELDS[src], FIELDS[dst]))

    def end_step(self):
        self._ck(self.L.cup2d_end_step(self.h_))

    def advance(self, nsteps=1):
        self._ck(self.L.cup2d_advance(self.h_, nsteps))

    def sync(self):
        self._ck(self.L.cup2d_sync(self.h_))

    def get(self, name):
        a = np.empty((self.ny, self.nx), dtype=np.float64)
        self._ck(self.L.cup2d_get_field(self.h_, FIELDS[name], _dp(a)))
        return a

    def set(self, name, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == (self.ny, self.nx)
        self._ck(self.L.cup2d_set_field(self.h_, FIELDS[name], _dp(a)))

    def shape(self, k=0):
        s = ShapeState()
        self._ck(self.L.cup2d_get_shape(self.h_, k, ctypes.byref(s)))
        return {n: getattr(s, n) for n in SHAPE_STATE_FIELDS}

    def shape_state(self, k=0, out=None):
        """cup2d_get_shape into a cup2d_shape_state (`out`, reused when
        given), as a C or C++ caller reads it: no per-field conversion."""
        s = out if out is not None else ShapeState()
        self._ck(self.L.cup2d_get_shape(self.h_, k, ctypes.byref(s)))
        return s

    def set_shape(self, k, state):
        s = ShapeState()
        self._ck(self.L.cup2d_get_shape(self.h_, k, ctypes.byref(s)))
        for n, v in state.items():
            setattr(s, n, v)
        self._ck(self.L.cup2d_set_shape(self.h_, k, ctypes.byref(s)))

    def scalars(self):
        t, dt, ux, uy = ctypes.c_double(), ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        st = ctypes.c_int()
        self._ck(self.L.cup2d_get_scalars(self.h_, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(st),
                                          ctypes.byref(ux), ctypes.byref(uy)))
        return {"time": t.value, "dt": dt.value, "step": st.value, "uinfx": ux.value, "uinfy": uy.value}

    def set_scalars(self, time, dt, step, uinfx, uinfy):
        self._ck(self.L.cup2d_set_scalars(self.h_, time, dt, step, uinfx, uinfy))

    def time_step(self, nsteps=1):
        """cup2d_advance between CUDA events on the library's stream (ms)."""
        ms = ctypes.c_double()
        self._ck(self.L.cup2d_advance_timed(self.h_, nsteps, ctypes.byref(ms)))
        return ms.value

    def time_kernel(self, name, reps, flush_l2=True):
        """Mean ms of one launch of a pipeline kernel (CUDA events around each
        launch); with flush_l2 the L2 is flushed before every launch."""
        ms = ctypes.c_double()
        self._ck(self.L.cup2d_time_kernel(self.h_, KERNELS[name], reps, int(bool(flush_l2)), ctypes.byref(ms)))
        return ms.value

    def iteration_stats(self):
        """(iterations, last relative momentum change) of the latest iterated
        pressure call (-iterativePenalization)."""
        n, r = ctypes.c_int(), ctypes.c_double()
        self._ck(self.L.cup2d_iteration_stats(self.h_, ctypes.byref(n), ctypes.byref(r)))
        return n.value, r.value

    def checkpoint_size(self):
        n = ctypes.c_size_t()
        self._ck(self.L.cup2d_checkpoint_size(self.h_, ctypes.byref(n)))
        return n.value

    def checkpoint(self, out=None):
        """The state between steps as a uint8 array (or into ``out``: a host
        array, or any object with a device pointer ``data_ptr()`` and
        ``numel()``, e.g. a CUDA uint8 tensor)."""
        n = self.checkpoint_size()
        if out is None:
            out = np.empty(n, dtype=np.uint8)
        ptr, size = _buffer(out)
        self._ck(self.L.cup2d_checkpoint_save(self.h_, ptr, size))
        return out

    def fish_gait(self, k=0):
        """The gait parameters of curvature swimmer k: StefanFish's
        (amplitudeFactor, phi, the six scales of its curvature control
        values), or the envelope swimmer's eight Fourier coefficients of its
        curvature amplitude."""
        a = np.zeros(8, dtype=np.float64)
        self._ck(self.L.cup2d_fish_gait_get(self.h_, k, _dp(a)))
        return a

    def set_fish_gait(self, k, theta):
        a = np.ascontiguousarray(theta, dtype=np.float64)
        assert a.size == 8
        self._ck(self.L.cup2d_fish_gait_set(self.h_, k, _dp(a)))

    def adjoint(self, nsteps, box=None, every=20, dt=None, gradient=True, w_energy=1.0, w_force=(0.0, 0.0),
                w_body=(0.0, 0.0, 0.0), w_torque=0.0, gait=False, gait_step=0.0):
        """The time-averaged objective over nsteps steps from the current state,
        J = (1/nsteps) sum_n [w_energy (h^2/2) sum_box (u^2 + v^2) + w_force . force
        + w_torque |torque| + w_body . (u_b, v_b, omega)] (box = (x0, x1, y0, y1) in domain units;
        force = ComputeForces' (forcex, forcey) on the body), and its gradient
        with respect to the current velocity and to the body's velocity (u_b,
        v_b, omega: a forced body's held one, a free body's initial one) by the discrete adjoint
        (forward recomputed from checkpoints every ``every`` steps).  dt: the
        frozen step sizes (nsteps values) or None for calcMaxTimestep's.
        Returns (J, grad_u, grad_v, grad_body, dts, (forward_ms, backward_ms)),
        the gradients None when gradient is False; with gait=True (a tethered
        curvature swimmer) the times gain the placement replays' and
        grad_gait (8 values, fish_gait's order) is appended; gait_step: the
        placement's central-difference step (0: 1e-7).
        The context ends in the forward's final state."""
        dp = ctypes.POINTER(ctypes.c_double)
        obj = AdjointObjective()
        if box is not None:
            for k in range(4):
                obj.box[k] = float(box[k])
        obj.w_energy = float(w_energy) if box is not None else 0.0
        obj.w_force[0], obj.w_force[1] = float(w_force[0]), float(w_force[1])
        for k in range(3):
            obj.w_body[k] = float(w_body[k])
        obj.gait_step = float(gait_step)
        obj.w_torque = float(w_torque)
        dts = np.empty(nsteps, dtype=np.float64)
        dti = None if dt is None else np.ascontiguousarray(dt, dtype=np.float64)
        if dti is not None and dti.size != nsteps:
            raise ValueError("dt needs nsteps values")
        J = ctypes.c_double()
        ms = np.zeros(3, dtype=np.float64)
        gu = np.empty((self.ny, self.nx), dtype=np.float64) if gradient else None
        gv = np.empty((self.ny, self.nx), dtype=np.float64) if gradient else None
        gb = np.zeros(3, dtype=np.float64) if gradient else None
        gg = np.zeros(8, dtype=np.float64) if gait else None
        ptr = lambda a: None if a is None else a.ctypes.data_as(dp)  # noqa: E731
        self._ck(self.L.cup2d_adjoint_run(self.h_, nsteps, every, ctypes.byref(obj), ptr(dti), ptr(dts),
                                          ctypes.byref(J), ptr(gu), ptr(gv), ptr(gb), ptr(gg), ptr(ms)))
        if gait:
            return J.value, gu, gv, gb, dts, (float(ms[0]), float(ms[1]), float(ms[2])), gg
        return J.value, gu, gv, gb, dts, (float(ms[0]), float(ms[1]))

    def restore(self, blob):
        """Loads a checkpoint of this configuration (host array or device tensor)."""
        if isinstance(blob, (bytes, bytearray)):
            blob = np.frombuffer(blob, dtype=np.uint8)
        ptr, size = _buffer(blob)
        self._ck(self.L.cup2d_checkpoint_load(self.h_, ptr, size))

    def dump(self, directory, name):
        """SimulationData::dumpAll: velChi, pres, invRho (float32 + XDMF)."""
        self._ck(self.L.cup2d_dump(self.h_, str(directory).encode(), name.encode()))

    # ---- RL actuation (StefanFish.cpp:373-577) ----
    def fish_act(self, k, t_action, action):
        """StefanFish::act: action[0] turns the body, action[1] (optional)
        sets the tail period to Tperiod (1 + action[1]), both from t_action."""
        a = np.ascontiguousarray(action, dtype=np.float64)
        self._ck(self.L.cup2d_fish_act(self.h_, k, t_action, _dp(a), len(a)))

    def fish_period(self, k):
        """StefanFish::getLearnTPeriod."""
        p = ctypes.c_double()
        self._ck(self.L.cup2d_fish_period(self.h_, k, ctypes.byref(p)))
        return p.value

    def fish_state(self, k, other):
        """StefanFish::state(shape other): 16 values (with the head sensors)."""
        out = np.zeros(16)
        self._ck(self.L.cup2d_fish_state(self.h_, k, other, _dp(out), 16))
        return out

    def kernel_launches(self):
        n = ctypes.c_longlong()
        self._ck(self.L.cup2d_kernel_launches(self.h_, ctypes.byref(n)))
        return n.value


class Operator:
    """Operator.h:14-27: one pipeline stage, called as op(dt)."""
    name = ""
    _fn = ""

    def __init__(self, sim):
        self.sim = sim

    def __call__(self, dt):
        getattr(self.sim.ctx, self._fn)(dt)

    def getName(self):
        return self.name


class PutObjectsOnGrid(Operator):
    name, _fn = "PutObjectsOnGrid", "put_objects"


class advDiff(Operator):
    name, _fn = "advDiff", "adv_diff"


class PressureSingle(Operator):
    name, _fn = "PressureSingle", "pressure_single"


class ComputeForces(Operator):
    name, _fn = "ComputeForces", "compute_forces"


class PressureIterator_unif(Operator):
    name, _fn = "PressureIterator_unif", "pressure_single"


class advDiffGrav(Operator):
    name, _fn = "advDiffGrav", "adv_diff"


class PressureVarRho_approx(Operator):
    name, _fn = "PressureVarRho_approx", "pressure_single"


def variable_density(shape_params):
    """SimulationData::checkVariableDensity (SimulationData.cpp:122-130)."""
    return any(abs(p.rhoS - 1.0) > 2.220446049250313e-16 for _, p in shape_params)


def parse_dump_args(argline):
    """The dump options of Simulation::parseRuntime (Simulation.cpp:79-83):
    -fdump (steps between dumps), -tdump (time between dumps),
    -serialization (directory, default -file, default "./")."""
    toks = shlex.split(argline)
    out = {"fdump": 0, "tdump": 0.0, "dir": "./"}
    for i, t in enumerate(toks[:-1]):
        if t == "-fdump":
            out["fdump"] = int(toks[i + 1])
        elif t == "-tdump":
            out["tdump"] = float(toks[i + 1])
        elif t == "-file" and "-serialization" not in toks:
            out["dir"] = toks[i + 1]
        elif t == "-serialization":
            out["dir"] = toks[i + 1]
    return out


class Simulation:
    """Simulation.h:19-40 on the device pipeline."""

    def __init__(self, argline):
        self.cfg, self.shape_params = parse_args(argline)
        self.dumps = parse_dump_args(argline)
        self.next_dump_time = 0.0
        self.ctx = None
        self.pipeline = []

    def init(self):
        self.ctx = Context(self.cfg, self.shape_params)
        # Simulation.cpp:183-220 (the library routes each call by the same test)
        if variable_density(self.shape_params):
            self.pipeline = [PutObjectsOnGrid(self), advDiffGrav(self), PressureVarRho_approx(self)]
        elif self.cfg.iterative:
            self.pipeline = [PutObjectsOnGrid(self), advDiff(self), PressureIterator_unif(self)]
        else:
            self.pipeline = [PutObjectsOnGrid(self), advDiff(self), PressureSingle(self)]
        self.pipeline.append(ComputeForces(self))
        self.ctx.init()
        self.next_dump_time = 0.0
        if self.dumping():                     # Simulation.cpp:229 (only when dumps are asked for)
            self.ctx.dump(self.dumps["dir"], "IC")

    def dumping(self):
        return self.dumps["fdump"] > 0 or self.dumps["tdump"] > 0

    def bDump(self, st):  # SimulationData.cpp:179-185
        time_dump = self.dumps["tdump"] > 0 and st["time"] >= self.next_dump_time
        step_dump = self.dumps["fdump"] > 0 and st["step"] % self.dumps["fdump"] == 0
        return time_dump or step_dump

    def calcMaxTimestep(self):
        return self.ctx.calc_dt(sync=True)

    def advance(self, dt):
        dump = self.dumping() and self.bDump(self.ctx.scalars())
        for op in self.pipeline:
            op(dt)
        self.ctx.end_step()
        st = self.ctx.scalars()
        if dump:                               # Simulation.cpp:293-297
            self.next_dump_time += self.dumps["tdump"]
            self.ctx.dump(self.dumps["dir"], "avemaria_")
        return self.bOver(st)

    def bOver(self, st=None):  # SimulationData.cpp:172-177
        st = st or self.ctx.scalars()
        timeEnd = self.cfg.tend > 0 and st["time"] >= self.cfg.tend
        stepEnd = self.cfg.nsteps > 0 and st["step"] > self.cfg.nsteps
        return timeEnd or stepEnd

    def simulate(self):
        """Runs nsteps+1 steps as Simulation::simulate does: on the graph path,
        or operator by operator with -iterativePenalization."""
        if self.cfg.nsteps <= 0:
            raise Cup2DError(EINVAL, "simulate() needs -nsteps")
        if self.cfg.iterative or self.dumping():   # host decisions between steps
            for _ in range(self.cfg.nsteps + 1):
                self.advance(self.calcMaxTimestep())
        else:
            self.ctx.advance(self.cfg.nsteps + 1)
        self.ctx.sync()

    def getShapes(self):
        return [self.ctx.shape(k) for k in range(self.ctx.nshapes)]


class Ensemble:
    """Independent simulations advanced together (cup2d_ensemble_*): one CUDA
    graph holds one step of every member, so one launch advances them all.
    Each member ends bitwise where its own ``ctx.advance(n)`` would leave it;
    members stay usable on their own between ensemble advances."""

    def __init__(self, sims):
        self.L = lib()
        self.sims = list(sims)
        self.ctxs = [s.ctx for s in self.sims]     # keeps the member contexts alive
        if any(c is None or not getattr(c, "h_", None) for c in self.ctxs):
            raise Cup2DError(ESTATE, "every member needs a context")
        handles = (ctypes.c_void_p * len(self.ctxs))(*[c.h_.value for c in self.ctxs])
        h = ctypes.c_void_p()
        rc = self.L.cup2d_ensemble_create(handles, len(self.sims), ctypes.byref(h))
        if rc != OK:
            raise Cup2DError(rc, "cup2d_ensemble_create failed")
        self.h_ = h

    def _ck(self, rc):
        if rc != OK:
            raise Cup2DError(rc, self.L.cup2d_ensemble_last_error(self.h_).decode())

    def _members_current(self):
        for i, (s, c) in enumerate(zip(self.sims, self.ctxs)):
            if s.ctx is not c:
                raise Cup2DError(ESTATE, f"member {i} has a new context since the ensemble was made")

    def advance(self, nsteps=1):
        self._members_current()
        self._ck(self.L.cup2d_ensemble_advance(self.h_, nsteps))

    def advance_timed(self, nsteps=1):
        """Milliseconds of the graph launches alone (CUDA events; synchronises)."""
        self._members_current()
        ms = ctypes.c_double()
        self._ck(self.L.cup2d_ensemble_advance_timed(self.h_, nsteps, ctypes.byref(ms)))
        return ms.value

    def sync(self):
        self._ck(self.L.cup2d_ensemble_sync(self.h_))

    def shape_states(self):
        """Every member's shape states, member by member, as an (n, 42) array
        in SHAPE_STATE_FIELDS order (one wait after an ensemble advance)."""
        self._members_current()
        n = sum(c.nshapes for c in self.ctxs)
        buf = (ShapeState * max(n, 1))()
        cnt = ctypes.c_int()
        self._ck(self.L.cup2d_ensemble_get_shapes(self.h_, buf, n, ctypes.byref(cnt)))
        return np.ctypeslib.as_array(ctypes.cast(buf, ctypes.POINTER(ctypes.c_double)),
                                     shape=(n, len(SHAPE_STATE_FIELDS))).copy()

    def shapes(self):
        """shape_states() as one list of dicts per member."""
        a, out, o = self.shape_states(), [], 0
        for c in self.ctxs:
            out.append([dict(zip(SHAPE_STATE_FIELDS, a[o + k].tolist())) for k in range(c.nshapes)])
            o += c.nshapes
        return out

    def close(self):
        if getattr(self, "h_", None):
            self.L.cup2d_ensemble_destroy(self.h_)
            self.h_ = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
