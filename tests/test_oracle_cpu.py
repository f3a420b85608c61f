"""CPU tests of the oracle (test infrastructure; no GPU needed).

1. Known-answer tests of the project-written stand-ins the reference is
   compiled against (oracle/shim): the FFTW-API FFT and DCTs against
   numpy/scipy, the GSL 3x3 LU against numpy.
2. The reference compiled from its own sources (oracle/_ref) reproduces the
   committed golden fixtures of tests/golden (made by make_golden.py).
3. The numpy restatement (oracle/cup2d_oracle.py) reproduces the disk
   fixtures: element-wise stages follow the reference's operation order, sums
   and FFTs do not (numpy's pairwise sums, scipy's FFT), so the bar is
   rounding-level agreement, stated per quantity below.
"""
import ctypes
import os

import numpy as np
import pytest
import scipy.fft

from oracle import cup2d_oracle as O
from cubismup_2d_b200.synthetic import noise_field

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DISK_CASES = {
    # fixture: DiskSimulation arguments (the same configuration as make_golden.py)
    "disk_forced_freespace": dict(bpdx=2, bpdy=1, extent=1.0, nu=1e-3, CFL=0.1, center=(0.3, 0.25),
                                  radius=0.1, xvel=0.2, bForced=True, bFixed=True, poisson="freespace"),
    "disk_free_periodic": dict(bpdx=2, bpdy=1, extent=1.0, nu=1e-3, CFL=0.1, center=(0.4, 0.22),
                               radius=0.08, xvel=0.1, yvel=0.05, poisson="periodic"),
    "disk_free_cosine": dict(bpdx=2, bpdy=1, extent=1.0, nu=1e-3, CFL=0.1, center=(0.4, 0.22),
                             radius=0.08, xvel=0.1, yvel=0.05, poisson="cosine"),
}


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = {k: z[k] for k in z.files}
    d["shape"] = dict(zip(d["shape_keys"].tolist(), d["shape_values"].tolist()))
    return d


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@pytest.fixture(scope="module")
def kat(ref):
    L = ref.lib()
    for f in ("kat_dft_r2c_2d", "kat_dft_c2r_2d"):
        getattr(L, f).argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    L.kat_r2r_2d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    L.kat_lu_solve3.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return L


# ---- 1. stand-ins: known answers ---------------------------------------------

@pytest.mark.parametrize("n0,n1", [(8, 8), (7, 9), (12, 10), (31, 33), (63, 127)])
def test_shim_fft_r2c_c2r(kat, n0, n1):
    rng = np.random.default_rng(n0 * 1000 + n1)
    x = rng.standard_normal((n0, n1))
    X = np.empty((n0, n1 // 2 + 1), dtype=np.complex128)
    kat.kat_dft_r2c_2d(n0, n1, x.ctypes.data, X.ctypes.data)
    assert rel(X, np.fft.rfft2(x)) < 1e-13
    y = np.empty((n0, n1))
    kat.kat_dft_c2r_2d(n0, n1, X.ctypes.data, y.ctypes.data)
    assert rel(y / (n0 * n1), x) < 1e-13                     # FFTW's unnormalised inverse


@pytest.mark.parametrize("n0,n1", [(8, 8), (6, 10), (32, 64), (31, 17)])
def test_shim_dct(kat, n0, n1):
    rng = np.random.default_rng(n0 + 7 * n1)
    x = rng.standard_normal((n0, n1))
    y = np.empty_like(x)
    kat.kat_r2r_2d(n0, n1, 0, x.ctypes.data, y.ctypes.data)          # REDFT10 = DCT-II
    assert rel(y, scipy.fft.dctn(x, type=2)) < 1e-13
    kat.kat_r2r_2d(n0, n1, 1, x.ctypes.data, y.ctypes.data)          # REDFT01 = DCT-III
    assert rel(y, scipy.fft.dctn(x, type=3)) < 1e-13


def test_shim_lu(kat):
    rng = np.random.default_rng(5)
    for _ in range(20):
        A = rng.standard_normal((3, 3)) + 3 * np.eye(3)
        b = rng.standard_normal(3)
        x = np.empty(3)
        assert kat.kat_lu_solve3(A.ctypes.data, b.ctypes.data, x.ctypes.data) == 0
        assert np.allclose(x, np.linalg.solve(A, b), rtol=1e-13, atol=1e-13)
        assert np.allclose(O.lu_solve3(A, b), np.linalg.solve(A, b), rtol=1e-13, atol=1e-13)


# ---- 2. the compiled reference reproduces the fixtures ------------------------

GOLDEN_NAMES = ["disk_forced_freespace", "disk_free_periodic", "disk_free_cosine", "stefanfish", "carlingfish"]


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_reference_reproduces_golden(ref, name):
    import sys
    sys.path.insert(0, GOLDEN)
    import make_golden
    g = load(name)
    args, nsteps, fields = make_golden.CASES[name]
    assert str(g["args"]) == args
    out = make_golden.run_case(args, nsteps, fields)
    if name.startswith("disk"):
        assert np.array_equal(out["init_chi"], g["init_chi"])        # element-wise: exact
    else:
        # the fish's midline integrals are OpenMP reductions in the reference,
        # so two runs of the same binary differ at rounding level
        assert rel(out["init_chi"], g["init_chi"]) < 1e-12
    # OpenMP reductions may sum in another order on another host: rounding level
    assert rel(out["dt"], g["dt"]) < 1e-12
    if fields:
        for f in ("u", "v", "pres", "chi"):
            assert rel(out["final_" + f], g["final_" + f]) < 1e-10, f
    sv, gv = out["shape_values"], g["shape_values"]
    # relative 1e-8, with an absolute floor for quantities at rounding level (~1e-13)
    assert np.all(np.abs(sv - gv) <= 1e-8 * np.abs(gv) + 1e-18)


# ---- 3. the numpy restatement reproduces them ---------------------------------

@pytest.mark.parametrize("name", list(DISK_CASES))
def test_numpy_oracle_matches_golden(name):
    g = load(name)
    sim = O.DiskSimulation(**DISK_CASES[name])
    assert np.array_equal(np.maximum(0.0, sim.CHI), g["init_chi"])   # Towers chi: same arithmetic
    seed = int(g["noise_seed"])
    sim.u = sim.u + noise_field(seed, 0, sim.g.ny, sim.g.nx)
    sim.v = sim.v + noise_field(seed, 1, sim.g.ny, sim.g.nx)
    dts = []
    for _ in range(int(g["nsteps"])):
        dts.append(sim.calc_dt())
        sim.advance()
    assert rel(np.array(dts), g["dt"]) < 1e-12
    assert abs(sim.time - float(g["time"])) <= 1e-12 * float(g["time"])
    # fields after the steps: FFT (scipy vs the stand-in) and sum orders differ
    assert rel(sim.u, g["final_u"]) < 1e-9
    assert rel(sim.v, g["final_v"]) < 1e-9
    assert rel(sim.p, g["final_pres"]) < 1e-8
    assert rel(np.maximum(0.0, sim.CHI), g["final_chi"]) < 1e-12
    sh = g["shape"]
    for key, mine in (("u", sim.S.u), ("v", sim.S.v), ("omega", sim.S.omega),
                      ("com_x", sim.S.com[0]), ("com_y", sim.S.com[1])):
        assert abs(mine - sh[key]) <= 1e-9 * max(abs(sh[key]), 1e-3), key
    for key in ("forcex", "forcey", "torque", "perimeter"):
        assert abs(sim.S.forces[key] - sh[key]) <= 1e-7 * max(abs(sh["forcex"]), abs(sh["forcey"])), key


def test_numpy_freespace_point_source():
    """Analytic check of the free-space solver: a unit point source gives
    ln(r)/(2 pi) away from the source (Hockney's kernel, FFTW_freespace.cpp:108-119)."""
    g = O.Grid(4, 4, 1.0)
    rhs = np.zeros((g.ny, g.nx))
    i0, j0 = g.ny // 2, g.nx // 2
    rhs[i0, j0] = 1.0
    p = O.poisson_freespace(rhs, g.h)
    r = np.hypot(g.X - g.X[i0, j0], g.Y - g.Y[i0, j0])
    far = r > 5 * g.h
    expect = np.log(r[far]) / (2 * np.pi)
    assert np.max(np.abs(p[far] - expect)) < 1e-12
