"""Oracle test infrastructure: a CPU restatement of the reference's timestep
pipeline in numpy (fp64), for the constant-density pipeline with disks.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it;
the product never does.  It is pinned against the reference's own code
(oracle/_ref, built from the reference's sources by oracle/Makefile) in
tests/test_oracle_cpu.py, and against the committed fixtures of
tests/golden/.

Arrays are (ny, nx) row-major fields, x fastest; block (bx, by) of the
reference is the 32x32 tile at (32 by, 32 bx).  Every expression keeps the
reference's operation order, so element-wise stages agree bit for bit with
the reference; sums do not (numpy's pairwise order differs from OpenMP's).
"""
import numpy as np
import scipy.fft

BS = 32
EPS = np.finfo(np.float64).eps


# ---- grid geometry -------------------------------------------------------

class Grid:
    """SimulationData::allocateGrid (SimulationData.cpp:17-47) with the
    Cubism uniform grid: h = extent / max(bpdx, bpdy) / 32, cell centres at
    origin + h (i + 1/2), origin = 32 b h (BlockInfo::pos)."""

    def __init__(self, bpdx, bpdy, extent=1.0):
        self.bpdx, self.bpdy = bpdx, bpdy
        self.nx, self.ny = BS * bpdx, BS * bpdy
        self.h = extent / max(bpdx * BS, bpdy * BS)
        self.extent = extent
        self.ext = (bpdx * self.h * BS, bpdy * self.h * BS)
        gx, gy = np.arange(self.nx), np.arange(self.ny)
        self.x1 = (gx // BS * BS).astype(np.float64) * self.h + self.h * ((gx % BS) + 0.5)
        self.y1 = (gy // BS * BS).astype(np.float64) * self.h + self.h * ((gy % BS) + 0.5)
        self.X, self.Y = np.meshgrid(self.x1, self.y1)

    def block_of(self, by, bx):
        return slice(by * BS, (by + 1) * BS), slice(bx * BS, (bx + 1) * BS)


def pad_zero_gradient(a):
    """BlockLabOpen ghosts at the domain edge: copy of the edge cell
    (Definitions.h:125-157); interior ghosts are neighbour cells."""
    return np.pad(a, 1, mode="edge")


# ---- Simulation::calcMaxTimestep / findMaxU ------------------------------

def find_max_u(u, v, uinf):
    """findMaxU::run, Helpers.cpp:136-176 (ZERO_TOTAL_MOM undefined)."""
    return max(np.max(np.abs(u + uinf[0])), np.max(np.abs(v + uinf[1])),
               np.max(np.abs(u)), np.max(np.abs(v)))


def calc_dt(maxU, h, nu, CFL, step, maxUbody):
    """Simulation::calcMaxTimestep, Simulation.cpp:254-277."""
    dtFourier = h * h / nu
    dtCFL = 1 if maxU < 2.2e-16 else h / maxU
    dtBody = 1 if maxUbody < 2.2e-16 else h / maxUbody
    dt = CFL * min(dtCFL, dtFourier, dtBody)
    if step < 100:
        x = (step + 1.0) / 100
        rampCFL = np.exp(np.log(1e-3) * (1 - x) + np.log(CFL) * x)
        dt = rampCFL * min(dtCFL, dtFourier, dtBody)
    return float(dt)


# ---- advDiff ---------------------------------------------------------------

def adv_diff(u, v, uinf, dt, h, nu):
    """advDiff::operator(), advDiff.cpp:36-118: explicit Euler, central
    advection + 5-point diffusion; inflow-fade ghosts; outflow correction."""
    dfac = (nu / h) * (dt / h)
    afac = -0.5 * dt / h
    norUinf = max(abs(uinf[0]), abs(uinf[1]), EPS)
    fadeW = 1 - (max(uinf[0], 0) / norUinf) ** 2 / 100
    fadeS = 1 - (max(uinf[1], 0) / norUinf) ** 2 / 100
    fadeE = 1 - (min(uinf[0], 0) / norUinf) ** 2 / 100
    fadeN = 1 - (min(uinf[1], 0) / norUinf) ** 2 / 100
    U, V = pad_zero_gradient(u), pad_zero_gradient(v)
    for A in (U, V):
        A[:, 0] *= fadeW
        A[0, :] *= fadeS
        A[:, -1] *= fadeE
        A[-1, :] *= fadeN
    ucc, vcc = U[1:-1, 1:-1], V[1:-1, 1:-1]
    upx, ulx, upy, uly = U[1:-1, 2:], U[1:-1, :-2], U[2:, 1:-1], U[:-2, 1:-1]
    vpx, vlx, vpy, vly = V[1:-1, 2:], V[1:-1, :-2], V[2:, 1:-1], V[:-2, 1:-1]
    dUadv = (ucc + uinf[0]) * (upx - ulx) + (vcc + uinf[1]) * (upy - uly)
    dUdif = upx + upy + ulx + uly - 4 * ucc
    dVadv = (ucc + uinf[0]) * (vpx - vlx) + (vcc + uinf[1]) * (vpy - vly)
    dVdif = vpx + vpy + vlx + vly - 4 * vcc
    un = ucc + (afac * dUadv + dfac * dUdif)
    vn = vcc + (afac * dVadv + dfac * dVdif)
    ny, nx = u.shape
    IF = -np.sum(un[:, 0]) + np.sum(un[:, -1]) - np.sum(vn[0, :]) + np.sum(vn[-1, :])
    corr = IF / (2 * ny + 2 * nx)
    un[:, 0] += corr
    un[:, -1] -= corr
    vn[0, :] += corr
    vn[-1, :] -= corr
    return un, vn


# ---- PressureSingle --------------------------------------------------------

def rhs_div(u, v, h, dt):
    """PressureSingle::updatePressureRHS, divergence part, PressureSingle.cpp:112-128."""
    facDiv = 0.5 * h / dt
    U, V = pad_zero_gradient(u), pad_zero_gradient(v)
    divVx = U[1:-1, 2:] - U[1:-1, :-2]
    divVy = V[2:, 1:-1] - V[:-2, 1:-1]
    return facDiv * (divVx + divVy)


def rhs_obstacles(rhs, CHI, shapes):
    """Per-shape source and perimeter correction, PressureSingle.cpp:130-213.
    shapes: list of (chi_s, mask_s) with chi_s the shape's obstacle chi on the
    grid and mask_s the cells of its obstacle blocks."""
    rhs = rhs.copy()
    C = pad_zero_gradient(CHI)
    gradXx = C[1:-1, 2:] - C[1:-1, :-2]
    gradXy = C[2:, 1:-1] - C[:-2, 1:-1]
    isPerim = gradXx * gradXx + gradXy * gradXy > 0
    sums = []
    for chi_s, mask_s in shapes:
        own = mask_s & ~(CHI > chi_s)
        srcBulk = -chi_s * rhs
        sumRHS = np.sum(srcBulk[own])
        rhs = np.where(own, rhs + srcBulk, rhs)
        pos = np.sum(np.where(own & isPerim & (rhs > 0), rhs, 0.0))
        neg = np.sum(np.where(own & isPerim & (rhs < 0), -rhs, 0.0))
        sums.append((sumRHS, pos, neg))
    for (chi_s, mask_s), (sumRHS, pos, neg) in zip(shapes, sums):
        own = mask_s & ~(CHI > chi_s)
        corrDenom = pos if sumRHS > 0 else neg
        corr = sumRHS / max(corrDenom, EPS)
        dec = own & isPerim & (rhs > 0) & (corr > 0)
        inc = own & isPerim & (rhs < 0) & (corr < 0) & ~dec
        rhs = np.where(dec, rhs - corr * rhs, np.where(inc, rhs + corr * rhs, rhs))
    return rhs


def fade_args(g, fadeLen):
    fadeLenX = fadeLenY = fadeLen * g.extent
    invFadeX, invFadeY = 1 / max(fadeLenX, EPS), 1 / max(fadeLenY, EPS)
    yt = invFadeY * np.maximum(0.0, fadeLenY - g.ext[1] + g.Y)
    yb = invFadeY * np.maximum(0.0, fadeLenY - g.Y)
    xt = invFadeX * np.maximum(0.0, fadeLenX - g.ext[0] + g.X)
    xb = invFadeX * np.maximum(0.0, fadeLenX - g.X)
    return np.minimum(np.maximum(np.maximum(yt, yb), np.maximum(xt, xb)), 1.0)


def cub2rhs(rhs, g, fadeLen=0.01):
    """PoissonSolver::cub2rhs fade with sign-matched mean correction,
    PoissonSolver.cpp:61-125."""
    fa = fade_args(g, fadeLen)
    faded = rhs * (fa * fa)
    sumRHS = np.sum(faded)
    sumPOS = max(np.sum(faded[faded > 0]), EPS)
    sumNEG = max(-np.sum(faded[faded < 0]), EPS)
    corr = sumRHS / sumPOS if sumRHS > 0 else sumRHS / sumNEG
    fadeCorrection = corr * (np.maximum(faded, 0.0) if corr > 0 else -np.minimum(faded, 0.0))
    return rhs * (1 - fa * fa) + fadeCorrection


def freespace_kernel(nx, ny, h, pad=-1):
    """FFTW_freespace constructor, FFTW_freespace.cpp:100-137: G = ln(h r)/(2 pi)
    on the (2N+pad) periodic grid, self term (1/4pi)(2 ln(h/sqrt(pi)) - 1),
    G^ = Re FFT[G] / (MX MY).  pad=-1 is the reference's 2N-1 size."""
    MX, MY = 2 * nx + pad, 2 * ny + pad
    i, j = np.arange(MX), np.arange(MY)
    xi = np.where(i >= nx, MX - i, i).astype(np.float64)
    yi = np.where(j >= ny, MY - j, j).astype(np.float64)
    XI, YI = np.meshgrid(xi, yi)
    r = np.sqrt(XI * XI + YI * YI)
    fac = 1 / (2 * np.pi)
    with np.errstate(divide="ignore"):
        G = fac * np.log(h * r)
    G[0, 0] = fac / 2 * (2 * np.log(h / np.sqrt(np.pi)) - 1)
    return np.real(np.fft.rfft2(G)) / (MX * MY)


def poisson_freespace(rhs, h, pad=-1, ghat=None):
    """FFTW_freespace::solve, FFTW_freespace.cpp:14-56 (after cub2rhs)."""
    ny, nx = rhs.shape
    MX, MY = 2 * nx + pad, 2 * ny + pad
    if ghat is None:
        ghat = freespace_kernel(nx, ny, h, pad)
    buf = np.zeros((MY, MX))
    buf[:ny, :nx] = rhs
    out = np.fft.irfft2(np.fft.rfft2(buf) * ghat, s=(MY, MX)) * (MX * MY)
    return out[:ny, :nx]


def poisson_periodic(rhs):
    """FFTW_periodic::_solve_spectral, FFTW_periodic.h:77-92."""
    ny, nx = rhs.shape
    F = np.fft.rfft2(rhs)
    kx = np.arange(nx // 2 + 1)
    j = np.arange(ny)
    ky = np.where(j <= ny // 2, j, ny - j)
    rkx, rky = kx * (2 * np.pi / nx), ky * (2 * np.pi / ny)
    RKX, RKY = np.meshgrid(rkx, rky)
    with np.errstate(divide="ignore", invalid="ignore"):     # k = 0: zeroed below
        kinv = -1 / (RKX * RKX + RKY * RKY)
        F = F * (kinv * (1.0 / (nx * ny)))
    F[0, 0] = 0
    return np.fft.irfft2(F, s=(ny, nx)) * (nx * ny)


def poisson_cosine(rhs, tol=0.1):
    """FFTW_dirichlet::_solve, FFTW_dirichlet.h:30-60: DCT-II, the blended
    finite-difference / spectral multiplier with float cosine tables, DCT-III."""
    ny, nx = rhs.shape
    F = scipy.fft.dctn(rhs, type=2)             # = FFTW REDFT10 (unnormalised)
    cx = np.cos(np.pi / nx * 2.0 * np.arange(nx)).astype(np.float32)
    cy = np.cos(np.pi / ny * 2.0 * np.arange(ny)).astype(np.float32)
    rkx = (np.arange(nx) + 0.5) * (np.pi / nx)
    rky = (np.arange(ny) + 0.5) * (np.pi / ny)
    RKX, RKY = np.meshgrid(rkx, rky)
    CX, CY = np.meshgrid(cx, cy)
    # float tables and float arithmetic, as FFTW_dirichlet.h:59 evaluates it
    denomFD = (np.float32(1) - CX / np.float32(2) - CY / np.float32(2)).astype(np.float64)
    denomSP = RKX * RKX + RKY * RKY
    norm = 0.25 / (nx * ny)
    with np.errstate(divide="ignore", invalid="ignore"):
        F = F * (-norm / ((1 - tol) * denomFD + tol * denomSP))
    F[0, 0] = 0
    return scipy.fft.idctn(F, type=2) * (4 * nx * ny)   # REDFT01 = (2n) * idct-II per axis


def pressure_correction(u, v, p, h, dt):
    """PressureSingle::pressureCorrection, PressureSingle.cpp:216-241."""
    pFac = -0.5 * dt / h
    P = pad_zero_gradient(p)
    return u + pFac * (P[1:-1, 2:] - P[1:-1, :-2]), v + pFac * (P[2:, 1:-1] - P[:-2, 1:-1])


# ---- disk obstacle ----------------------------------------------------------

def disk_blocks(g, center, radius):
    """FillBlocks_Cylinder::is_touching, ShapeLibrary.h:24-57 (bbox R + 2h)."""
    safety = 2 * g.h
    bb = ((center[0] - radius - safety, center[0] + radius + safety),
          (center[1] - radius - safety, center[1] + radius + safety))
    mask = np.zeros((g.ny, g.nx), dtype=bool)
    for by in range(g.bpdy):
        for bx in range(g.bpdx):
            mn = (g.x1[bx * BS], g.y1[by * BS])
            mx = (g.x1[bx * BS + BS - 1], g.y1[by * BS + BS - 1])
            i0 = (max(mn[0], bb[0][0]), min(mx[0], bb[0][1]))
            i1 = (max(mn[1], bb[1][0]), min(mx[1], bb[1][1]))
            if i0[1] - i0[0] > 0 and i1[1] - i1[0] > 0:
                mask[g.block_of(by, bx)] = True
    return mask


def disk_sdf(g, center, radius):
    """FillBlocks_Cylinder::operator(), ShapeLibrary.cpp:21-34."""
    x = g.X - center[0]
    y = g.Y - center[1]
    return radius - np.sqrt(x * x + y * y)


def towers_chi(g, dist, mask, sdf_grid):
    """PutObjectsOnGrid::putChiOnGrid, PutObjectsOnGrid.cpp:17-116 for one
    shape: Towers chi and the surface delta D with gradient gradU.  Inside a
    block the shape's own distance is used, across block edges the max-SDF
    grid (SDIST lab, zero-gradient at the domain edge)."""
    h = g.h
    i2h, fac = 0.5 / h, 0.5 * h
    D = np.where(mask, dist, -1.0)
    S = pad_zero_gradient(sdf_grid)
    own = pad_zero_gradient(D)
    ny, nx = dist.shape
    gx, gy = np.arange(nx), np.arange(ny)
    edgeR = ((gx % BS) == BS - 1)[None, :]
    edgeL = ((gx % BS) == 0)[None, :]
    edgeT = ((gy % BS) == BS - 1)[:, None]
    edgeB = ((gy % BS) == 0)[:, None]
    distPx = np.where(edgeR, S[1:-1, 2:], own[1:-1, 2:])
    distMx = np.where(edgeL, S[1:-1, :-2], own[1:-1, :-2])
    distPy = np.where(edgeT, S[2:, 1:-1], own[2:, 1:-1])
    distMy = np.where(edgeB, S[:-2, 1:-1], own[:-2, 1:-1])
    I = lambda a: np.where(a < 0, 0.0, a)
    gradIX, gradIY = i2h * (I(distPx) - I(distMx)), i2h * (I(distPy) - I(distMy))
    gradUX, gradUY = i2h * (distPx - distMx), i2h * (distPy - distMy)
    gradUSq = gradUX * gradUX + gradUY * gradUY
    denum = 1 / np.where(gradUSq < EPS, EPS, gradUSq)
    far = (dist > 2 * h) | (dist < -2 * h)
    X = np.where(far, np.where(dist > 0, 1.0, 0.0), (gradIX * gradUX + gradIY * gradUY) * denum)
    H = lambda a: np.where(np.abs(a) < EPS, 0.5, np.where(a < 0, 0.0, 1.0))
    gradHX, gradHY = H(distPx) - H(distMx), H(distPy) - H(distMy)
    Dv = fac * (gradHX * gradUX + gradHY * gradUY) * denum
    surf = mask & ~far & (Dv > 0)
    X = np.where(mask, X, 0.0)
    return X, np.where(surf, Dv, 0.0), np.where(surf, -Dv * gradUX, 0.0), np.where(surf, -Dv * gradUY, 0.0)


def lu_solve3(A, b):
    """3x3 Gaussian elimination with partial pivoting (Golub & Van Loan Alg.
    3.4.1), as the GSL call of Shape::updateVelocity, Shape.cpp:48-54."""
    A = [list(map(float, r)) for r in A]
    p = [0, 1, 2]
    for j in range(2):
        piv, vmax = j, abs(A[j][j])
        for i in range(j + 1, 3):
            if abs(A[i][j]) > vmax:
                vmax, piv = abs(A[i][j]), i
        if piv != j:
            A[j], A[piv] = A[piv], A[j]
            p[j], p[piv] = p[piv], p[j]
        if A[j][j] != 0.0:
            for i in range(j + 1, 3):
                lij = A[i][j] / A[j][j]
                A[i][j] = lij
                for k in range(j + 1, 3):
                    A[i][k] = A[i][k] - lij * A[j][k]
    x = [float(b[p[i]]) for i in range(3)]
    for i in range(3):
        s = x[i]
        for j in range(i):
            s = s - A[i][j] * x[j]
        x[i] = s
    for i in (2, 1, 0):
        s = x[i]
        for j in range(i + 1, 3):
            s = s - A[i][j] * x[j]
        x[i] = s / A[i][i]
    return x


class DiskState:
    """Shape state of one disk (Shape.h:22-62) with its forcing flags."""

    def __init__(self, center, radius, xvel=0.0, yvel=0.0, bForced=False, bFixed=False, rhoS=1.0):
        self.radius, self.rhoS = radius, rhoS
        self.bForcedx = self.bForcedy = bForced
        self.bBlockang = bForced
        self.bFixedx = self.bFixedy = bFixed
        self.forcedu, self.forcedv, self.forcedomega = -xvel, -yvel, -0.0
        self.timeForced = np.finfo(np.float64).max
        self.center = list(center)
        self.com = list(center)
        self.orientation = 0.0
        self.u, self.v, self.omega = self.forcedu, self.forcedv, self.forcedomega
        self.d_gm = [0.0, 0.0]
        self.M = self.J = 0.0
        self.forces = {}


def put_disk(g, S, sdf_grid_init=-1.0):
    """PutObjectsOnGrid for a single disk (PutObjectsOnGrid.cpp:186-241):
    SDF, Towers chi, CoM correction, moments (Shape::removeMoments)."""
    mask = disk_blocks(g, S.center, S.radius)
    dist = disk_sdf(g, S.center, S.radius)
    sdf_grid = np.where(mask, np.maximum(sdf_grid_init, dist), sdf_grid_init)
    X, Dsurf, sdx, sdy = towers_chi(g, dist, mask, sdf_grid)
    h = g.h
    rho = S.rhoS
    pos = X > 0
    w = rho * X * h * h
    _x = np.sum((w * (g.X - S.com[0]))[pos])
    _y = np.sum((w * (g.Y - S.com[1]))[pos])
    _m = np.sum(w[pos])
    if _m > EPS:
        S.com[0] += _x / _m
        S.com[1] += _y / _m
        S.M = _m
    hsq = h * h
    rhochi = X * rho * hsq
    p0, p1 = g.X - S.com[0], g.Y - S.com[1]
    S.M = np.sum(rhochi[pos])
    S.J = np.sum((rhochi * (p0 * p0 + p1 * p1))[pos])
    dCx, dCy = S.center[0] - S.com[0], S.center[1] - S.com[1]
    co, si = np.cos(S.orientation), np.sin(S.orientation)
    S.d_gm = [dCx * co + dCy * si, -dCx * si + dCy * co]
    return dict(mask=mask, chi=X, D=Dsurf, sdx=sdx, sdy=sdy, udx=np.zeros_like(X), udy=np.zeros_like(X))


def momenta_and_velocity(g, S, ob, u, v, dt, time):
    """PressureSingle::integrateMomenta (PressureSingle.cpp:23-67) and
    Shape::updateVelocity (Shape.cpp:25-59), disk only (no tAccel)."""
    pos = ob["chi"] > 0
    F = g.h * g.h * S.rhoS * ob["chi"]
    p0, p1 = g.X - S.com[0], g.Y - S.com[1]
    ud0, ud1 = u - ob["udx"], v - ob["udy"]
    PM = np.sum(F[pos]); PJ = np.sum((F * (p0 * p0 + p1 * p1))[pos])
    PX = np.sum((F * p0)[pos]); PY = np.sum((F * p1)[pos])
    UM = np.sum((F * ud0)[pos]); VM = np.sum((F * ud1)[pos])
    AM = np.sum((F * (p0 * ud1 - p1 * ud0))[pos])
    A = [[PM, 0, -PY], [0, PM, PX], [-PY, PX, PJ]]
    b = [UM, VM, AM]
    if S.bForcedx and time < S.timeForced:
        A[0][1] = 0; A[0][2] = 0; b[0] = PM * S.forcedu
    if S.bForcedy and time < S.timeForced:
        A[1][0] = 0; A[1][2] = 0; b[1] = PM * S.forcedv
    if S.bBlockang and time < S.timeForced:
        A[2][0] = 0; A[2][1] = 0; b[2] = PJ * S.forcedomega
    x = lu_solve3(A, b)
    if not S.bForcedy or time > S.timeForced:
        S.u = x[0]
    if not S.bForcedy or time > S.timeForced:
        S.v = x[1]
    if not S.bBlockang or time > S.timeForced:
        S.omega = x[2]


def penalize(g, S, ob, CHI, u, v):
    """PressureSingle::penalize, PressureSingle.cpp:69-108 (alpha = 1 - chi)."""
    X = ob["chi"]
    sel = ob["mask"] & ~(CHI > X) & (X > 0)
    p0, p1 = g.X - S.com[0], g.Y - S.com[1]
    alpha = 1 - X
    US = S.u - S.omega * p1 + ob["udx"]
    VS = S.v + S.omega * p0 + ob["udy"]
    return (np.where(sel, alpha * u + (1 - alpha) * US, u), np.where(sel, alpha * v + (1 - alpha) * VS, v))


def compute_forces(g, S, ob, u, v, p, nu):
    """ComputeForces::operator() and Shape::computeForces for one shape,
    ComputeForces.cpp:16-111, Shape.cpp:252-282 (17 sums + derived)."""
    NUoH = nu / g.h
    U, V = pad_zero_gradient(u), pad_zero_gradient(v)
    D11 = NUoH * (U[1:-1, 2:] - U[1:-1, :-2])
    D22 = NUoH * (V[2:, 1:-1] - V[:-2, 1:-1])
    D12 = NUoH / 2 * (U[2:, 1:-1] - U[:-2, 1:-1] + V[1:-1, 2:] - V[1:-1, :-2])
    s = ob["D"] > 0
    nX, nY = ob["sdx"], ob["sdy"]
    fXV, fXP = D11 * nX + D12 * nY, -p * nX
    fYV, fYP = D12 * nX + D22 * nY, -p * nY
    fXT, fYT = fXV + fXP, fYV + fYP
    vn = np.sqrt(S.u * S.u + S.v * S.v)
    vu = (S.u / vn, S.v / vn) if vn > 0 else (0.0, 0.0)
    Cx, Cy = S.com
    forcePar = fXT * vu[0] + fYT * vu[1]
    powOut = fXT * u + fYT * v
    powDef = fXT * ob["udx"] + fYT * ob["udy"]
    f = {
        "perimeter": np.sqrt(nX * nX + nY * nY), "forcex": fXT, "forcey": fYT,
        "forcex_P": fXP, "forcey_P": fYP, "forcex_V": fXV, "forcey_V": fYV,
        "torque": (g.X - Cx) * fYT - (g.Y - Cy) * fXT,
        "torque_P": (g.X - Cx) * fYP - (g.Y - Cy) * fXP,
        "torque_V": (g.X - Cx) * fYV - (g.Y - Cy) * fXV,
        "drag": -(.5 * (forcePar - np.abs(forcePar))), "thrust": .5 * (forcePar + np.abs(forcePar)),
        "circulation": nX * v - nY * u, "Pout": powOut, "PoutBnd": np.minimum(0, powOut),
        "defPower": powDef, "defPowerBnd": np.minimum(0, powDef),
    }
    return {k: float(np.sum(a[s])) for k, a in f.items()}


class DiskSimulation:
    """The constant-density pipeline for one disk (Simulation.cpp:175-305),
    restated: PutObjectsOnGrid, advDiff, PressureSingle, ComputeForces."""

    def __init__(self, bpdx, bpdy, extent, nu, CFL, center, radius, xvel=0.0, yvel=0.0,
                 bForced=False, bFixed=False, fadeLen=0.01, poisson="freespace"):
        self.g = Grid(bpdx, bpdy, extent)
        self.nu, self.CFL, self.fadeLen, self.poisson = nu, CFL, fadeLen, poisson
        self.S = DiskState(center, radius, xvel, yvel, bForced, bFixed)
        self.time, self.step, self.dt = 0.0, 0, 0.0
        self.uinf = [0.0, 0.0]
        g = self.g
        self.u = np.zeros((g.ny, g.nx)); self.v = np.zeros((g.ny, g.nx))
        self.p = np.zeros((g.ny, g.nx))
        self._ghat = None
        self.put_objects(0.0)
        X = self.CHI                               # ApplyObjVel, Helpers.cpp:290-307
        self.u = self.u * (1 - X) + self.ob["udx"] * X
        self.v = self.v * (1 - X) + self.ob["udy"] * X

    def put_objects(self, dt):
        S = self.S
        if S.bFixedx:
            self.uinf[0] = -S.u
        if S.bFixedy:
            self.uinf[1] = -S.v
        S.com[0] += dt * (S.u + self.uinf[0])
        S.com[1] += dt * (S.v + self.uinf[1])
        S.orientation += dt * S.omega
        co, si = np.cos(S.orientation), np.sin(S.orientation)
        S.center = [S.com[0] + co * S.d_gm[0] - si * S.d_gm[1], S.com[1] + si * S.d_gm[0] + co * S.d_gm[1]]
        self.ob = put_disk(self.g, S)
        self.CHI = np.maximum(0.0, self.ob["chi"])

    def calc_dt(self):
        maxU = find_max_u(self.u, self.v, self.uinf)
        ub = np.sqrt(self.S.u ** 2 + self.S.v ** 2)
        self.dt = calc_dt(maxU, self.g.h, self.nu, self.CFL, self.step, ub)
        return self.dt

    def pressure_single(self, dt):
        g, S = self.g, self.S
        rhs = rhs_div(self.u, self.v, g.h, dt)
        rhs = rhs_obstacles(rhs, self.CHI, [(self.ob["chi"], self.ob["mask"])])
        rhs = cub2rhs(rhs, g, self.fadeLen)
        self.rhs = rhs
        if self.poisson == "freespace":
            if self._ghat is None:
                self._ghat = freespace_kernel(g.nx, g.ny, g.h)
            self.p = poisson_freespace(rhs, g.h, ghat=self._ghat)
        elif self.poisson == "periodic":
            self.p = poisson_periodic(rhs)
        else:
            self.p = poisson_cosine(rhs)
        self.u, self.v = pressure_correction(self.u, self.v, self.p, g.h, dt)
        momenta_and_velocity(g, S, self.ob, self.u, self.v, dt, self.time)
        self.u, self.v = penalize(g, S, self.ob, self.CHI, self.u, self.v)

    def advance(self):
        dt = self.dt
        self.put_objects(dt)
        self.u, self.v = adv_diff(self.u, self.v, self.uinf, dt, self.g.h, self.nu)
        self.pressure_single(dt)
        self.S.forces = compute_forces(self.g, self.S, self.ob, self.u, self.v, self.p, self.nu)
        self.time += dt
        self.step += 1
