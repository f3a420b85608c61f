// The variable-density pipeline the reference runs when a body has
// rhoS != 1 and -iterativePenalization is set (Simulation.cpp:185-195):
// PutObjectsOnGrid's 1/rho blend, advDiffGrav (advDiffGrav.cpp:14-137) and
// the iterated penalization and projection of PressureVarRho_approx
// (PressureIterator_approx.cpp:81-468).  The host loop is in context.cu.
//
// Stencils follow the reference's labs: zero-gradient ghosts (the edge
// cell's value), finDiff(B) = (B[+1] - B[-1]) / 2 and the wide laplacian
// of finDiffs (a two-cell stencil); one CTA per 32x32 block, 32 x 8
// threads, 4 rows each.  Operation order as the reference writes it.
#include <cfloat>
#include <cmath>
#include "context.hpp"

namespace cup2d {

namespace {

// value of plane f at (gx + dx, gy + dy) with zero-gradient ghosts
__device__ __forceinline__ double at(const GridDesc& g, const double* __restrict__ f, int gx, int gy,
                                     int dx, int dy) {
  int x = gx + dx, y = gy + dy;
  x = x < 0 ? 0 : (x > g.nx - 1 ? g.nx - 1 : x);
  y = y < 0 ? 0 : (y > g.ny - 1 ? g.ny - 1 : y);
  return f[(size_t)y * g.nx + x];
}
__device__ __forceinline__ double fdx(const GridDesc& g, const double* f, int gx, int gy, int dy = 0) {
  return (at(g, f, gx, gy, 1, dy) - at(g, f, gx, gy, -1, dy)) / 2;
}
__device__ __forceinline__ double fdy(const GridDesc& g, const double* f, int gx, int gy, int dx = 0) {
  return (at(g, f, gx, gy, dx, 1) - at(g, f, gx, gy, dx, -1)) / 2;
}
// finDiffX of finDiffX and Y of Y (PressureIterator_approx.cpp:40-44): the
// outer differences are taken at neighbour cells, each with its own ghosts
__device__ __forceinline__ double fdx_at(const GridDesc& g, const double* f, int gx, int gy, int ox) {
  // finDiffX(B, gx + ox, gy): a lab of two ghost layers, both the edge cell
  return (at(g, f, gx, gy, ox + 1, 0) - at(g, f, gx, gy, ox - 1, 0)) / 2;
}
__device__ __forceinline__ double fdy_at(const GridDesc& g, const double* f, int gx, int gy, int oy) {
  return (at(g, f, gx, gy, 0, oy + 1) - at(g, f, gx, gy, 0, oy - 1)) / 2;
}

__global__ void k_invrho_fill(size_t n, double* invRho) {
  pdl_begin();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    invRho[i] = 1;
}

// putChiOnGrid's blend (PutObjectsOnGrid.cpp:65-73) for shape k, shapes in
// order: where the shape's chi is at least the grid's chi so far (the
// largest chi of the shapes before it, 0 if none),
// invRho = X / rho + (1 - X) invRho.
__global__ void __launch_bounds__(1024)
k_invrho_blend(GridDesc g, const DevShape* sh, int k, AllTiles T, double* invRho)
{
  pdl_begin();
  const DevShape& S = sh[k];
  const ObstTiles& t = T.t[k];
  const double rho = S.rhoTile;
  for (int s = blockIdx.x; s < S.ntiles; s += gridDim.x) {
    const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
    const int i = threadIdx.y * BS + threadIdx.x;
    const double X = t.chi[(size_t)s * BS2 + i];
    double chiSoFar = 0;
    for (int j = 0; j < k; j++) {
      const int sj = T.t[j].slot[b];
      if (sj >= 0) chiSoFar = fmax(chiSoFar, T.t[j].chi[(size_t)sj * BS2 + i]);
    }
    if (X >= chiSoFar) {
      const size_t c = (size_t)(by * BS + threadIdx.y) * g.nx + bx * BS + threadIdx.x;
      invRho[c] = X / rho + (1 - X) * invRho[c];
    }
  }
}

// advDiffGrav.cpp:42-80 for one cell: the advDiff update, then the buoyancy
// term G dt (1 - invRho); inflow-fade ghosts at the domain edge.
struct GravCoef { double afac, dfac, fadeW, fadeS, fadeE, fadeN, U0, U1, G0, G1, dt; };
__device__ __forceinline__ GravCoef grav_coef(const GridDesc& g, const Scalars* sc, const double* G) {
  GravCoef k;
  const double dt = sc->dt, h = g.h;
  k.U0 = sc->uinfx; k.U1 = sc->uinfy; k.dt = dt; k.G0 = G[0]; k.G1 = G[1];
  k.dfac = (g.nu / h) * (dt / h);
  k.afac = -0.5 * dt / h;
  const double norUinf = fmax(fmax(fabs(k.U0), fabs(k.U1)), EPSd);
  const double rW = fmax(k.U0, 0.0) / norUinf, rS = fmax(k.U1, 0.0) / norUinf;
  const double rE = fmin(k.U0, 0.0) / norUinf, rN = fmin(k.U1, 0.0) / norUinf;
  k.fadeW = 1 - rW * rW / 100; k.fadeS = 1 - rS * rS / 100;   // BC_KILL_FAC = 100
  k.fadeE = 1 - rE * rE / 100; k.fadeN = 1 - rN * rN / 100;
  return k;
}
__device__ __forceinline__ void grav_cell(const GridDesc& g, const GravCoef& k, const double* __restrict__ u,
                                          const double* __restrict__ v, const double* __restrict__ ir,
                                          int gx, int gy, double& unew, double& vnew) {
  const int nx = g.nx, ny = g.ny;
  const size_t c = (size_t)gy * nx + gx;
  const double ucc = u[c], vcc = v[c];
  double ulx, vlx, upx, vpx, uly, vly, upy, vpy;
  if (gx > 0) { ulx = u[c - 1]; vlx = v[c - 1]; } else { ulx = ucc * k.fadeW; vlx = vcc * k.fadeW; }
  if (gx < nx - 1) { upx = u[c + 1]; vpx = v[c + 1]; } else { upx = ucc * k.fadeE; vpx = vcc * k.fadeE; }
  if (gy > 0) { uly = u[c - nx]; vly = v[c - nx]; } else { uly = ucc * k.fadeS; vly = vcc * k.fadeS; }
  if (gy < ny - 1) { upy = u[c + nx]; vpy = v[c + nx]; } else { upy = ucc * k.fadeN; vpy = vcc * k.fadeN; }
  const double gravFac = k.dt * (1 - ir[c]);
  const double dUdif = upx + upy + ulx + uly - 4 * ucc;
  const double dVdif = vpx + vpy + vlx + vly - 4 * vcc;
  const double dUadv = (ucc + k.U0) * (upx - ulx) + (vcc + k.U1) * (upy - uly);
  const double dVadv = (ucc + k.U0) * (vpx - vlx) + (vcc + k.U1) * (vpy - vly);
  const double dUAdvDiff = k.afac * dUadv + k.dfac * dUdif;
  const double dVAdvDiff = k.afac * dVadv + k.dfac * dVdif;
  unew = ucc + dUAdvDiff + k.G0 * gravFac;
  vnew = vcc + dVAdvDiff + k.G1 * gravFac;
}

struct Grav { double g[2]; };

// advDiffGrav.cpp:91-122: the net and the absolute outflow of the new
// velocity over the boundary cells, formed (as k_outflow_flux does) from
// the old velocity with the update's own arithmetic; the last CTA leaves
// corr = IF / max(AF, EPS).
__global__ void __launch_bounds__(256)
k_outflow_grav(GridDesc g, Scalars* sc, Grav G, const double* __restrict__ u, const double* __restrict__ v,
               const double* __restrict__ ir, double* partials, unsigned* counter)
{
  pdl_begin();
  __shared__ double red[64];
  const GravCoef kc = grav_coef(g, sc, G.g);
  const int nx = g.nx, ny = g.ny, nitems = 2 * (nx + ny);
  double s[2] = {0, 0};                                // IF, AF
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nitems; q += gridDim.x * blockDim.x) {
    int gx, gy, comp;
    double sgn;
    if (q < ny) { gx = 0; gy = q; comp = 0; sgn = -1; }
    else if (q < 2 * ny) { gx = nx - 1; gy = q - ny; comp = 0; sgn = 1; }
    else if (q < 2 * ny + nx) { gx = q - 2 * ny; gy = 0; comp = 1; sgn = -1; }
    else { gx = q - 2 * ny - nx; gy = ny - 1; comp = 1; sgn = 1; }
    double un, vn;
    grav_cell(g, kc, u, v, ir, gx, gy, un, vn);
    const double f = comp == 0 ? un : vn;
    if (sgn < 0) s[0] -= f; else s[0] += f;
    s[1] += fabs(f);
  }
  block_sum<2>(s, red);
  if (threadIdx.x == 0) { partials[2 * blockIdx.x] = s[0]; partials[2 * blockIdx.x + 1] = s[1]; }
  if (!last_block_done(counter, gridDim.x)) return;
  double t[2] = {0.0, 0.0};
  for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
    t[0] += __ldcg(&partials[2 * i]);
    t[1] += __ldcg(&partials[2 * i + 1]);
  }
  block_sum<2>(t, red);
  if (threadIdx.x == 0) sc->outflowCorr = t[0] / fmax(t[1], EPSd);
}

// advDiffGrav.cpp:42-89, 111-122: the update, then the relative outflow
// correction of the boundary cells (u on the west / east columns, v on the
// south / north rows), V +-= corr |V|.
__global__ void __launch_bounds__(256)
k_advdiff_grav(GridDesc g, const Scalars* sc, Grav G, const double* __restrict__ u,
               const double* __restrict__ v, const double* __restrict__ ir,
               double* __restrict__ un, double* __restrict__ vn)
{
  pdl_begin();
  const GravCoef kc = grav_coef(g, sc, G.g);
  const double corr = sc->outflowCorr;
  const int nx = g.nx, ny = g.ny, gx = blockIdx.x * BS + threadIdx.x;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int gy = blockIdx.y * BS + threadIdx.y + 8 * r;
    double a, b;
    grav_cell(g, kc, u, v, ir, gx, gy, a, b);
    if (gx == 0) a += corr * fabs(a);
    if (gx == nx - 1) a -= corr * fabs(a);
    if (gy == 0) b += corr * fabs(b);
    if (gy == ny - 1) b -= corr * fabs(b);
    const size_t c = (size_t)gy * nx + gx;
    un[c] = a; vn[c] = b;
  }
}

// pressureCorrectionInit (PressureIterator_approx.cpp:81-122): the fluid
// velocity corrected by the last pressure, vPres = V + pFac dP/dx invRho,
// and the velocity RHS div V - chi div UDEF; the penalization force F = 0.
// The reference clears each block's uDef inside the loop that reads uDef
// with one ghost layer (:119), blocks in index order (x fastest): run in
// that order, a block's west and south neighbours are already cleared, so
// its ghost cells there read zero.  div UDEF follows that order (the one a
// single thread gives; with more threads the reference's result depends on
// their schedule).
__global__ void __launch_bounds__(256)
k_vr_init(GridDesc g, const Scalars* sc, const double* __restrict__ P, const double* __restrict__ u,
          const double* __restrict__ v, const double* __restrict__ udx, const double* __restrict__ udy,
          const double* __restrict__ chi, const double* __restrict__ ir, double* __restrict__ uf,
          double* __restrict__ vf, double* __restrict__ prhs, double* __restrict__ fu, double* __restrict__ fv)
{
  pdl_begin();
  const double pFac = -sc->dt / g.h;
  const int gx = blockIdx.x * BS + threadIdx.x;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int gy = blockIdx.y * BS + threadIdx.y + 8 * r;
    const size_t c = (size_t)gy * g.nx + gx;
    const double divVf = fdx(g, u, gx, gy) + fdy(g, v, gx, gy);
    const double udW = gx % BS == 0 && gx > 0 ? 0.0 : at(g, udx, gx, gy, -1, 0);
    const double udS = gy % BS == 0 && gy > 0 ? 0.0 : at(g, udy, gx, gy, 0, -1);
    const double divDef = (at(g, udx, gx, gy, 1, 0) - udW) / 2 + (at(g, udy, gx, gy, 0, 1) - udS) / 2;
    uf[c] = u[c] + pFac * fdx(g, P, gx, gy) * ir[c];
    vf[c] = v[c] + pFac * fdy(g, P, gx, gy) * ir[c];
    prhs[c] = divVf - chi[c] * divDef;
    fu[c] = 0; fv[c] = 0;
  }
}

// penalize (PressureIterator_approx.cpp:224-287) for shape k (shapes in
// order): where the shape owns chi, F = (chi / dt) (U_s - UF); per CTA the
// sums of F^2 and of its change^2 per component.
__global__ void __launch_bounds__(1024)
k_vr_penalize(GridDesc g, const Scalars* sc, const DevShape* sh, int k, ObstTiles t,
              const double* __restrict__ chig, const double* __restrict__ uf, const double* __restrict__ vf,
              double* fu, double* fv, double* part)
{
  pdl_begin();
  __shared__ double red[32 * 4];
  const DevShape& S = sh[k];
  const double lambda = 1 / sc->dt;
  double a[4] = {0, 0, 0, 0};                 // MX, MY, DMX, DMY
  for (int s = blockIdx.x; s < S.ntiles; s += gridDim.x) {
    const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
    const int ix = threadIdx.x, iy = threadIdx.y;
    const size_t o = (size_t)s * BS2 + iy * BS + ix;
    const size_t c = (size_t)(by * BS + iy) * g.nx + bx * BS + ix;
    const double X = t.chi[o];
    if (chig[c] > X) continue;
    if (X <= 0) continue;
    const double p0 = cell_x(g, bx, ix) - S.s.com[0], p1 = cell_y(g, by, iy) - S.s.com[1];
    double ux, uy;
    udef_at(t, o, S, p0, p1, ux, uy);
    const double US = S.s.u - S.s.omega * p1 + ux;
    const double VS = S.s.v + S.s.omega * p0 + uy;
    const double pFac = lambda * X;
    const double old0 = fu[c], old1 = fv[c];
    const double new0 = pFac * (US - uf[c]), new1 = pFac * (VS - vf[c]);
    fu[c] = new0; fv[c] = new1;
    a[0] += new0 * new0; a[2] += (new0 - old0) * (new0 - old0);
    a[1] += new1 * new1; a[3] += (new1 - old1) * (new1 - old1);
  }
  block_sum<4>(a, red);
  if (lin_tid() == 0) for (int q = 0; q < 4; q++) part[4 * blockIdx.x + q] = a[q];
}

// updatePressureRHS (PressureIterator_approx.cpp:289-335):
// RHS = (1 - rho0 invRho) lap(P) - rho0 (dP/dx dinvRho/dx + dP/dy dinvRho/dy)
//       + rho0 h/dt (vRHS + dt div F),
// with the fade sums of the strip blocks for the Poisson solve.
__global__ void __launch_bounds__(256)
k_vr_rhs(GridDesc g, const Scalars* sc, double rho0, const double* __restrict__ P,
         const double* __restrict__ ir, const double* __restrict__ fu, const double* __restrict__ fv,
         const double* __restrict__ prhs, double* __restrict__ rhs,
         const int* __restrict__ fadeSlot, double* __restrict__ fadePartials)
{
  pdl_begin();
  const double dt = sc->dt, facDiv = rho0 * g.h / dt;
  const int bx = blockIdx.x, by = blockIdx.y, gx = bx * BS + threadIdx.x;
  const bool touch = fade_touch(g, bx, by);
  double s[3] = {0, 0, 0};
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int iy = threadIdx.y + 8 * r, gy = by * BS + iy;
    const size_t c = (size_t)gy * g.nx + gx;
    const double lap = (fdx_at(g, P, gx, gy, 1) - fdx_at(g, P, gx, gy, -1) +
                        fdy_at(g, P, gx, gy, 1) - fdy_at(g, P, gx, gy, -1)) / 2;
    const double lapP = (1 - rho0 * ir[c]) * lap;
    const double dPdRx = fdx(g, P, gx, gy) * fdx(g, ir, gx, gy);
    const double dPdRy = fdy(g, P, gx, gy) * fdy(g, ir, gx, gy);
    const double hatPfac = lapP - rho0 * (dPdRx + dPdRy);
    const double divF = fdx(g, fu, gx, gy) + fdy(g, fv, gx, gy);
    const double b = hatPfac + facDiv * (prhs[c] + dt * divF);
    rhs[c] = b;
    if (touch) fade_accumulate(g, bx, by, threadIdx.x, iy, b, s);
  }
  if (touch) {
    __shared__ double red[96];
    block_sum<3>(s, red);
    if (lin_tid() == 0) {
      const int q = fadeSlot[bx + g.bpdx * by];
      for (int k = 0; k < 3; k++) fadePartials[3 * q + k] = s[k];
    }
  }
}

// pressureCorrection (PressureIterator_approx.cpp:124-169):
// vPres = V + pFac (dPcur/dx / rho0 + dP/dx (invRho - 1/rho0)), and per CTA
// the sums of (Pcur - P)^2 and Pcur^2; the last CTA forms
// relDP = sqrt(DP / max(EPS, NP)).  FINAL: finalizePressure (:337-376),
// V += dt F + pFac (...) instead.
template <bool FINAL>
__global__ void __launch_bounds__(256)
k_vr_pcorr(GridDesc g, Scalars* sc, double iRho0, const double* __restrict__ Pcur,
           const double* __restrict__ P, const double* __restrict__ ir, double* u, double* v,
           double* __restrict__ uf, double* __restrict__ vf, const double* __restrict__ fu,
           const double* __restrict__ fv, double* partials, unsigned* counter)
{
  pdl_begin();
  __shared__ double red[64];
  const double dt = sc->dt, pFac = -dt / g.h;
  const int gx = blockIdx.x * BS + threadIdx.x;
  double s[2] = {0, 0};
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int gy = blockIdx.y * BS + threadIdx.y + 8 * r;
    const size_t c = (size_t)gy * g.nx + gx;
    const double dUdiv = fdx(g, P, gx, gy) * (ir[c] - iRho0);
    const double dVdiv = fdy(g, P, gx, gy) * (ir[c] - iRho0);
    const double dUpre = fdx(g, Pcur, gx, gy) * iRho0;
    const double dVpre = fdy(g, Pcur, gx, gy) * iRho0;
    if (FINAL) {
      u[c] += dt * fu[c] + pFac * (dUpre + dUdiv);
      v[c] += dt * fv[c] + pFac * (dVpre + dVdiv);
    } else {
      uf[c] = u[c] + pFac * (dUpre + dUdiv);
      vf[c] = v[c] + pFac * (dVpre + dVdiv);
      const double dp = Pcur[c] - P[c];
      s[0] += dp * dp;
      s[1] += Pcur[c] * Pcur[c];
    }
  }
  if (FINAL) return;
  block_sum<2>(s, red);
  const unsigned nb = gridDim.x * gridDim.y, bid = blockIdx.x + gridDim.x * blockIdx.y;
  if (lin_tid() == 0) { partials[2 * bid] = s[0]; partials[2 * bid + 1] = s[1]; }
  if (!last_block_done(counter, nb)) return;
  double t[2] = {0, 0};
  for (unsigned i = lin_tid(); i < nb; i += 256) {
    t[0] += __ldcg(&partials[2 * i]);
    t[1] += __ldcg(&partials[2 * i + 1]);
  }
  block_sum<2>(t, red);
  if (lin_tid() == 0) sc->it.relDP = sqrt(t[0] / fmax(EPSd, t[1]));
}

inline int fill_grid(const Ctx& c) {
  int n = (int)((c.ncells() + 255) / 256);
  return n < 148 * 8 ? n : 148 * 8;
}

} // namespace

void launch_invrho(Ctx& c) {
  launch_k(k_invrho_fill, fill_grid(c), 256, 0, c.stream, c.ncells(), c.invRho);
  CUP2D_LAUNCHED(c);
  for (int k = 0; k < c.nshapes; k++) {
    launch_k(k_invrho_blend, tile_ctas(c, c.tiles[k].capacity), dim3(32, 32), 0, c.stream, c.g,
             (const DevShape*)c.dshapes, k, all_tiles(c), c.invRho);
    CUP2D_LAUNCHED(c);
  }
}

void launch_advdiff_grav(Ctx& c) {
  const Grav G{{c.cfg.gravity[0], c.cfg.gravity[1]}};
  const int items = 2 * (c.g.nx + c.g.ny);
  int grid = (items + 255) / 256;
  if (grid > c.sms) grid = c.sms;
  launch_k(k_outflow_grav, grid, 256, 0, c.stream, c.g, c.dsc, G, (const double*)c.u(), (const double*)c.v(),
           (const double*)c.invRho, c.partials, c.counters + CNT_ADV);
  CUP2D_LAUNCHED(c);
  launch_k(k_advdiff_grav, dim3(c.g.bpdx, c.g.bpdy), dim3(32, 8), 0, c.stream, c.g, (const Scalars*)c.dsc, G,
           (const double*)c.u(), (const double*)c.v(), (const double*)c.invRho, c.uo(), c.vo());
  CUP2D_LAUNCHED(c);
  c.cur = 1 - c.cur;
}

void launch_vr_init(Ctx& c) {
  launch_k(k_vr_init, dim3(c.g.bpdx, c.g.bpdy), dim3(32, 8), 0, c.stream, c.g, (const Scalars*)c.dsc,
           (const double*)c.pres, (const double*)c.u(), (const double*)c.v(), (const double*)c.udefx,
           (const double*)c.udefy, (const double*)c.chi, (const double*)c.invRho, c.ifluid[0], c.ifluid[1],
           c.prhs, c.itmp[0], c.itmp[1]);
  CUP2D_LAUNCHED(c);
}

void launch_vr_penalize(Ctx& c) {
  PenalCtas nc{};
  for (int k = 0; k < c.nshapes; k++) {
    nc.n[k] = tile_ctas(c, c.tiles[k].capacity);
    launch_k(k_vr_penalize, nc.n[k], dim3(32, 32), 0, c.stream, c.g, (const Scalars*)c.dsc,
             (const DevShape*)c.dshapes, k, c.tiles[k], (const double*)c.chi, (const double*)c.ifluid[0],
             (const double*)c.ifluid[1], c.itmp[0], c.itmp[1], shape_partials(c) + (size_t)k * shape_region(c));
    CUP2D_LAUNCHED(c);
  }
  launch_reldf(c, nc);
}

void launch_vr_rhs(Ctx& c) {
  launch_k(k_vr_rhs, dim3(c.g.bpdx, c.g.bpdy), dim3(32, 8), 0, c.stream, c.g, (const Scalars*)c.dsc, c.rho0,
           (const double*)c.pres, (const double*)c.invRho, (const double*)c.itmp[0], (const double*)c.itmp[1],
           (const double*)c.prhs, c.rhs, (const int*)c.fadeSlot, fade_partials(c));
  CUP2D_LAUNCHED(c);
}

void launch_vr_pcorr(Ctx& c, bool final_) {
  const dim3 grid(c.g.bpdx, c.g.bpdy), block(32, 8);
  const double iRho0 = 1 / c.rho0;
  if (final_)
    launch_k(k_vr_pcorr<true>, grid, block, 0, c.stream, c.g, c.dsc, iRho0, (const double*)c.rhs,
             (const double*)c.pres, (const double*)c.invRho, c.u(), c.v(), c.ifluid[0], c.ifluid[1],
             (const double*)c.itmp[0], (const double*)c.itmp[1], c.partials, c.counters + CNT_ADV);
  else
    launch_k(k_vr_pcorr<false>, grid, block, 0, c.stream, c.g, c.dsc, iRho0, (const double*)c.rhs,
             (const double*)c.pres, (const double*)c.invRho, c.u(), c.v(), c.ifluid[0], c.ifluid[1],
             (const double*)c.itmp[0], (const double*)c.itmp[1], c.partials, c.counters + CNT_ADV);
  CUP2D_LAUNCHED(c);
}

} // namespace cup2d
