// Obstacle kernels: PutObjectsOnGrid (body motion, obstacle tile lists,
// disk signed distance, Towers chi and surface delta, moment removal), the
// obstacle terms of PressureSingle (RHS source and perimeter correction,
// momentum integrals + 3x3 rigid-body solve, collisions, penalization) and
// ComputeForces.
//
// Obstacle work is sparse: each shape owns a list of touched 32x32 tiles
// (the reference's obstacleBlocks), built on the device every step in
// increasing block order.  Per-tile kernels run one CTA of 32x32 threads per
// tile, one thread per cell, so every per-cell sequence of the reference
// (including the "first writer wins" tests) is evaluated in the reference's
// order; sums are block reductions per tile followed by a fixed-order sum
// over tiles.
#include <cfloat>
#include <cmath>
#include "context.hpp"
#include "rigid_body.cuh"
#include "step_begin.cuh"
#include "fish.cuh"

namespace cup2d {

namespace {

// ---------------------------------------------------------------------------
// PutObjectsOnGrid.cpp:186-220 for the operator entry point: last step's
// tiles are reset on the grid (all CTAs), then thread 0 of CTA 0 moves the
// bodies.  The step graph runs the same work inside k_step_begin instead.
__global__ void __launch_bounds__(256)
k_obj_begin(GridDesc g, Scalars* sc, DevShape* sh, int nsh, AllTiles T, double* chi, double* sdf)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_OBJBEGIN);
  clear_old_tiles(g, sh, nsh, T.t, chi, sdf, blockIdx.x, gridDim.x);
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    sc->maxNext = 0.0;                        // the next step's findMaxU, formed by this step
    bodies_motion(g, sc, sh, nsh);
  }
}

// Fused start of a graph step: calcMaxTimestep's reduction (every CTA), the
// reset of last step's tiles (every CTA; neither reads the other's data) and,
// in the thread that formed dt, the body motion of PutObjectsOnGrid.
__global__ void __launch_bounds__(512)
k_step_begin(GridDesc g, Scalars* sc, DevShape* sh, int nsh, AllTiles T, double* chi, double* sdf,
             const double* __restrict__ u, const double* __restrict__ v, double* partials, unsigned* counter,
             PrefetchList pf)
{
  // the fish frame that follows stages its inputs from the previous step
  // while this grid runs
  pdl_launch_dependents();
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_MAXU);
  __shared__ double red[64];
  prefetch_region(pf, blockIdx.x);
  clear_old_tiles(g, sh, nsh, T.t, chi, sdf, blockIdx.x, gridDim.x);
  if (blockIdx.x == 0 && threadIdx.x == 0) sc->maxNext = 0.0;
  if (sc->dtNextValid) {
    // calcMaxTimestep was formed at the end of the previous graph step from
    // this very state (any host-side change since would have cleared the flag)
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      const double dt = sc->dtNext;
      sc->dt = dt;
      sc->maxU = sc->maxUNext;
      if (g.dlm > 0) sc->lambda = g.dlm / dt;
      bodies_motion(g, sc, sh, nsh);
    }
    return;
  }
  if (max_u_dt_cta(g, sc, sh, nsh, u, v, partials, counter, red)) bodies_motion(g, sc, sh, nsh);
}

__device__ __forceinline__ bool disk_touching(const GridDesc& g, const DevShape& S, int bx, int by) {
  // _is_touching, ShapeLibrary.h:24-36
  const double MINP0 = cell_x(g, bx, 0), MINP1 = cell_y(g, by, 0);
  const double MAXP0 = cell_x(g, bx, BS - 1), MAXP1 = cell_y(g, by, BS - 1);
  const double i00 = fmax(MINP0, S.bbox[0][0]), i01 = fmin(MAXP0, S.bbox[0][1]);
  const double i10 = fmax(MINP1, S.bbox[1][0]), i11 = fmin(MAXP1, S.bbox[1][1]);
  return i01 - i00 > 0 && i11 - i10 > 0;
}

// Obstacle tiles of the disks (_is_touching, ShapeLibrary.h:24-36): one CTA
// per shape, searching the blocks under the disk's bounding box.
__global__ void __launch_bounds__(512)
k_disk_place(GridDesc g, Scalars* sc, DevShape* sh, AllTiles T)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_DISK_PLACE);
  const int k = blockIdx.x;
  DevShape& S = sh[k];
  if (S.cfg.kind != CUP2D_SHAPE_DISK) return;
  int bx0, bx1, by0, by1;
  block_range(S.bbox[0][0], S.bbox[0][1], g.h, 0.0, bx0, bx1);
  block_range(S.bbox[1][0], S.bbox[1][1], g.h, 0.0, by0, by1);
  select_tiles(g, T.t[k], bx0, bx1, by0, by1,
               [&](int, int bx, int by) { return disk_touching(g, S, bx, by); }, &S.ntiles, &sc->status);
}

// FillBlocks_Cylinder::operator() (ShapeLibrary.cpp:21-34): dist = R - |p - c|
// on every cell of a touched block; tmp = max(tmp, dist); rho = rhoS.
__global__ void __launch_bounds__(1024)
k_raster_disk(GridDesc g, const DevShape* sh, AllTiles T, double* sdf)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_RASTER_DISK);
  const int k = blockIdx.y;
  const DevShape& S = sh[k];
  if (S.cfg.kind != CUP2D_SHAPE_DISK) return;
  const ObstTiles& t = T.t[k];
  for (int s = blockIdx.x; s < S.ntiles; s += gridDim.x) {
    const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
    const int ix = threadIdx.x, iy = threadIdx.y, i = iy * BS + ix;
    const double pos0 = S.s.center[0], pos1 = S.s.center[1];
    const double x = cell_x(g, bx, ix) - pos0, y = cell_y(g, by, iy) - pos1;
    const double dist = S.cfg.radius - sqrt(x * x + y * y);
    const size_t o = (size_t)s * BS2 + i;
    t.dist[o] = dist; t.chi[o] = 0; t.udx[o] = 0; t.udy[o] = 0;
    atomic_max_double(&sdf[(size_t)(by * BS + iy) * g.nx + bx * BS + ix], dist);
  }
}

// PutObjectsOnGrid::putChiOnGrid (PutObjectsOnGrid.cpp:17-124) and the
// moments of the CoM correction (:118-122) + Shape::removeMoments
// (Shape.cpp:117-212) in one pass over the tiles: Towers chi from the
// shape's signed distance (ghosts from the max-SDF grid), chi grid = max
// over shapes, the surface delta list, and per tile seven integrals of
// w = rho chi h^2 about the shape's CoM C before its correction:
//   J = sum w p, M = sum w, Q = sum w |p|^2, U = sum w u, V = sum w v,
//   A = sum w (p_x v - p_y u)       (p = x - C, u = udef).
// J/M is the CoM correction d of putChiOnGrid; the moments about the
// corrected CoM C + d that removeMoments integrates follow exactly in
// algebra: M, U, V unchanged, Q - 2 d.J + M |d|^2, A - d_x V + d_y U.  The
// last CTA of the shape adds the tile sums (fixed order) and finalises M,
// J, the rigid udef part (removed where udef is read, udef_at) and d_gm.
__global__ void __launch_bounds__(1024)
k_chi_moments(GridDesc g, DevShape* sh, AllTiles T, const double* __restrict__ sdfg,
              double* chig, double* partials, int partStride, unsigned* counters)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_CHI);
  __shared__ double red[32 * 7];
  __shared__ double tile[BS][BS + 1];
  const int k = blockIdx.y;
  DevShape& S = sh[k];
  const ObstTiles& t = T.t[k];
  const int nt = S.ntiles;
  double* mp = partials + (size_t)k * partStride;
  const double C0 = S.s.com[0], C1 = S.s.com[1];
  for (int s = blockIdx.x; s < S.ntiles; s += gridDim.x) {
  double I[7] = {0, 0, 0, 0, 0, 0, 0};
  {
    const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
    const int ix = threadIdx.x, iy = threadIdx.y;
    const size_t o = (size_t)s * BS2 + iy * BS + ix;
    const double sdf = t.dist[o];
    tile[iy][ix] = sdf;
    __syncthreads();
    const double h = g.h, i2h = 0.5 / h, fac = 0.5 * h;
    const int gx = bx * BS + ix, gy = by * BS + iy;
    auto G = [&](int x, int y) -> double {        // ScalarLab on tmp, zero-gradient
      x = x < 0 ? 0 : (x >= g.nx ? g.nx - 1 : x);
      y = y < 0 ? 0 : (y >= g.ny ? g.ny - 1 : y);
      return sdfg[(size_t)y * g.nx + x];
    };
    const double distPx = ix + 1 == BS ? G(gx + 1, gy) : tile[iy][ix + 1];
    const double distMx = ix == 0 ? G(gx - 1, gy) : tile[iy][ix - 1];
    const double distPy = iy + 1 == BS ? G(gx, gy + 1) : tile[iy + 1][ix];
    const double distMy = iy == 0 ? G(gx, gy - 1) : tile[iy - 1][ix];
    double X;
    if (sdf > +2 * h || sdf < -2 * h) {
      X = sdf > 0 ? 1 : 0;
    } else {
      const double IplusX = distPx < 0 ? 0 : distPx, IminuX = distMx < 0 ? 0 : distMx;
      const double IplusY = distPy < 0 ? 0 : distPy, IminuY = distMy < 0 ? 0 : distMy;
      const double gradIX = i2h * (IplusX - IminuX), gradIY = i2h * (IplusY - IminuY);
      const double gradUX = i2h * (distPx - distMx), gradUY = i2h * (distPy - distMy);
      const double gradUSq = gradUX * gradUX + gradUY * gradUY;
      const double denum = 1 / (gradUSq < EPSd ? EPSd : gradUSq);
      X = (gradIX * gradUX + gradIY * gradUY) * denum;
    }
    t.chi[o] = X;
    atomic_max_double(&chig[(size_t)gy * g.nx + gx], X);   // CHI = max over shapes (:69-73)
    if (X > 0) {
      const double p0 = cell_x(g, bx, ix) - C0, p1 = cell_y(g, by, iy) - C1;
      const double w = X * S.rhoTile * (h * h);
      const double ux = t.udx[o], uy = t.udy[o];
      I[0] = w * p0;
      I[1] = w * p1;
      I[2] = w;
      I[3] = w * (p0 * p0 + p1 * p1);
      I[4] = w * ux;
      I[5] = w * uy;
      I[6] = w * (p0 * uy - p1 * ux);
    }
    double D = 0, sdx = 0, sdy = 0;
    if (!(sdf > +2 * h || sdf < -2 * h)) {                   // :86-106 (shift = 0)
      const double HplusX = fabs(distPx) < EPSd ? 0.5 : (distPx < 0 ? 0 : 1);
      const double HminuX = fabs(distMx) < EPSd ? 0.5 : (distMx < 0 ? 0 : 1);
      const double HplusY = fabs(distPy) < EPSd ? 0.5 : (distPy < 0 ? 0 : 1);
      const double HminuY = fabs(distMy) < EPSd ? 0.5 : (distMy < 0 ? 0 : 1);
      const double gradUX = i2h * (distPx - distMx), gradUY = i2h * (distPy - distMy);
      const double gradHX = (HplusX - HminuX), gradHY = (HplusY - HminuY);
      const double gradUSq = gradUX * gradUX + gradUY * gradUY;
      const double denum = 1 / (gradUSq < EPSd ? EPSd : gradUSq);
      const double Dv = fac * (gradHX * gradUX + gradHY * gradUY) * denum;
      if (Dv > 0) { D = Dv; sdx = -Dv * gradUX; sdy = -Dv * gradUY; }  // ObstacleBlock::write
    }
    t.sD[o] = D; t.sdx[o] = sdx; t.sdy[o] = sdy;
  }
  block_sum<7>(I, red);
  if (lin_tid() == 0) for (int q = 0; q < 7; q++) mp[7 * s + q] = I[q];
  }
  if (!last_block_done(counters + k, gridDim.x)) return;
  const int tid = lin_tid();
  if (tid >= 32) return;                               // one warp finishes
  double I[7];
  warp_sum_rows<7>(mp, nt, 7, I);
  if (tid != 0 || nt == 0) return;
  const double M = I[2];
  double d0 = 0, d1 = 0;
  if (M > EPSd) {                                      // PutObjectsOnGrid.cpp:118-122
    d0 = I[0] / M; d1 = I[1] / M;
    S.s.com[0] = C0 + d0; S.s.com[1] = C1 + d1;
  }
  const double Q = I[3] - 2 * (d0 * I[0] + d1 * I[1]) + M * (d0 * d0 + d1 * d1);
  const double A = I[6] - d0 * I[5] + d1 * I[4];
  S.Iu = I[4] / M; S.Iv = I[5] / M; S.Ia = A / Q;
  S.s.M = M; S.s.J = Q;
  const double dCx = S.s.center[0] - S.s.com[0], dCy = S.s.center[1] - S.s.com[1];
  const double co = S.cosO, si = S.sinO;         // cos/sin(orientation)
  S.s.d_gm[0] = dCx * co + dCy * si;
  S.s.d_gm[1] = -dCx * si + dCy * co;
}

// PutObjectsOnGrid::putObjectVelOnGrid (PutObjectsOnGrid.cpp:149-184), used at
// reset for ApplyObjVel; one launch per shape, in shape order.
__global__ void __launch_bounds__(1024)
k_udef_grid(GridDesc g, const DevShape* sh, int k, ObstTiles t, const double* chig,
            double* udx, double* udy)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_UDEF);
  for (int s = blockIdx.x; s < sh[k].ntiles; s += gridDim.x) {
    const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
    const int ix = threadIdx.x, iy = threadIdx.y;
    const size_t o = (size_t)s * BS2 + iy * BS + ix;
    const size_t c = (size_t)(by * BS + iy) * g.nx + bx * BS + ix;
    const double X = t.chi[o];
    if (X < chig[c] || X <= 0) continue;
    const DevShape& S = sh[k];
    double u0, u1;
    udef_at(t, o, S, cell_x(g, bx, ix) - S.s.com[0], cell_y(g, by, iy) - S.s.com[1], u0, u1);
    udx[c] += u0;
    udy[c] += u1;
  }
}

// ---------------------------------------------------------------------------
// PressureSingle::updatePressureRHS, per-shape source (PressureSingle.cpp:136-168)
__global__ void __launch_bounds__(1024)
k_rhs_obst(GridDesc g, DevShape* sh, int k, ObstTiles t, const double* __restrict__ chig,
           double* rhs, double* partials, unsigned* counter)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_RHSOBST);
  __shared__ double red[32 * 3];
  DevShape& S = sh[k];
  for (int s = blockIdx.x; s < S.ntiles; s += gridDim.x) {
  double acc[3] = {0, 0, 0};   // sumRHS, posRHS, negRHS
  {
    const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
    const int ix = threadIdx.x, iy = threadIdx.y;
    const int gx = bx * BS + ix, gy = by * BS + iy;
    auto CHI = [&](int x, int y) -> double {
      x = x < 0 ? 0 : (x >= g.nx ? g.nx - 1 : x);
      y = y < 0 ? 0 : (y >= g.ny ? g.ny - 1 : y);
      return chig[(size_t)y * g.nx + x];
    };
    const double chi = t.chi[(size_t)s * BS2 + iy * BS + ix];
    if (!(CHI(gx, gy) > chi)) {
      const double gradXx = CHI(gx + 1, gy) - CHI(gx - 1, gy);
      const double gradXy = CHI(gx, gy + 1) - CHI(gx, gy - 1);
      const size_t c = (size_t)gy * g.nx + gx;
      const double tmp0 = rhs[c];
      const double srcBulk = -chi * tmp0;
      acc[0] = srcBulk;
      const double tmp = tmp0 + srcBulk;
      rhs[c] = tmp;
      const bool isPerim = gradXx * gradXx + gradXy * gradXy > 0;
      if (isPerim && tmp > 0) acc[1] = tmp;
      if (isPerim && tmp < 0) acc[2] = -tmp;
    }
  }
  block_sum<3>(acc, red);
  if (lin_tid() == 0) for (int q = 0; q < 3; q++) partials[3 * s + q] = acc[q];
  }
  if (!last_block_done(counter, gridDim.x)) return;
  if (lin_tid() >= 32) return;                           // one warp finishes
  double tot[3];
  warp_sum_rows<3>(partials, S.ntiles, 3, tot);
  if (lin_tid() == 0) {                                  // PressureSingle.cpp:185-186
    const double corrDenom = tot[0] > 0 ? tot[1] : tot[2];
    S.rhsCorr = tot[0] / fmax(corrDenom, EPSd);
  }
}

// PressureSingle.cpp:173-212: perimeter correction of the same-sign RHS.
// A tile that reaches the fade strip then rewrites its block's fade sums
// (PoissonSolver.cpp:61-100) from the final RHS.
__global__ void __launch_bounds__(1024)
k_rhs_corr(GridDesc g, const DevShape* sh, int k, ObstTiles t, const double* __restrict__ chig,
           double* rhs, const int* __restrict__ fadeSlot, double* fadePartials)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_RHSCORR);
  __shared__ double red[32 * 3];
  const DevShape& S = sh[k];
  const double corr = S.rhsCorr;
  auto CHI = [&](int x, int y) -> double {
    x = x < 0 ? 0 : (x >= g.nx ? g.nx - 1 : x);
    y = y < 0 ? 0 : (y >= g.ny ? g.ny - 1 : y);
    return chig[(size_t)y * g.nx + x];
  };
  for (int s = blockIdx.x; s < S.ntiles; s += gridDim.x) {
    const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
    const int ix = threadIdx.x, iy = threadIdx.y;
    const int gx = bx * BS + ix, gy = by * BS + iy;
    const double chi = t.chi[(size_t)s * BS2 + iy * BS + ix];
    if (!(CHI(gx, gy) > chi)) {
      const double gradXx = CHI(gx + 1, gy) - CHI(gx - 1, gy);
      const double gradXy = CHI(gx, gy + 1) - CHI(gx, gy - 1);
      const bool isPerim = gradXx * gradXx + gradXy * gradXy > 0;
      const size_t c = (size_t)gy * g.nx + gx;
      const double tmp = rhs[c];
      if (isPerim && tmp > 0 && corr > 0) rhs[c] = tmp - corr * tmp;
      else if (isPerim && tmp < 0 && corr < 0) rhs[c] = tmp + corr * tmp;
    }
    if (fade_touch(g, bx, by)) {                         // uniform over the CTA
      __syncthreads();                                   // the tile's final RHS
      double f[3] = {0, 0, 0};
      if (iy < 8)
        for (int r = 0; r < 4; r++)
          fade_accumulate(g, bx, by, ix, iy + 8 * r, rhs[(size_t)(by * BS + iy + 8 * r) * g.nx + gx], f);
      block_sum<3>(f, red);
      if (lin_tid() == 0) {
        const int q = fadeSlot[b];
        for (int k2 = 0; k2 < 3; k2++) fadePartials[3 * q + k2] = f[k2];
      }
    }
  }
}

// PressureSingle::integrateMomenta (PressureSingle.cpp:23-67) with the
// EXPL_INTEGRATE_MOM weights (:20): 7 sums per tile, then the last CTA of
// the shape runs Shape::updateVelocity.  It runs beside the pressure
// correction: the corrected velocity of each cell it reads is evaluated
// here with k_pcorr's expression (PressureSingle.cpp:216-241) from the
// pressure and the advected velocity (ui, vi).
// ITER: PressureIterator_unif::integrateMomenta (PressureIterator_unif.cpp:
// 80-135) on its fluid velocity: F = h^2 chi (no density), the velocity
// itself instead of its difference to udef, and no displacement sums.
// VARRHO: PressureVarRho_approx::integrateMomenta (PressureIterator_approx
// .cpp:171-222) on its fluid velocity (ui, vi, read as they are):
// F = h^2 rho chi, the velocity itself, displacement sums kept.
template <bool ITER, bool VARRHO = false>
__global__ void __launch_bounds__(1024)
k_momenta(GridDesc g, const Scalars* sc, DevShape* sh, AllTiles T, const double* __restrict__ p,
          const double* __restrict__ ui, const double* __restrict__ vi,
          double* parts, int partStride, unsigned* counters)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_MOMENTA);
  __shared__ double red[32 * 7];
  const int k = blockIdx.y, tid = lin_tid();
  DevShape& S = sh[k];
  const ObstTiles& t = T.t[k];
  const int nt = S.ntiles;
  double* mp = parts + (size_t)k * partStride + 10 * (size_t)t.capacity;
  for (int s = blockIdx.x; s < nt; s += gridDim.x) {
    const double Cx = S.s.com[0], Cy = S.s.com[1];
    const double hsq = g.h * g.h, rho = S.rhoTile;
    double A[7] = {0, 0, 0, 0, 0, 0, 0};   // PM, PJ, PX, PY, UM, VM, AM
    const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
    const int ix = tid % BS, iy = tid / BS;
    const size_t o = (size_t)s * BS2 + tid;
    const double chi = t.chi[o];
    if (chi > 0) {
      const int gx = bx * BS + ix, gy = by * BS + iy, nx = g.nx, ny = g.ny;
      const size_t c = (size_t)gy * nx + gx;
      double uc, vc;
      if (VARRHO) {
        uc = ui[c]; vc = vi[c];
      } else {
        const double pFac = -0.5 * sc->dt / g.h;
        const double pW = p[gx > 0 ? c - 1 : c], pE = p[gx < nx - 1 ? c + 1 : c];
        const double pS = p[gy > 0 ? c - nx : c], pN = p[gy < ny - 1 ? c + nx : c];
        uc = ui[c] + pFac * (pE - pW); vc = vi[c] + pFac * (pN - pS);
      }
      const double p0 = cell_x(g, bx, ix) - Cx, p1 = cell_y(g, by, iy) - Cy;
      double ud0 = uc, ud1 = vc;
      if (!ITER && !VARRHO) {
        double ux, uy;
        udef_at(t, o, S, p0, p1, ux, uy);
        ud0 = uc - ux; ud1 = vc - uy;
      }
      double F;
      if (ITER) F = hsq * chi;
      else if (!VARRHO && g.implicitPenal) {            // PressureSingle.cpp:39-40, 51-53
        const double Xlamdt = chi * (sc->lambda * sc->dt);
        F = hsq * rho * Xlamdt / (1 + Xlamdt);
      } else F = hsq * rho * chi;
      A[0] = F;
      A[1] = F * (p0 * p0 + p1 * p1);
      A[2] = F * p0;
      A[3] = F * p1;
      A[4] = F * ud0;
      A[5] = F * ud1;
      A[6] = F * (p0 * ud1 - p1 * ud0);
    }
    block_sum<7>(A, red);
    if (tid == 0) for (int q = 0; q < 7; q++) mp[7 * s + q] = A[q];
  }
  if (!last_block_done(counters + k, gridDim.x)) return;
  if (tid >= 32) return;                                // one warp finishes
  double A[7];
  warp_sum_rows<7>(mp, nt, 7, A);
  if (tid != 0) return;
  S.s.fluidAngMom = A[6]; S.s.fluidMomX = A[4]; S.s.fluidMomY = A[5];
  S.s.penalDX = ITER ? 0.0 : A[2]; S.s.penalDY = ITER ? 0.0 : A[3];
  S.s.penalM = A[0]; S.s.penalJ = A[1];
  shape_update_velocity(S, sc->dt, sc->time);
}

// PressureIterator_unif::penalize (PressureIterator_unif.cpp:137-187), one
// shape (shapes run in order, as the reference's inner loop visits them per
// cell): where the shape owns chi, V += (TMPV + chi (U_s - UF)) - V, with
// TMPV the velocity before the operator and UF the fluid velocity of this
// iteration.  Per CTA: the sums of V^2 and of the change^2 per component.
__global__ void __launch_bounds__(1024)
k_penalize_iter(GridDesc g, const DevShape* sh, int k, ObstTiles t, const double* __restrict__ chig,
                double* u, double* v, const double* __restrict__ tu, const double* __restrict__ tv,
                const double* __restrict__ fu, const double* __restrict__ fv, double* part)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_PENALIZE);
  __shared__ double red[32 * 4];
  const DevShape& S = sh[k];
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
    const double DFX = X * (US - fu[c]), DFY = X * (VS - fv[c]);
    const double DPX = tu[c] + DFX - u[c], DPY = tv[c] + DFY - v[c];
    const double un = u[c] + DPX, vn = v[c] + DPY;
    u[c] = un;
    v[c] = vn;
    a[0] += un * un; a[1] += vn * vn; a[2] += DPX * DPX; a[3] += DPY * DPY;
  }
  block_sum<4>(a, red);
  if (lin_tid() == 0) for (int q = 0; q < 4; q++) part[4 * blockIdx.x + q] = a[q];
}

// The relative momentum change sqrt((DMX + DMY) / (eps + MX + MY)) of all
// shapes' penalized cells (PressureIterator_unif.cpp:185-186), from the
// per-CTA sums in a fixed order.
__global__ void __launch_bounds__(256)
k_reldf(Scalars* sc, int nsh, PenalCtas nc, const double* __restrict__ parts, int partStride)
{
  pdl_begin();
  __shared__ double red[32 * 4];
  double a[4] = {0, 0, 0, 0};
  for (int k = 0; k < nsh; k++) {
    const double* pk = parts + (size_t)k * partStride;
    for (int i = threadIdx.x; i < nc.n[k]; i += blockDim.x)
      for (int q = 0; q < 4; q++) a[q] += pk[4 * i + q];
  }
  block_sum<4>(a, red);
  if (threadIdx.x == 0) sc->it.relDF = sqrt((a[2] + a[3]) / (DBL_EPSILON + a[0] + a[1]));
}

__global__ void k_set_iter_state(Scalars* sc, IterState st) { pdl_begin(); sc->it = st; }

// PressureSingle::preventCollidingObstacles (PressureSingle.cpp:243-344).
// As in the reference, shape i's overlap sums accumulate over every j != i
// before the impulses are applied once per j.
__global__ void __launch_bounds__(1024)
k_collide(GridDesc g, const Scalars* sc, DevShape* sh, int nsh, AllTiles T)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_COLLIDE);
  __shared__ double red[32 * 10];
  __shared__ double coll[MAX_SHAPES][10];
  const int tid = threadIdx.x;
  for (int i = 0; i < nsh; i++) {
    double a[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = 0; j < nsh; j++) {
      if (i == j) continue;
      const DevShape& Si = sh[i]; const DevShape& Sj = sh[j];
      const double iUl = Si.s.u, iVl = Si.s.v, iW = Si.s.omega;
      const double jUl = Sj.s.u, jVl = Sj.s.v, jW = Sj.s.omega;
      const double iCx = Si.s.com[0], iCy = Si.s.com[1], jCx = Sj.s.com[0], jCy = Sj.s.com[1];
      for (int s = 0; s < Si.ntiles; s++) {
        const int b = T.t[i].tiles[s];
        const int sj = T.t[j].slot[b];
        if (sj < 0) continue;
        const int bx = b % g.bpdx, by = b / g.bpdx, ix = tid % BS, iy = tid / BS;
        const double iChi = T.t[i].chi[(size_t)s * BS2 + tid], jChi = T.t[j].chi[(size_t)sj * BS2 + tid];
        if (iChi <= 0 || jChi <= 0) continue;
        const double p0 = cell_x(g, bx, ix), p1 = cell_y(g, by, iy);
        const double iUr = -iW * (p1 - iCy), iVr = iW * (p0 - iCx);
        const double jUr = -jW * (p1 - jCy), jVr = jW * (p0 - jCx);
        a[0] += iChi; a[1] += iChi * p0; a[2] += iChi * p1;
        double iu0, iu1, ju0, ju1;
        udef_at(T.t[i], (size_t)s * BS2 + tid, Si, p0 - iCx, p1 - iCy, iu0, iu1);
        udef_at(T.t[j], (size_t)sj * BS2 + tid, Sj, p0 - jCx, p1 - jCy, ju0, ju1);
        a[3] += iChi * (iUl + iUr + iu0);
        a[4] += iChi * (iVl + iVr + iu1);
        a[5] += jChi; a[6] += jChi * p0; a[7] += jChi * p1;
        a[8] += jChi * (jUl + jUr + ju0);
        a[9] += jChi * (jVl + jVr + ju1);
      }
    }
    block_sum<10>(a, red);
    if (tid == 0) for (int q = 0; q < 10; q++) coll[i][q] = a[q];
    __syncthreads();
  }
  if (tid != 0) return;
  const double time = sc->time;
  for (int i = 0; i < nsh; i++)
  for (int j = 0; j < nsh; j++) {
    if (i == j) continue;
    const double* cl = coll[i];
    if (cl[0] < 1 || cl[5] < 1) continue;
    const double iPX = cl[1] / cl[0], iPY = cl[2] / cl[0];
    const double iUX = cl[3] / cl[0], iUY = cl[4] / cl[0];
    const double jPX = cl[6] / cl[5], jPY = cl[7] / cl[5];
    const double jUX = cl[8] / cl[5], jUY = cl[9] / cl[5];
    const double CX = (iPX + jPX) / 2, CY = (iPY + jPY) / 2;
    const double dirX = iPX - jPX, dirY = iPY - jPY;
    const double hitVelX = jUX - iUX, hitVelY = jUY - iUY;
    const double normF = fmax(sqrt(dirX * dirX + dirY * dirY), EPSd);
    const double NX = dirX / normF, NY = dirY / normF;
    const double projVel = hitVelX * NX + hitVelY * NY;
    if (projVel <= 0) continue;
    DevShape& Si = sh[i]; const DevShape& Sj = sh[j];
    const bool iForcedX = Si.cfg.bForcedx && time < Si.cfg.timeForced;
    const bool iForcedY = Si.cfg.bForcedy && time < Si.cfg.timeForced;
    const bool iForcedA = Si.cfg.bBlockang && time < Si.cfg.timeForced;
    const bool jForcedX = Sj.cfg.bForcedx && time < Sj.cfg.timeForced;
    const bool jForcedY = Sj.cfg.bForcedy && time < Sj.cfg.timeForced;
    const double iInvMassX = iForcedX ? 0 : 1 / Si.s.M, iInvMassY = iForcedY ? 0 : 1 / Si.s.M;
    const double jInvMassX = jForcedX ? 0 : 1 / Sj.s.M, jInvMassY = jForcedY ? 0 : 1 / Sj.s.M;
    const double iInvJ = iForcedA ? 0 : 1 / Si.s.J;
    const double meanMassX = 2 / fmax(iInvMassX + jInvMassX, EPSd);
    const double meanMassY = 2 / fmax(iInvMassY + jInvMassY, EPSd);
    const double FXdt = meanMassX * projVel * NX, FYdt = meanMassY * projVel * NY;
    Si.s.u += FXdt * iInvMassX;
    Si.s.v += FYdt * iInvMassY;
    const double RcrossF = (CX - Si.s.com[0]) * FYdt - (CY - Si.s.com[1]) * FXdt;
    Si.s.omega += iInvJ * RcrossF;
  }
}

// PressureSingle::penalize (PressureSingle.cpp:69-108), alpha = 1 - chi
__global__ void __launch_bounds__(1024)
k_penalize(GridDesc g, const Scalars* sc, const DevShape* sh, int k, ObstTiles t,
           const double* __restrict__ chig, double* u, double* v)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_PENALIZE);
  const DevShape& S = sh[k];
  for (int s = blockIdx.x; s < S.ntiles; s += gridDim.x) {
    const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
    const int ix = threadIdx.x, iy = threadIdx.y;
    const size_t o = (size_t)s * BS2 + iy * BS + ix;
    const size_t c = (size_t)(by * BS + iy) * g.nx + bx * BS + ix;
    const double X = t.chi[o];
    if (chig[c] > X) continue;
    if (X <= 0) continue;
    const double p0 = cell_x(g, bx, ix) - S.s.com[0], p1 = cell_y(g, by, iy) - S.s.com[1];
    // PressureSingle.cpp:93-97: 1 / (1 + lambda dt X) without EXPL_INTEGRATE_MOM
    const double alpha = g.implicitPenal ? 1 / (1 + sc->lambda * sc->dt * X) : 1 - X;
    double ux, uy;
    udef_at(t, o, S, p0, p1, ux, uy);
    const double US = S.s.u - S.s.omega * p1 + ux;
    const double VS = S.s.v + S.s.omega * p0 + uy;
    u[c] = alpha * u[c] + (1 - alpha) * US;
    v[c] = alpha * v[c] + (1 - alpha) * VS;
  }
}

// ComputeForces::operator() (ComputeForces.cpp:16-111) + Shape::computeForces
// (Shape.cpp:252-282): per surface point traction, 17 sums per tile, then
// the fixed-order sum over tiles and the derived powers/efficiencies.
__global__ void __launch_bounds__(1024)
k_forces(GridDesc g, Scalars* sc, int maxNext, DevShape* sh, AllTiles T, const double* __restrict__ u,
         const double* __restrict__ v, const double* __restrict__ p,
         double* partials, int partStride, unsigned* counters, cup2d_shape_state* out,
         unsigned long long* seqOut, unsigned long long seqVal)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_FORCES);
  __shared__ double red[32 * NFORCE];
  const int k = blockIdx.y;
  DevShape& S = sh[k];
  const ObstTiles& t = T.t[k];
  double* part = partials + (size_t)k * partStride;
  // maxNext (graph steps): the next step's findMaxU over this shape's tiles,
  // penalized by now (the blocks outside every tile are k_pcorr<true>'s)
  const double UINF = sc->uinfx, VINF = sc->uinfy;
  double mx = 0.0;
  int bad = 0;
  for (int s = blockIdx.x; s < S.ntiles; s += gridDim.x) {
  double F[NFORCE];
#pragma unroll
  for (int q = 0; q < NFORCE; q++) F[q] = 0;
  {
    const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
    const int ix = threadIdx.x, iy = threadIdx.y;
    const size_t o = (size_t)s * BS2 + iy * BS + ix;
    if (maxNext) {
      const size_t c = (size_t)(by * BS + iy) * g.nx + bx * BS + ix;
      const double a = u[c], w = v[c];
      mx = fmax(mx, cell_speed(a, w, UINF, VINF));
      bad |= !isfinite(a) || !isfinite(w);
    }
    if (t.sD[o] > 0) {
      const int gx = bx * BS + ix, gy = by * BS + iy;
      auto I = [&](int x, int y) -> size_t {
        x = x < 0 ? 0 : (x >= g.nx ? g.nx - 1 : x);
        y = y < 0 ? 0 : (y >= g.ny ? g.ny - 1 : y);
        return (size_t)y * g.nx + x;
      };
      const double NUoH = g.nu / g.h;
      const double Cx = S.s.com[0], Cy = S.s.com[1];
      const double vel_norm = sqrt(S.s.u * S.s.u + S.s.v * S.s.v);
      const double vu0 = vel_norm > 0 ? S.s.u / vel_norm : 0.0;
      const double vu1 = vel_norm > 0 ? S.s.v / vel_norm : 0.0;
      const double p0 = cell_x(g, bx, ix), p1 = cell_y(g, by, iy);
      const double D11 = NUoH * (u[I(gx + 1, gy)] - u[I(gx - 1, gy)]);
      const double D22 = NUoH * (v[I(gx, gy + 1)] - v[I(gx, gy - 1)]);
      const double D12 = NUoH / 2 * (u[I(gx, gy + 1)] - u[I(gx, gy - 1)]
                                     + v[I(gx + 1, gy)] - v[I(gx - 1, gy)]);
      const double normX = t.sdx[o], normY = t.sdy[o];
      const double P = p[I(gx, gy)];
      const double fXV = D11 * normX + D12 * normY, fXP = -P * normX;
      const double fYV = D12 * normX + D22 * normY, fYP = -P * normY;
      const double fXT = fXV + fXP, fYT = fYV + fYP;
      const double vx = u[I(gx, gy)], vy = v[I(gx, gy)];
      double vxDef, vyDef;
      udef_at(t, o, S, p0 - Cx, p1 - Cy, vxDef, vyDef);
      F[0] = sqrt(normX * normX + normY * normY);          // perimeter
      F[1] = fXT; F[2] = fYT;                               // forcex, forcey
      F[3] = fXP; F[4] = fYP;                               // forcex_P, forcey_P
      F[5] = fXV; F[6] = fYV;                               // forcex_V, forcey_V
      F[7] = (p0 - Cx) * fYT - (p1 - Cy) * fXT;             // torque
      F[8] = (p0 - Cx) * fYP - (p1 - Cy) * fXP;             // torque_P
      F[9] = (p0 - Cx) * fYV - (p1 - Cy) * fXV;             // torque_V
      const double forcePar = fXT * vu0 + fYT * vu1;
      F[10] = -(.5 * (forcePar - fabs(forcePar)));          // drag
      F[11] = .5 * (forcePar + fabs(forcePar));             // thrust
      F[12] = normX * vy - normY * vx;                      // circulation
      const double powOut = fXT * vx + fYT * vy;
      const double powDef = fXT * vxDef + fYT * vyDef;
      F[13] = powOut;                                       // Pout
      F[14] = fmin(0.0, powOut);                            // PoutBnd
      F[15] = powDef;                                       // defPower
      F[16] = fmin(0.0, powDef);                            // defPowerBnd
    }
  }
  block_sum<NFORCE>(F, red);
  if (lin_tid() == 0) for (int q = 0; q < NFORCE; q++) part[NFORCE * s + q] = F[q];
  }
  if (maxNext) {                                       // uniform over the launch
    __shared__ double redm[32];
    mx = block_max(mx, redm);
    const int anyBad = __syncthreads_or(bad);
    if (lin_tid() == 0) {
      atomic_max_nonneg(&sc->maxNext, mx);
      if (anyBad) atomicOr(&sc->status, ST_NAN);
    }
  }
  if (!last_block_done(counters + k, gridDim.x)) return;
  if (lin_tid() >= 32) return;                          // one warp finishes
  double tot[NFORCE];
  warp_sum_rows<NFORCE>(part, S.ntiles, NFORCE, tot);
  if (lin_tid() != 0) return;
  cup2d_shape_state& st = S.s;
  st.perimeter = tot[0]; st.forcex = tot[1]; st.forcey = tot[2];
  st.forcex_P = tot[3]; st.forcey_P = tot[4]; st.forcex_V = tot[5]; st.forcey_V = tot[6];
  st.torque = tot[7]; st.torque_P = tot[8]; st.torque_V = tot[9];
  st.drag = tot[10]; st.thrust = tot[11]; st.circulation = tot[12];
  st.Pout = tot[13]; st.PoutBnd = tot[14]; st.defPower = tot[15]; st.defPowerBnd = tot[16];
  const double un = sqrt(st.u * st.u + st.v * st.v);
  st.Pthrust = st.thrust * un;
  st.Pdrag = st.drag * un;
  const double denUnb = st.Pthrust - fmin(st.defPower, 0.0);
  const double demBnd = st.Pthrust - st.defPowerBnd;
  st.EffPDef = st.Pthrust / fmax(denUnb, EPSd);
  st.EffPDefBnd = st.Pthrust / fmax(demBnd, EPSd);
  if (out) out[k] = st;                       // the final state, to mapped host memory
  signal_host(seqOut ? seqOut + k : nullptr, seqVal);
}


} // namespace

void launch_objects_begin(Ctx& c, bool midlineReady) {
  if (c.nshapes == 0) return;
  // the last step's tiles reset and the body motion first: the midline
  // reads neither (a graph step runs them side by side)
  launch_k(k_obj_begin, tile_ctas(c, c.maxCapacity), 256, 0, c.stream, 
      c.g, c.dsc, c.dshapes, c.nshapes, all_tiles(c), c.chi, c.sdf);
  CUP2D_LAUNCHED(c);
  // fish midlines at the current time (Fish.cpp:79-95) unless the previous
  // step already computed them on its side branch
  if (!midlineReady) {
    if (c.sideMidPending) {                 // formed ahead on the side stream
      cudaStreamWaitEvent(c.stream, c.evSideMid, 0);
      c.sideMidPending = false;
    }
    for (int k = 0; k < c.nshapes; k++)
      if (c.hshapes[k].cfg.kind != CUP2D_SHAPE_DISK)
        launch_fish_midline(c, k, c.stream, midline_in_step(c, k) ? 0 : 4);
  }
}

void launch_step_begin(Ctx& c) {
  int nb = (int)((c.ncells() / 2 + 511) / 512);
  if (nb > 2 * c.sms) nb = 2 * c.sms;
  PrefetchList pf{};
  auto add = [&](const void* p, size_t bytes) {
    if (p && bytes && pf.n < MAX_PREFETCH) { pf.p[pf.n] = (const char*)p; pf.bytes[pf.n] = bytes; pf.n++; }
  };
  add(c.dsc, sizeof(Scalars));
  add(c.dshapes, sizeof(DevShape) * c.nshapes);
  for (int k = 0; k < c.nshapes; k++)
    if (c.hshapes[k].cfg.kind != CUP2D_SHAPE_DISK) {
      const FishArrays& F = c.fish[k];
      add(F.pool, sizeof(double) * (27 * (size_t)F.nm + 16));
      add(F.ipIdx, sizeof(int2) * (size_t)F.nint);
    }
  launch_k(k_step_begin, nb, 512, 0, c.stream, c.g, c.dsc, c.dshapes, c.nshapes, all_tiles(c), c.chi, c.sdf,
                                         c.u(), c.v(), c.partials, c.counters + CNT_MAXU, pf);
  CUP2D_LAUNCHED(c);
}

void launch_objects_rest(Ctx& c) {
  if (c.nshapes == 0) return;
  const AllTiles T = all_tiles(c);
  const int cap = c.maxCapacity;
  bool anyDisk = false, anyFish = false;
  for (int k = 0; k < c.nshapes; k++) {
    if (c.hshapes[k].cfg.kind == CUP2D_SHAPE_DISK) anyDisk = true; else anyFish = true;
  }
  // frames, AreaSegments and the touched tiles (Fish.cpp:95-173)
  for (int k = 0; k < c.nshapes; k++)
    if (c.hshapes[k].cfg.kind != CUP2D_SHAPE_DISK) launch_fish_place(c, k);
  if (anyDisk) {
    launch_k(k_disk_place, c.nshapes, 512, 0, c.stream, c.g, c.dsc, c.dshapes, T);
    CUP2D_LAUNCHED(c);
  }
  if (c.recordPlaced) cudaEventRecord(c.evPlaced, c.stream);
  if (anyDisk) {
    launch_k(k_raster_disk, dim3(tile_ctas(c, cap), c.nshapes), dim3(32, 32), 0, c.stream, c.g, c.dshapes, T, c.sdf);
    CUP2D_LAUNCHED(c);
  }
  if (anyFish)
    for (int k = 0; k < c.nshapes; k++)
      if (c.hshapes[k].cfg.kind != CUP2D_SHAPE_DISK) launch_fish_raster(c, k);
  const int stride = (int)shape_region(c);
  launch_k(k_chi_moments, dim3(tile_ctas(c, cap), c.nshapes), dim3(32, 32), 0, c.stream, c.g, c.dshapes, T,
           (const double*)c.sdf, c.chi, shape_partials(c), stride, c.counters + CNT_MOMENTS);
  CUP2D_LAUNCHED(c);
}

void launch_objects(Ctx& c, bool midlineReady) {
  launch_objects_begin(c, midlineReady);
  launch_objects_rest(c);
}

void launch_obj_vel_on_grid(Ctx& c) {
  for (int k = 0; k < c.nshapes; k++) {
    launch_k(k_udef_grid, tile_ctas(c, c.tiles[k].capacity), dim3(32, 32), 0, c.stream, c.g, c.dshapes, k, c.tiles[k],
                                                                   c.chi, c.udefx, c.udefy);
    CUP2D_LAUNCHED(c);
  }
}

void launch_rhs_obstacles(Ctx& c) {
  for (int k = 0; k < c.nshapes; k++) {
    launch_k(k_rhs_obst, tile_ctas(c, c.tiles[k].capacity), dim3(32, 32), 0, c.stream, 
        c.g, c.dshapes, k, c.tiles[k], c.chi, c.rhs, shape_partials(c) + (size_t)k * shape_region(c),
        c.counters + CNT_RHSOBST + k);
    CUP2D_LAUNCHED(c);
  }
  for (int k = 0; k < c.nshapes; k++) {
    launch_k(k_rhs_corr, tile_ctas(c, c.tiles[k].capacity), dim3(32, 32), 0, c.stream, c.g, c.dshapes, k, c.tiles[k],
             (const double*)c.chi, c.rhs, (const int*)c.fadeSlot, fade_partials(c));
    CUP2D_LAUNCHED(c);
  }
}

void launch_momenta(Ctx& c, const double* ui, const double* vi) {
  if (c.nshapes == 0) return;
  launch_k(k_momenta<false>, dim3(tile_ctas(c, c.maxCapacity), c.nshapes), 1024, 0, c.stream, 
      c.g, c.dsc, c.dshapes, all_tiles(c), c.pres, ui, vi, shape_partials(c), (int)shape_region(c),
      c.counters + CNT_MOMENTA);
  CUP2D_LAUNCHED(c);
}

void launch_momenta_varrho(Ctx& c, const double* ui, const double* vi) {
  if (c.nshapes == 0) return;
  launch_k(k_momenta<false, true>, dim3(tile_ctas(c, c.maxCapacity), c.nshapes), 1024, 0, c.stream,
      c.g, c.dsc, c.dshapes, all_tiles(c), (const double*)nullptr, ui, vi, shape_partials(c), (int)shape_region(c),
      c.counters + CNT_MOMENTA);
  CUP2D_LAUNCHED(c);
}
void launch_momenta_iter(Ctx& c, const double* ui, const double* vi) {
  if (c.nshapes == 0) return;
  launch_k(k_momenta<true>, dim3(tile_ctas(c, c.maxCapacity), c.nshapes), 1024, 0, c.stream, 
      c.g, c.dsc, c.dshapes, all_tiles(c), c.pres, ui, vi, shape_partials(c), (int)shape_region(c),
      c.counters + CNT_MOMENTA);
  CUP2D_LAUNCHED(c);
}

// the per-CTA sums of shape k sit at the start of its partial region (free
// while the iterated operator runs: the placement's sums are consumed)
void launch_penalize_iter(Ctx& c, const double* tu, const double* tv, const double* fu, const double* fv) {
  PenalCtas nc{};
  for (int k = 0; k < c.nshapes; k++) {
    nc.n[k] = tile_ctas(c, c.tiles[k].capacity);
    launch_k(k_penalize_iter, nc.n[k], dim3(32, 32), 0, c.stream, c.g, (const DevShape*)c.dshapes, k,
             c.tiles[k], (const double*)c.chi, c.u(), c.v(), tu, tv, fu, fv,
             shape_partials(c) + (size_t)k * shape_region(c));
    CUP2D_LAUNCHED(c);
  }
  launch_reldf(c, nc);
}

void launch_reldf(Ctx& c, const PenalCtas& nc) {
  launch_k(k_reldf, 1, 256, 0, c.stream, c.dsc, c.nshapes, nc, (const double*)shape_partials(c),
           (int)shape_region(c));
  CUP2D_LAUNCHED(c);
}

void launch_set_iter_state(Ctx& c, const IterState& st) {
  launch_k(k_set_iter_state, 1, 1, 0, c.stream, c.dsc, st);
  CUP2D_LAUNCHED(c);
}

void launch_collide_penalize(Ctx& c) {
  if (c.nshapes == 0) return;
  const AllTiles T = all_tiles(c);
  if (c.nshapes > 1) {
    launch_k(k_collide, 1, 1024, 0, c.stream, c.g, c.dsc, c.dshapes, c.nshapes, T);
    CUP2D_LAUNCHED(c);
  }
  for (int k = 0; k < c.nshapes; k++) {
    launch_k(k_penalize, tile_ctas(c, c.tiles[k].capacity), dim3(32, 32), 0, c.stream, c.g,
             (const Scalars*)c.dsc, (const DevShape*)c.dshapes, k, c.tiles[k], (const double*)c.chi, c.u(), c.v());
    CUP2D_LAUNCHED(c);
  }
}

void launch_forces(Ctx& c, cup2d_shape_state* out, bool maxNext, unsigned long long* seqOut,
                   unsigned long long seqVal) {
  if (c.nshapes == 0) return;
  const AllTiles T = all_tiles(c);
  launch_k(k_forces, dim3(tile_ctas(c, c.maxCapacity), c.nshapes), dim3(32, 32), 0, c.stream,
      c.g, c.dsc, maxNext ? 1 : 0, c.dshapes, T, (const double*)c.u(), (const double*)c.v(),
      (const double*)c.pres, shape_partials(c), (int)shape_region(c), c.counters + CNT_FORCES, out,
      seqOut, seqVal);
  CUP2D_LAUNCHED(c);
}

} // namespace cup2d

#ifdef CUP2D_TRACE
namespace cup2d { void trace_bind_obstacles(unsigned long long* p) { trace_bind_this_unit(p); } }
#endif
