// Discrete adjoint of the step (no counterpart in the reference): the
// gradient of a time-averaged objective (kinetic energy in a probe box, the
// body's force, the body's velocity) with respect to the initial velocity
// field, the body's velocity and, for a tethered swimmer, its gait, for a
// body held on the grid (bFixed): a disk forced or free, or a curvature
// swimmer forced in x, y and angle (its chi moves with its gait alone).
//
// The step u^n -> u^(n+1) (operator order of Simulation::advance):
//   u1 = A(u^n)             advDiff with its inflow fades and outflow
//                           correction (advDiff.cpp:36-116)
//   T  = (h/2dt) D u1       the RHS divergence (PressureSingle.cpp:112-128)
//   f  = O(T)               the obstacle terms (PressureSingle.cpp:130-213)
//   b  = F(f)               the boundary-strip fade (PoissonSolver.cpp:61-118)
//   p  = K b                the Poisson convolution
//   u2 = u1 - (dt/2h) G p   pressureCorrection (PressureSingle.cpp:216-241)
//   U_b = A^-1 b(u2)        a free body: integrateMomenta + updateVelocity
//                           (PressureSingle.cpp:23-67, Shape.cpp:25-59)
//   u^(n+1) = Pen(u2, U_b)  penalize (PressureSingle.cpp:69-108)
//   F^n = forces(u, p)      ComputeForces (ComputeForces.cpp:16-111)
// with U_b held for a forced body.  A, O and F are nonlinear; each is
// linearized about the forward values of its step (O and F are piecewise
// linear in their input: the linearization is the active piece, with the
// rank-one terms of their sign-selected corrections).  The backward step
// applies the transposes in reverse order: Pen^T, then lambda_p = -(dt/2h)
// G^T lambda, K^T = K, F'^T, O'^T, (h/2dt) D^T added to lambda, A'^T.  The
// three solvers are symmetric: the free-space and periodic ones convolve
// with an even kernel, and the cosine one is DCT-III . diag . DCT-II, where
// the DCT-III is the DCT-II's transpose times a diagonal weight (its zero
// term's) that commutes with the multiplier.
//
// The forward is stored as checkpoints (the context's own checkpoint blob,
// kept in device memory) every `every` steps; the backward recomputes each
// segment forward from its checkpoint, keeping the values the
// linearizations need (and, for a swimmer, each step's obstacle tiles),
// then runs the segment's adjoint steps.  dt is frozen (the forward's
// schedule, or one given): it is not differentiated.  The gait gradient
// contracts each step's sensitivity to the body's geometry with central
// differences of the placement (see k_adj_geo_pen).
#include <algorithm>
#include <array>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <string>
#include <thread>
#include <vector>
#include "context.hpp"
#include "rigid_body.cuh"

namespace cup2d {

namespace {

// zero-gradient neighbour indices (the labs' clamped ghosts)
struct Nb { size_t c, W, E, S, N; int x, y; };
__device__ __forceinline__ Nb nb_of(const GridDesc& g, int gx, int gy) {
  Nb n;
  n.x = gx; n.y = gy;
  n.c = (size_t)gy * g.nx + gx;
  n.W = gx > 0 ? n.c - 1 : n.c;
  n.E = gx < g.nx - 1 ? n.c + 1 : n.c;
  n.S = gy > 0 ? n.c - g.nx : n.c;
  n.N = gy < g.ny - 1 ? n.c + g.nx : n.c;
  return n;
}

// transpose of q -> fac (q[E] - q[W]) (x) and fac (q[N] - q[S]) (y) with
// clamped ghosts, evaluated at cell j: the cells whose E / W / N / S
// neighbour is j
__device__ __forceinline__ double diff_T(const GridDesc& g, const double* __restrict__ lx,
                                         const double* __restrict__ ly, const Nb& j) {
  const int nx = g.nx, ny = g.ny;
  double a = 0;
  if (j.x >= 1) a += lx[j.c - 1];          // j is the E neighbour of j - 1
  if (j.x == nx - 1) a += lx[j.c];         // j is its own (clamped) E neighbour
  if (j.x <= nx - 2) a -= lx[j.c + 1];     // j is the W neighbour of j + 1
  if (j.x == 0) a -= lx[j.c];
  if (j.y >= 1) a += ly[j.c - nx];
  if (j.y == ny - 1) a += ly[j.c];
  if (j.y <= ny - 2) a -= ly[j.c + nx];
  if (j.y == 0) a -= ly[j.c];
  return a;
}

// lambda_p = pFac G^T (lu, lv): the pressure correction's transpose
__global__ void __launch_bounds__(256)
k_adj_grad_T(GridDesc g, double pFac, const double* __restrict__ lu, const double* __restrict__ lv,
             double* __restrict__ lp)
{
  const int gx = blockIdx.x * BS + threadIdx.x;
  for (int r = 0; r < 4; r++) {
    const Nb j = nb_of(g, gx, blockIdx.y * BS + threadIdx.y + 8 * r);
    lp[j.c] = pFac * diff_T(g, lu, lv, j);
  }
}

// (lu, lv) += facDiv D^T lr: the RHS divergence's transpose
__global__ void __launch_bounds__(256)
k_adj_div_T(GridDesc g, double facDiv, const double* __restrict__ lr, double* __restrict__ lu,
            double* __restrict__ lv)
{
  const int gx = blockIdx.x * BS + threadIdx.x;
  const int nx = g.nx, ny = g.ny;
  for (int r = 0; r < 4; r++) {
    const Nb j = nb_of(g, gx, blockIdx.y * BS + threadIdx.y + 8 * r);
    double ax = 0, ay = 0;
    if (j.x >= 1) ax += lr[j.c - 1];
    if (j.x == nx - 1) ax += lr[j.c];
    if (j.x <= nx - 2) ax -= lr[j.c + 1];
    if (j.x == 0) ax -= lr[j.c];
    if (j.y >= 1) ay += lr[j.c - nx];
    if (j.y == ny - 1) ay += lr[j.c];
    if (j.y <= ny - 2) ay -= lr[j.c + nx];
    if (j.y == 0) ay -= lr[j.c];
    lu[j.c] += facDiv * ax;
    lv[j.c] += facDiv * ay;
  }
}

// Pen^T: lambda *= 1 - chi where the shape owns the cell (penalize's
// alpha); gb += the derivative of u = (1 - chi) u + chi U_s, U_s = (u_b -
// omega p_y, v_b + omega p_x) about the centre of mass, with respect to the
// body velocity (u_b, v_b, omega)
__global__ void __launch_bounds__(1024)
k_adj_pen(GridDesc g, const DevShape* sh, int k, ObstTiles t, const double* __restrict__ chig,
          double* lu, double* lv, double* gb)
{
  const DevShape& S = sh[k];
  const double Cx = S.s.com[0], Cy = S.s.com[1];
  double a[3] = {0, 0, 0};
  for (int s = blockIdx.x; s < S.ntiles; s += gridDim.x) {
    const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
    const size_t o = (size_t)s * BS2 + threadIdx.y * BS + threadIdx.x;
    const size_t c = (size_t)(by * BS + threadIdx.y) * g.nx + bx * BS + threadIdx.x;
    const double X = t.chi[o];
    if (chig[c] > X || X <= 0) continue;
    const double p0 = cell_x(g, bx, threadIdx.x) - Cx, p1 = cell_y(g, by, threadIdx.y) - Cy;
    a[0] += X * lu[c];
    a[1] += X * lv[c];
    a[2] += X * (p0 * lv[c] - p1 * lu[c]);
    lu[c] *= 1 - X;
    lv[c] *= 1 - X;
  }
  for (int q = 0; q < 3; q++) {
    double v = a[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0) atomicAdd(&gb[q], v);
  }
}

// ---- a free body: Shape::updateVelocity's 3x3 solve (Shape.cpp:25-59) of
// the momentum integrals (PressureSingle.cpp:23-67), transposed.  With chi
// fixed the matrix (penalM, penalJ, penalDX, penalDY) is a constant and
// symmetric: lb = A^-1 lx, by the forward's own LU.
__global__ void k_adj_solve(const DevShape* sh, int k, const double* lx, double* lb)
{
  const cup2d_shape_state& s = sh[k].s;
  double A[3][3] = {{s.penalM, 0, -s.penalDY}, {0, s.penalM, s.penalDX}, {-s.penalDY, s.penalDX, s.penalJ}};
  const double b[3] = {lx[0], lx[1], lx[2]};
  lu_solve3(A, b, lb);
}

// the momenta's transpose: (fluidMomX, fluidMomY, fluidAngMom) = sum F (u,
// v, p_x v - p_y u), F = h^2 rho chi, over the tile cells with chi > 0, of
// the pressure-corrected velocity: lambda += F (lb_0 - p_y lb_2, lb_1 + p_x lb_2)
__global__ void __launch_bounds__(1024)
k_adj_momenta(GridDesc g, const DevShape* sh, int k, ObstTiles t, const double* __restrict__ lb,
              double* lu, double* lv)
{
  const DevShape& S = sh[k];
  const double Cx = S.s.com[0], Cy = S.s.com[1];
  const double l0 = lb[0], l1 = lb[1], l2 = lb[2];
  for (int s = blockIdx.x; s < S.ntiles; s += gridDim.x) {
    const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
    const size_t o = (size_t)s * BS2 + threadIdx.y * BS + threadIdx.x;
    const double chi = t.chi[o];
    if (!(chi > 0)) continue;
    const size_t c = (size_t)(by * BS + threadIdx.y) * g.nx + bx * BS + threadIdx.x;
    const double p0 = cell_x(g, bx, threadIdx.x) - Cx, p1 = cell_y(g, by, threadIdx.y) - Cy;
    const double F = g.h * g.h * S.rhoTile * chi;
    lu[c] += F * (l0 - p1 * l2);
    lv[c] += F * (l1 + p0 * l2);
  }
}

// the objective's body-velocity weights of a step, added to lx
__global__ void k_adj_add3(double* lx, double a, double b, double c)
{
  lx[0] += a; lx[1] += b; lx[2] += c;
}

// ---- the body's force (ComputeForces.cpp:16-111, the surface cells of
// k_forces): forcex = sum over cells with a surface delta of
//   nu/h [ (u_E - u_W) nx + (u_N - u_S + v_E - v_W) ny / 2 ] - p nx
// and forcey alike, and the torque sum p_x fy - p_y fx about the centre of
// mass, linear in u, v and p with clamped neighbours.  With weights (wx, wy,
// wt) on (forcex, forcey, torque): part 0 adds the velocity terms'
// transpose to (lu, lv), part 1 the pressure term's to lp.
__global__ void __launch_bounds__(1024)
k_adj_force(GridDesc g, const DevShape* sh, int k, ObstTiles t, double wx, double wy, double wt, int part,
            double* lu, double* lv, double* lp)
{
  const DevShape& S = sh[k];
  const double Cx = S.s.com[0], Cy = S.s.com[1];
  for (int s = blockIdx.x; s < S.ntiles; s += gridDim.x) {
    const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
    const size_t o = (size_t)s * BS2 + threadIdx.y * BS + threadIdx.x;
    if (!(t.sD[o] > 0)) continue;
    const int gx = bx * BS + threadIdx.x, gy = by * BS + threadIdx.y;
    const Nb j = nb_of(g, gx, gy);
    const double nX = t.sdx[o], nY = t.sdy[o];
    // torque = sum p_x fy - p_y fx about the centre of mass (weight wt)
    const double P0 = cell_x(g, bx, threadIdx.x) - Cx, P1 = cell_y(g, by, threadIdx.y) - Cy;
    if (part == 1) {
      atomicAdd(&lp[j.c], -(wx * nX + wy * nY) + wt * (P1 * nX - P0 * nY));
      continue;
    }
    const double NUoH = g.nu / g.h;
    const double a = (wx - wt * P1) * nX * NUoH;                              // on u_E - u_W
    const double q = (wx * nY + wy * nX + wt * (P0 * nX - P1 * nY)) * NUoH / 2;  // on u_N - u_S, v_E - v_W
    const double d = (wy + wt * P0) * nY * NUoH;                              // on v_N - v_S
    atomicAdd(&lu[j.E], a); atomicAdd(&lu[j.W], -a);
    atomicAdd(&lu[j.N], q); atomicAdd(&lu[j.S], -q);
    atomicAdd(&lv[j.E], q); atomicAdd(&lv[j.W], -q);
    atomicAdd(&lv[j.N], d); atomicAdd(&lv[j.S], -d);
  }
}

// the objective's body terms of a step: acc += wx forcex + wy forcey + wt
// |torque| + wb . (u, v, omega) of the state the step left; *tau = torque
__global__ void k_adj_body_sum(const DevShape* sh, int k, double wx, double wy, double wt, double wb0,
                               double wb1, double wb2, double* acc, double* tau)
{
  const cup2d_shape_state& s = sh[k].s;
  *acc += wx * s.forcex + wy * s.forcey + wt * fabs(s.torque) + (wb0 * s.u + wb1 * s.v + wb2 * s.omega);
  *tau = s.torque;
}

// ---- the obstacle RHS terms O (k_rhs_obst, k_rhs_corr) --------------------
// over the shape's tile cells not owned by a larger chi: T' = T - X T; the
// sums s = sum -X T, pos / neg over perimeter cells of T' > 0 / T' < 0, and
// with the adjoint input lo (the adjoint of O's output): Lp = sum over
// perimeter T' > 0 of T' lo, Ln = the same over T' < 0.
// acc: s, pos, neg, Lp, Ln
__device__ __forceinline__ bool obst_cell(const GridDesc& g, const ObstTiles& t, int s, const double* chig,
                                          size_t& c, double& X, bool& perim) {
  const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
  const int gx = bx * BS + threadIdx.x, gy = by * BS + threadIdx.y;
  auto CHI = [&](int x, int y) -> double {
    x = x < 0 ? 0 : (x >= g.nx ? g.nx - 1 : x);
    y = y < 0 ? 0 : (y >= g.ny ? g.ny - 1 : y);
    return chig[(size_t)y * g.nx + x];
  };
  X = t.chi[(size_t)s * BS2 + threadIdx.y * BS + threadIdx.x];
  c = (size_t)gy * g.nx + gx;
  if (CHI(gx, gy) > X) return false;
  const double gxx = CHI(gx + 1, gy) - CHI(gx - 1, gy), gxy = CHI(gx, gy + 1) - CHI(gx, gy - 1);
  perim = gxx * gxx + gxy * gxy > 0;
  return true;
}

__global__ void __launch_bounds__(1024)
k_adj_obst_sums(GridDesc g, const DevShape* sh, int k, ObstTiles t, const double* __restrict__ chig,
                const double* __restrict__ T, const double* __restrict__ lo, double* acc)
{
  const DevShape& S = sh[k];
  double a[5] = {0, 0, 0, 0, 0};
  for (int s = blockIdx.x; s < S.ntiles; s += gridDim.x) {
    size_t c; double X; bool perim = false;
    if (!obst_cell(g, t, s, chig, c, X, perim)) continue;
    const double T0 = T[c], src = -X * T0, Tp = T0 + src;
    a[0] += src;
    if (perim && Tp > 0) { a[1] += Tp; a[3] += Tp * lo[c]; }
    if (perim && Tp < 0) { a[2] -= Tp; a[4] += Tp * lo[c]; }
  }
  for (int q = 0; q < 5; q++) {
    double v = a[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0) atomicAdd(&acc[q], v);
  }
}

// l = O'^T l in place over the processed cells (each reads and writes its
// own cell; the others pass unchanged)
__global__ void __launch_bounds__(1024)
k_adj_obst_apply(GridDesc g, const DevShape* sh, int k, ObstTiles t, const double* __restrict__ chig,
                 const double* __restrict__ T, double* lo, const double* __restrict__ acc)
{
  const DevShape& S = sh[k];
  const double s = acc[0], pos = acc[1], neg = acc[2], Lp = acc[3], Ln = acc[4];
  const double posF = fmax(pos, EPSd), negF = fmax(neg, EPSd);
  const double corr = s / (s > 0 ? posF : negF);
  for (int st = blockIdx.x; st < S.ntiles; st += gridDim.x) {
    size_t c; double X; bool perim = false;
    if (!obst_cell(g, t, st, chig, c, X, perim)) continue;
    const double T0 = T[c], Tp = T0 + (-X * T0), a = 1 - X;
    double r;
    if (s > 0) {
      // corr = s / pos: T'' = T' (1 - corr) on perimeter cells of T' > 0
      const bool q = perim && Tp > 0 && corr > 0;
      const double dcorr = (-X - (pos > EPSd && q ? corr * a : 0.0)) / posF;   // d corr / d T_c
      r = a * (q ? 1 - corr : 1.0) * lo[c] + dcorr * (-Lp);
    } else {
      // corr = s / neg (<= 0): T'' = T' (1 + corr) on perimeter cells of T' < 0
      const bool q = perim && Tp < 0 && corr < 0;
      const double dcorr = (-X + (neg > EPSd && q ? corr * a : 0.0)) / negF;
      r = a * (q ? 1 + corr : 1.0) * lo[c] + dcorr * Ln;
    }
    lo[c] = r;
  }
}

// ---- the gait gradient of a tethered swimmer ------------------------------
// Each step's objective sensitivity to the body's geometry on the grid
// (dense planes of the step): gX to chi, gU / gV to the penalization's
// target velocity U_s = (u_b - omega p_y + udef_x, v_b + omega p_x + udef_y),
// gSX / gSY to the force kernel's surface normals (sdx, sdy).  The gait moves
// only these (the body is held), so dJ/dtheta = sum over the steps of
// <g, d(chi, U_s, sdx, sdy)/dtheta>, the latter by central differences of
// the placement alone (flow-independent for a held body).
//
// Penalization and forces, from lambda on u^(n+1) (before Pen^T):
// d u^(n+1)/d chi = U_s - u2, d u^(n+1)/d U_s = chi; forcex = sum nu/h [(u_E -
// u_W) sdx + (u_N - u_S + v_E - v_W) sdy / 2] - p sdx, forcey alike, the
// torque sum p_x fy - p_y fx about the centre of mass C (gCom: d/dC).
__global__ void __launch_bounds__(1024)
k_adj_geo_pen(GridDesc g, const DevShape* sh, int k, ObstTiles t, const double* __restrict__ chig,
              const double* __restrict__ u1, const double* __restrict__ v1, const double* __restrict__ p,
              double pFac, const double* __restrict__ un, const double* __restrict__ vn,
              const double* __restrict__ lu, const double* __restrict__ lv, double wFx, double wFy, double wt,
              double* gX, double* gU, double* gV, double* gSX, double* gSY, double* gCom)
{
  const DevShape& S = sh[k];
  const double Cx = S.s.com[0], Cy = S.s.com[1];
  const double NUoH = g.nu / g.h;
  // the torque about the centre of mass: d/dC = (-forcey, forcex)
  if (blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) {
    gCom[0] = -wt * S.s.forcey;
    gCom[1] = wt * S.s.forcex;
  }
  for (int s = blockIdx.x; s < S.ntiles; s += gridDim.x) {
    const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
    const size_t o = (size_t)s * BS2 + threadIdx.y * BS + threadIdx.x;
    const int gx = bx * BS + threadIdx.x, gy = by * BS + threadIdx.y;
    const Nb j = nb_of(g, gx, gy);
    const double X = t.chi[o];
    if (chig[j.c] > X) continue;
    const double p0 = cell_x(g, bx, threadIdx.x) - Cx, p1 = cell_y(g, by, threadIdx.y) - Cy;
    double ux, uy;
    udef_at(t, o, S, p0, p1, ux, uy);
    const double US = S.s.u - S.s.omega * p1 + ux, VS = S.s.v + S.s.omega * p0 + uy;
    const double u2 = u1[j.c] + pFac * (p[j.E] - p[j.W]), v2 = v1[j.c] + pFac * (p[j.N] - p[j.S]);
    const double Lu = lu[j.c], Lv = lv[j.c];
    gX[j.c] = Lu * (US - u2) + Lv * (VS - v2);
    gU[j.c] = Lu * X;
    gV[j.c] = Lv * X;
    const double D11 = NUoH * (un[j.E] - un[j.W]), D22 = NUoH * (vn[j.N] - vn[j.S]);
    const double D12 = NUoH / 2 * (un[j.N] - un[j.S] + vn[j.E] - vn[j.W]);
    const double P = p[j.c];
    gSX[j.c] = wFx * (D11 - P) + wFy * D12 + wt * (p0 * D12 - p1 * (D11 - P));
    gSY[j.c] = wFx * D12 + wFy * (D22 - P) + wt * (p0 * (D22 - P) - p1 * D12);
  }
}

// The obstacle terms' part of gX, from lambda on their output (lo) and the
// sums of k_adj_obst_sums: with T' = (1 - chi) T and s = sum -chi T,
// dJ/dchi = -T (dJ/dT' + dJ/ds) on the active piece.  Before
// k_adj_obst_apply overwrites lo.
__global__ void __launch_bounds__(1024)
k_adj_geo_obst(GridDesc g, const DevShape* sh, int k, ObstTiles t, const double* __restrict__ chig,
               const double* __restrict__ T, const double* __restrict__ lo, const double* __restrict__ acc,
               double* gX)
{
  const DevShape& S = sh[k];
  const double s = acc[0], pos = acc[1], neg = acc[2], Lp = acc[3], Ln = acc[4];
  const double posF = fmax(pos, EPSd), negF = fmax(neg, EPSd);
  const double corr = s / (s > 0 ? posF : negF);
  for (int st = blockIdx.x; st < S.ntiles; st += gridDim.x) {
    size_t c; double X; bool perim = false;
    if (!obst_cell(g, t, st, chig, c, X, perim)) continue;
    const double T0 = T[c], Tp = T0 + (-X * T0);
    double GT, Gs;
    if (s > 0) {
      const bool P = perim && Tp > 0;
      GT = lo[c] * (P && corr > 0 ? 1 - corr : 1.0) + (P && pos > EPSd ? corr / posF * Lp : 0.0);
      Gs = -Lp / posF;
    } else {
      const bool N = perim && Tp < 0;
      GT = lo[c] * (N && corr < 0 ? 1 + corr : 1.0) + (N && neg > EPSd ? corr / negF * Ln : 0.0);
      Gs = Ln / negF;
    }
    gX[c] += -T0 * (GT + Gs);
  }
}

// <g, geometry> over the tiles of the current placement (the replay of a
// perturbed gait): acc += sum gX chi + gU U_s + gV V_s + gSX sdx + gSY sdy,
// plus gCom . C
__global__ void __launch_bounds__(1024)
k_adj_geo_dot(GridDesc g, const DevShape* sh, int k, ObstTiles t, const double* __restrict__ chig,
              const double* __restrict__ gX, const double* __restrict__ gU, const double* __restrict__ gV,
              const double* __restrict__ gSX, const double* __restrict__ gSY, const double* __restrict__ gCom,
              double* acc)
{
  const DevShape& S = sh[k];
  const double Cx = S.s.com[0], Cy = S.s.com[1];
  double a = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) a = gCom[0] * Cx + gCom[1] * Cy;
  for (int s = blockIdx.x; s < S.ntiles; s += gridDim.x) {
    const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
    const size_t o = (size_t)s * BS2 + threadIdx.y * BS + threadIdx.x;
    const size_t c = (size_t)(by * BS + threadIdx.y) * g.nx + bx * BS + threadIdx.x;
    const double X = t.chi[o];
    if (chig[c] > X) continue;
    const double p0 = cell_x(g, bx, threadIdx.x) - Cx, p1 = cell_y(g, by, threadIdx.y) - Cy;
    double ux, uy;
    udef_at(t, o, S, p0, p1, ux, uy);
    const double US = S.s.u - S.s.omega * p1 + ux, VS = S.s.v + S.s.omega * p0 + uy;
    a += gX[c] * X + gU[c] * US + gV[c] * VS + gSX[c] * t.sdx[o] + gSY[c] * t.sdy[o];
  }
  for (int q = 16; q > 0; q >>= 1) a += __shfl_xor_sync(0xffffffffu, a, q);
  if ((threadIdx.x & 31) == 0 && a != 0) atomicAdd(acc, a);
}

// ---- the boundary-strip fade F (cub2rhs) ----------------------------------
__device__ __forceinline__ double fade_w2(const GridDesc& g, int gx, int gy) {
  const double fadeLenX = g.fadeLenX, invFadeX = 1 / fmax(fadeLenX, EPSd);
  const double fadeLenY = g.fadeLenY, invFadeY = 1 / fmax(fadeLenY, EPSd);
  const double px = cell_x(g, gx >> 5, gx & 31), py = cell_y(g, gy >> 5, gy & 31);
  const double yt = invFadeY * fmax(0.0, fadeLenY - g.ext[1] + py);
  const double yb = invFadeY * fmax(0.0, fadeLenY - py);
  const double xt = invFadeX * fmax(0.0, fadeLenX - g.ext[0] + px);
  const double xb = invFadeX * fmax(0.0, fadeLenX - px);
  const double fa = fmin(fmax(fmax(yt, yb), fmax(xt, xb)), 1.0);
  return fa * fa;
}

// over the strip blocks: S = sum w2 f, Sp, Sn (as the forward), Lp = sum
// over w2 f > 0 of w2 f lb, Ln = sum over w2 f < 0 of w2 f lb
__global__ void __launch_bounds__(256)
k_adj_fade_sums(GridDesc g, const double* __restrict__ f, const double* __restrict__ lb, double* acc)
{
  const int bx = blockIdx.x, by = blockIdx.y;
  if (!fade_touch(g, bx, by)) return;
  const int gx = bx * BS + threadIdx.x;
  double a[5] = {0, 0, 0, 0, 0};
  for (int r = 0; r < 4; r++) {
    const int gy = by * BS + threadIdx.y + 8 * r;
    const size_t c = (size_t)gy * g.nx + gx;
    const double w2 = fade_w2(g, gx, gy), fw = f[c] * w2;
    a[0] += fw;
    if (fw > 0) { a[1] += fw; a[3] += fw * lb[c]; }
    if (fw < 0) { a[2] -= fw; a[4] += fw * lb[c]; }
  }
  for (int q = 0; q < 5; q++) {
    double v = a[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0) atomicAdd(&acc[q], v);
  }
}

// lb = F'^T lb
__global__ void __launch_bounds__(256)
k_adj_fade_apply(GridDesc g, const double* __restrict__ f, double* lb, const double* __restrict__ acc)
{
  // in place; outside the strip blocks w2 = 0 and lambda passes unchanged
  if (!fade_touch(g, blockIdx.x, blockIdx.y)) return;
  const double S = acc[0], Sp = acc[1], Sn = acc[2], Lp = acc[3], Ln = acc[4];
  const double SpF = fmax(Sp, EPSd), SnF = fmax(Sn, EPSd);
  const double corr = S > 0 ? S / SpF : S / SnF;
  const int gx = blockIdx.x * BS + threadIdx.x;
  for (int r = 0; r < 4; r++) {
    const int gy = blockIdx.y * BS + threadIdx.y + 8 * r;
    const size_t c = (size_t)gy * g.nx + gx;
    const double w2 = fade_w2(g, gx, gy);
    const double fw = f[c] * w2;
    double r_;
    if (S > 0) {
      const bool P = fw > 0;
      const double dcorr = (w2 - (Sp > EPSd && P ? corr * w2 : 0.0)) / SpF;   // d corr / d f_c
      r_ = (1 - w2) * lb[c] + (P ? corr * w2 * lb[c] : 0.0) + dcorr * Lp;
    } else {
      const bool N = fw < 0;
      const double dcorr = (w2 + (Sn > EPSd && N ? corr * w2 : 0.0)) / SnF;
      r_ = (1 - w2) * lb[c] - (N ? corr * w2 * lb[c] : 0.0) - dcorr * Ln;
    }
    lb[c] = r_;
  }
}

// ---- advDiff, linearized about u^n (advDiff.cpp:57-116) -------------------
// dW..dN: the inflow fades' derivatives with respect to (U0, U1)
struct AdvC { double afac, dfac, fW, fS, fE, fN, U0, U1; double dW[2], dS[2], dE[2], dN[2]; int nb; };

// Gamma = sum of sigma lambda over the boundary cells (sigma: +1 on the W
// column / S row, -1 on the E column / N row; u on the columns, v on the
// rows): the outflow correction's rank-one transpose
__global__ void __launch_bounds__(256)
k_adj_adv_gamma(GridDesc g, const double* __restrict__ lu, const double* __restrict__ lv, double* acc)
{
  const int nx = g.nx, ny = g.ny, n = 2 * (nx + ny);
  double a = 0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    if (q < ny) a += lu[(size_t)q * nx];
    else if (q < 2 * ny) a -= lu[(size_t)(q - ny) * nx + nx - 1];
    else if (q < 2 * ny + nx) a += lv[q - 2 * ny];
    else a -= lv[(size_t)(ny - 1) * nx + (q - 2 * ny - nx)];
  }
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31) == 0 && a != 0) atomicAdd(acc, a);
}

// lambda before the correction: lambda - sigma Gamma / Nb
__device__ __forceinline__ double lpre_u(const GridDesc& g, const double* lu, size_t c, int x, double gn) {
  double v = lu[c];
  if (x == 0) v -= gn;
  if (x == g.nx - 1) v += gn;
  return v;
}
__device__ __forceinline__ double lpre_v(const GridDesc& g, const double* lv, size_t c, int y, double gn) {
  double v = lv[c];
  if (y == 0) v -= gn;
  if (y == g.ny - 1) v += gn;
  return v;
}

// (ou, ov) = A'^T (lu, lv); gb -= the derivative with respect to the lab
// velocity (U0, U1) = -(body velocity) of a fixed body
__global__ void __launch_bounds__(256)
k_adj_advdiff(GridDesc g, AdvC k, const double* __restrict__ u, const double* __restrict__ v,
              const double* __restrict__ lu, const double* __restrict__ lv, const double* __restrict__ acc,
              double* __restrict__ ou, double* __restrict__ ov, double* gb)
{
  const double gn = acc[0] / k.nb;
  const int nx = g.nx, ny = g.ny;
  const int gx = blockIdx.x * BS + threadIdx.x;
  double dU[2] = {0, 0};
  for (int r = 0; r < 4; r++) {
    const int gy = blockIdx.y * BS + threadIdx.y + 8 * r;
    const Nb j = nb_of(g, gx, gy);
    // the forward's neighbour values at j (ghosts: the cell scaled by the fade)
    const double uc = u[j.c], vc = v[j.c];
    const double uW = j.x > 0 ? u[j.W] : uc * k.fW, uE = j.x < nx - 1 ? u[j.E] : uc * k.fE;
    const double uS = j.y > 0 ? u[j.S] : uc * k.fS, uN = j.y < ny - 1 ? u[j.N] : uc * k.fN;
    const double vW = j.x > 0 ? v[j.W] : vc * k.fW, vE = j.x < nx - 1 ? v[j.E] : vc * k.fE;
    const double vS = j.y > 0 ? v[j.S] : vc * k.fS, vN = j.y < ny - 1 ? v[j.N] : vc * k.fN;
    const double Lu = lpre_u(g, lu, j.c, j.x, gn), Lv = lpre_v(g, lv, j.c, j.y, gn);
    // coefficients of the neighbours in u'_j, v'_j (the same for both)
    const double cE = k.afac * (uc + k.U0) + k.dfac, cW = -k.afac * (uc + k.U0) + k.dfac;
    const double cN = k.afac * (vc + k.U1) + k.dfac, cS = -k.afac * (vc + k.U1) + k.dfac;
    // j's own terms, with its ghost neighbours folded in
    double du = 1 + k.afac * (uE - uW) - 4 * k.dfac, dv = 1 + k.afac * (vN - vS) - 4 * k.dfac;
    double g_ = 0;
    if (j.x == 0) g_ += cW * k.fW;
    if (j.x == nx - 1) g_ += cE * k.fE;
    if (j.y == 0) g_ += cS * k.fS;
    if (j.y == ny - 1) g_ += cN * k.fN;
    double au = (du + g_) * Lu + k.afac * (vE - vW) * Lv;
    double av = (dv + g_) * Lv + k.afac * (uN - uS) * Lu;
    // d(u'_j, v'_j)/dU: the advecting velocity, and the fades of j's ghosts
    {
      double e[2] = {0, 0};                             // sum over j's ghosts of c_ghost df/dU
      for (int q = 0; q < 2; q++) {
        if (j.x == 0) e[q] += cW * k.dW[q];
        if (j.x == nx - 1) e[q] += cE * k.dE[q];
        if (j.y == 0) e[q] += cS * k.dS[q];
        if (j.y == ny - 1) e[q] += cN * k.dN[q];
      }
      dU[0] += Lu * (k.afac * (uE - uW) + e[0] * uc) + Lv * (k.afac * (vE - vW) + e[0] * vc);
      dU[1] += Lu * (k.afac * (uN - uS) + e[1] * uc) + Lv * (k.afac * (vN - vS) + e[1] * vc);
    }
    // neighbours d whose stencil holds j
    if (j.x >= 1) {                                   // j is the E neighbour of d = j - 1
      const size_t d = j.c - 1;
      const double cEd = k.afac * (u[d] + k.U0) + k.dfac;
      au += cEd * lpre_u(g, lu, d, j.x - 1, gn);
      av += cEd * lpre_v(g, lv, d, j.y, gn);
    }
    if (j.x <= nx - 2) {                              // the W neighbour of d = j + 1
      const size_t d = j.c + 1;
      const double cWd = -k.afac * (u[d] + k.U0) + k.dfac;
      au += cWd * lpre_u(g, lu, d, j.x + 1, gn);
      av += cWd * lpre_v(g, lv, d, j.y, gn);
    }
    if (j.y >= 1) {                                   // the N neighbour of d = j - nx
      const size_t d = j.c - nx;
      const double cNd = k.afac * (v[d] + k.U1) + k.dfac;
      au += cNd * lpre_u(g, lu, d, j.x, gn);
      av += cNd * lpre_v(g, lv, d, j.y - 1, gn);
    }
    if (j.y <= ny - 2) {                              // the S neighbour of d = j + nx
      const size_t d = j.c + nx;
      const double cSd = -k.afac * (v[d] + k.U1) + k.dfac;
      au += cSd * lpre_u(g, lu, d, j.x, gn);
      av += cSd * lpre_v(g, lv, d, j.y + 1, gn);
    }
    ou[j.c] = au;
    ov[j.c] = av;
  }
  for (int q = 0; q < 2; q++) {
    double w = dU[q];
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    if ((threadIdx.x & 31) == 0 && w != 0) atomicAdd(&gb[q], -w);
  }
}

// ---- the recomputation's copies, one launch for many regions ------------
constexpr int MAX_COPIES = 16;
struct CopyList {
  const unsigned* src[MAX_COPIES];
  unsigned* dst[MAX_COPIES];
  size_t words[MAX_COPIES];                       // 4-byte words
  int n;
};
static_assert(sizeof(DevShape) % 4 == 0, "the shape snapshot is copied in 4-byte words");
__global__ void __launch_bounds__(256) k_copy_many(CopyList L) {
  for (int q = 0; q < L.n; q++) {
    const unsigned* __restrict__ a = L.src[q];
    unsigned* __restrict__ b = L.dst[q];
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < L.words[q]; i += (size_t)gridDim.x * blockDim.x)
      b[i] = a[i];
  }
}

// ---- the objective: (1/N) sum over steps of (h^2/2) sum_box (u^2 + v^2) ---
struct ProbeBox { int x0, x1, y0, y1; };
__global__ void __launch_bounds__(256)
k_adj_probe(GridDesc g, ProbeBox bx, const double* __restrict__ u, const double* __restrict__ v, double w,
            double* acc, double* lu, double* lv)
{
  double a = 0;
  const int W = bx.x1 - bx.x0, H = bx.y1 - bx.y0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < W * H; q += gridDim.x * blockDim.x) {
    const size_t c = (size_t)(bx.y0 + q / W) * g.nx + bx.x0 + q % W;
    const double uc = u[c], vc = v[c];
    if (acc) a += 0.5 * w * (uc * uc + vc * vc);
    if (lu) { lu[c] += w * uc; lv[c] += w * vc; }
  }
  if (!acc) return;
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31) == 0 && a != 0) atomicAdd(acc, a);
}

} // namespace
} // namespace cup2d

using namespace cup2d;

namespace {

int adj_fail(cup2d_ctx* ctx, int code, const std::string& msg) {
  ctx->c.err = msg;
  return code;
}

#define ACK(call)                                                               \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) return adj_fail(ctx, CUP2D_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define ARC(call)                                                               \
  do { const int r_ = (call); if (r_ != CUP2D_OK) return r_; } while (0)

// a checkpoint of the run, loaded back (the error names which)
#define ALOAD(idx)                                                              \
  do {                                                                          \
    const int r_ = cup2d_checkpoint_load(ctx, ck[idx], ckBytes);                \
    if (r_ != CUP2D_OK) {                                                       \
      ctx->c.err += " (the adjoint's checkpoint " + std::to_string(idx) + " of " + std::to_string(nseg) + ")"; \
      return r_;                                                                \
    }                                                                           \
  } while (0)

// device scratch of the adjoint run, freed on every exit
struct AdjBufs {
  std::vector<void*> p;
  ~AdjBufs() { for (void* q : p) cudaFree(q); }
  template <typename T> T* get(size_t n) {
    void* q = nullptr;
    if (cudaMalloc(&q, sizeof(T) * (n ? n : 1)) != cudaSuccess) return nullptr;
    p.push_back(q);
    return static_cast<T*>(q);
  }
};

AdvC adv_coef_host(const Ctx& c, double dt, double U0, double U1) {
  AdvC k;
  const double h = c.g.h;
  k.U0 = U0; k.U1 = U1;
  k.afac = -0.5 * dt / h;
  k.dfac = (c.g.nu / h) * (dt / h);
  // fades 1 - r^2/100 of r = max/min(U, 0) / nor, nor = max(|U0|, |U1|, eps)
  const double nor = std::max({std::fabs(U0), std::fabs(U1), DBL_EPSILON});
  double dnor[2] = {0, 0};
  if (std::fabs(U0) >= std::fabs(U1) && std::fabs(U0) > DBL_EPSILON) dnor[0] = U0 > 0 ? 1 : -1;
  else if (std::fabs(U1) > DBL_EPSILON) dnor[1] = U1 > 0 ? 1 : -1;
  auto fade = [&](double m, int comp, bool pos, double* d) {
    // m = max(U, 0) (pos) or min(U, 0) of component comp
    const double r = m / nor;
    const double Uc = comp == 0 ? U0 : U1;
    const bool active = pos ? Uc > 0 : Uc < 0;
    for (int q = 0; q < 2; q++) {
      const double dr = (q == comp && active ? 1.0 / nor : 0.0) - m / (nor * nor) * dnor[q];
      d[q] = -2 * r / 100 * dr;
    }
    return 1 - r * r / 100;                               // BC_KILL_FAC = 100
  };
  k.fW = fade(std::max(U0, 0.0), 0, true, k.dW); k.fS = fade(std::max(U1, 0.0), 1, true, k.dS);
  k.fE = fade(std::min(U0, 0.0), 0, false, k.dE); k.fN = fade(std::min(U1, 0.0), 1, false, k.dN);
  k.nb = 2 * (BS * c.g.bpdy) + 2 * (BS * c.g.bpdx);
  return k;
}

// Contexts of ctx's configuration and shapes, initialised, for the gait's
// placement replays (one per perturbed gait, run side by side); kept in
// ctx.  Returns false if they cannot be made (the replays then run one
// after another on ctx itself).
bool gait_shadows(cup2d_ctx* ctx, int n) {
  Ctx& c = ctx->c;
  while ((int)c.gaitShadows.size() < n) {
    cup2d_ctx* sh = nullptr;
    cup2d_config cfg = c.cfg;
    if (cup2d_create(&cfg, &sh) != CUP2D_OK) return false;
    bool ok = true;
    for (size_t k = 0; ok && k < c.shapeParams.size(); k++)
      ok = cup2d_add_shape(sh, c.shapeKinds[k], &c.shapeParams[k], nullptr) == CUP2D_OK;
    if (!ok || cup2d_init(sh) != CUP2D_OK) { cup2d_destroy(sh); return false; }
    c.gaitShadows.push_back(sh);
  }
  return true;
}

} // namespace

extern "C" {

int cup2d_adjoint_run(cup2d_ctx* ctx, int nsteps, int every, const cup2d_adjoint_objective* obj,
                      const double* dt_in, double* dt_out, double* J, double* grad_u, double* grad_v,
                      double* grad_body, double* grad_gait, double* ms) {
  if (!ctx || nsteps <= 0 || every <= 0 || !obj || !J) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  if (!c.initialised) return adj_fail(ctx, CUP2D_ESTATE, "not initialised");
  if (c.cfg.iterative || c.varRho || c.cfg.implicit_penalization || c.cfg.precision != CUP2D_PREC_FP64)
    return adj_fail(ctx, CUP2D_ENOTSUP, "the adjoint covers the FP64 PressureSingle pipeline (explicit penalization)");
  if (c.nshapes != 1)
    return adj_fail(ctx, CUP2D_ENOTSUP, "the adjoint covers one body");
  const ShapeCfg& sf = c.hshapes[0].cfg;
  // forced: the body velocity is held (a parameter); free: solved each step
  // from the momentum integrals.  Either way fixed on the grid: a disk's chi
  // does not move, a swimmer's moves with its gait alone (the recomputation
  // keeps each step's obstacle tiles).
  const bool forced = sf.bForcedx && sf.bForcedy && sf.bBlockang;
  const bool freeBody = !sf.bForcedx && !sf.bForcedy && !sf.bBlockang;
  if (!(sf.bFixedx && sf.bFixedy) || !(forced || freeBody))
    return adj_fail(ctx, CUP2D_ENOTSUP, "the adjoint needs a body fixed on the grid (bFixed), "
                                        "either forced in x, y and angle or free in all three");
  if (sf.kind != CUP2D_SHAPE_DISK && (!forced || sf.pid || sf.pidpos))
    return adj_fail(ctx, CUP2D_ENOTSUP, "a swimmer must be tethered (forced in x, y and angle, no PID "
                                        "controller): a free swimmer's rotation moves its chi with the flow");
  const bool gait = grad_gait != nullptr;
  const bool curvFish = sf.kind == CUP2D_SHAPE_STEFANFISH || sf.kind == CUP2D_SHAPE_ENVELOPEFISH;
  if (gait && !(curvFish && forced))
    return adj_fail(ctx, CUP2D_ENOTSUP, "the gait gradient needs a tethered curvature swimmer");
  const GridDesc& g = c.g;
  {
    double t0, dtd, ux, uy; int st;
    ARC(cup2d_get_scalars(ctx, &t0, &dtd, &st, &ux, &uy));
    if (forced && sf.tAccel > 0 && t0 < sf.tAccel)
      return adj_fail(ctx, CUP2D_ENOTSUP, "the body is still accelerating (tAccel): its velocity is not held");
  }
  const size_t n = c.ncells(), nb = sizeof(double) * n;
  const bool energy = obj->w_energy != 0;
  const bool force = obj->w_force[0] != 0 || obj->w_force[1] != 0 || obj->w_torque != 0;
  const bool bodyTerm = obj->w_body[0] != 0 || obj->w_body[1] != 0 || obj->w_body[2] != 0;
  ProbeBox bx{0, 0, 0, 0};
  if (energy) {
    bx.x0 = std::max(0, (int)std::floor(obj->box[0] / g.h)); bx.x1 = std::min(g.nx, (int)std::ceil(obj->box[1] / g.h));
    bx.y0 = std::max(0, (int)std::floor(obj->box[2] / g.h)); bx.y1 = std::min(g.ny, (int)std::ceil(obj->box[3] / g.h));
    if (bx.x1 <= bx.x0 || bx.y1 <= bx.y0) return adj_fail(ctx, CUP2D_EINVAL, "empty probe box");
  }
  const double wE = obj->w_energy * g.h * g.h / nsteps;   // the energy term's weight per step
  const double wFx = obj->w_force[0] / nsteps, wFy = obj->w_force[1] / nsteps, wT = obj->w_torque / nsteps;
  const double wB[3] = {obj->w_body[0] / nsteps, obj->w_body[1] / nsteps, obj->w_body[2] / nsteps};
  const dim3 grid2(g.bpdx, g.bpdy), blk2(32, 8);
  const int probeGrid = energy ? std::min(1024, ((bx.x1 - bx.x0) * (bx.y1 - bx.y0) + 255) / 256) : 1;

  AdjBufs B;
  size_t ckBytes = 0;
  ARC(cup2d_checkpoint_size(ctx, &ckBytes));
  const int nseg = (nsteps + every - 1) / every;
  std::vector<void*> ck(nseg + 1);
  for (int s = 0; s <= nseg; s++)
    if (!(ck[s] = B.get<char>(ckBytes))) return adj_fail(ctx, CUP2D_ENOMEM, "adjoint checkpoints");
  double* acc = B.get<double>(8);          // [0..4] reductions of a transposed stage
  // [0] J; [1..3] the body-velocity gradient (forced: the held velocity's,
  // accumulated over the steps; free: the adjoint of the step's output
  // velocity); [4..6] a free body's adjoint of the previous output, formed
  // by advDiff's lab velocity; [8..10] the solve's transpose
  double* obv = B.get<double>(12);
  double* tauRec = B.get<double>(nsteps);    // each step's torque (the |torque| term's sign)
  if (!acc || !obv || !tauRec) return adj_fail(ctx, CUP2D_ENOMEM, "adjoint scratch");
  std::vector<double> dts(nsteps), U0s(nsteps), U1s(nsteps);
  struct Ev {
    cudaEvent_t e[3] = {nullptr, nullptr, nullptr};
    ~Ev() { for (cudaEvent_t x : e) if (x) cudaEventDestroy(x); }
  } ev;
  for (cudaEvent_t& x : ev.e) ACK(cudaEventCreate(&x));
  cudaEvent_t e0 = ev.e[0], e1 = ev.e[1], e2 = ev.e[2];

  // one step of Simulation::advance with dt given (PutObjectsOnGrid, advDiff,
  // PressureSingle, ComputeForces); T / F, when non-null, receive the RHS
  // before the obstacle terms and before the fade
  auto step = [&](double dt, double* T, double* F, double* U1, double* V1) -> int {
    ARC(cup2d_put_objects(ctx, dt));
    ARC(cup2d_adv_diff(ctx, dt));
    if (U1) {                                   // advDiff's velocity
      ACK(cudaMemcpyAsync(U1, c.u(), nb, cudaMemcpyDeviceToDevice, c.stream));
      ACK(cudaMemcpyAsync(V1, c.v(), nb, cudaMemcpyDeviceToDevice, c.stream));
    }
    ARC(pressure_single_keep(ctx, dt, T, F));
    ARC(cup2d_compute_forces(ctx, dt));
    ARC(cup2d_end_step(ctx));
    return CUP2D_OK;
  };

  // forward: checkpoints, the dt schedule, J
  ACK(cudaMemsetAsync(obv, 0, sizeof(double) * 12, c.stream));
  ACK(cudaEventRecord(e0, c.stream));
  for (int i = 0; i < nsteps; i++) {
    if (i % every == 0) ARC(cup2d_checkpoint_save(ctx, ck[i / every], ckBytes));
    double dt;
    if (dt_in) dt = dt_in[i];
    else ARC(cup2d_calc_dt(ctx, &dt));
    dts[i] = dt;
    ARC(step(dt, nullptr, nullptr, nullptr, nullptr));
    // the lab velocity of the step (set by the placement from the forced body)
    double t_, dtd, ux, uy; int st;
    ARC(cup2d_get_scalars(ctx, &t_, &dtd, &st, &ux, &uy));
    U0s[i] = ux; U1s[i] = uy;
    if (energy) k_adj_probe<<<probeGrid, 256, 0, c.stream>>>(g, bx, c.u(), c.v(), wE, obv, nullptr, nullptr);
    if (force || bodyTerm)
      k_adj_body_sum<<<1, 1, 0, c.stream>>>(c.dshapes, 0, wFx, wFy, wT, wB[0], wB[1], wB[2], obv, tauRec + i);
    ACK(cudaGetLastError());
  }
  ACK(cudaEventRecord(e1, c.stream));
  ARC(cup2d_checkpoint_save(ctx, ck[nseg], ckBytes));      // the final state, restored at the end
  {
    // the body stays forced over the whole run (Shape.cpp: forced while
    // time < timeForced)
    double tEnd, dtd, ux, uy; int st;
    ARC(cup2d_get_scalars(ctx, &tEnd, &dtd, &st, &ux, &uy));
    if (!(tEnd <= sf.timeForced))
      return adj_fail(ctx, CUP2D_ENOTSUP, "the body is released (timeForced) within the run");
  }
  ACK(cudaMemcpyAsync(J, obv, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  std::vector<double> taus(nsteps, 0.0), wTs(nsteps, 0.0);
  if (force || bodyTerm)
    ACK(cudaMemcpyAsync(taus.data(), tauRec, sizeof(double) * nsteps, cudaMemcpyDeviceToHost, c.stream));
  ACK(cudaStreamSynchronize(c.stream));
  for (int i = 0; i < nsteps; i++) wTs[i] = taus[i] > 0 ? wT : (taus[i] < 0 ? -wT : 0.0);   // d|torque|
  if (dt_out) std::copy(dts.begin(), dts.end(), dt_out);
  float fms = 0;
  ACK(cudaEventElapsedTime(&fms, e0, e1));
  if (ms) { ms[0] = fms; ms[1] = 0; if (gait) ms[2] = 0; }
  if (!grad_u && !grad_v && !grad_body && !gait) {
    ALOAD(nseg);
    return CUP2D_OK;
  }

  // backward
  const size_t segN = (size_t)std::min(every, nsteps);   // steps of a segment
  // the velocity at the segment's start and after each of its steps (u^n of
  // step j > 0 is u^(n+1) of step j - 1)
  double* su = B.get<double>(n);
  double* sv = B.get<double>(n);
  double* sT = B.get<double>(n * segN);      // RHS before the obstacle terms
  double* sF = B.get<double>(n * segN);      // RHS before the fade
  double* pu = B.get<double>(n * segN);
  double* pv = B.get<double>(n * segN);
  // the gait: advDiff's velocity and the pressure of each step, and the
  // geometry sensitivities of every step of the run
  double* su1 = gait ? B.get<double>(n * segN) : nullptr;
  double* sv1 = gait ? B.get<double>(n * segN) : nullptr;
  double* sp = gait ? B.get<double>(n * segN) : nullptr;
  double* gG[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};   // gX, gU, gV, gSX, gSY
  double* gCom = gait ? B.get<double>(2 * (size_t)nsteps) : nullptr;  // d/d(centre of mass)
  if (gait) {
    if (!gCom) return adj_fail(ctx, CUP2D_ENOMEM, "adjoint gait planes");
    ACK(cudaMemsetAsync(gCom, 0, sizeof(double) * 2 * nsteps, c.stream));
    for (double*& q : gG) {
      if (!(q = B.get<double>(n * (size_t)nsteps))) return adj_fail(ctx, CUP2D_ENOMEM, "adjoint gait planes");
      ACK(cudaMemsetAsync(q, 0, nb * nsteps, c.stream));
    }
    if (!su1 || !sv1 || !sp) return adj_fail(ctx, CUP2D_ENOMEM, "adjoint segment buffers");
  }
  double* lu = B.get<double>(n);
  double* lv = B.get<double>(n);
  double* l1 = B.get<double>(n);
  double* l2 = B.get<double>(n);
  double* tu = B.get<double>(n);
  double* tv = B.get<double>(n);
  if (!su || !sv || !sT || !sF || !pu || !pv || !lu || !lv || !l1 || !l2 || !tu || !tv)
    return adj_fail(ctx, CUP2D_ENOMEM, "adjoint segment buffers");
  // a swimmer: each recomputed step's obstacle state (the shape's tile
  // count and centre of mass, its tiles, the grid's chi); a disk's does not
  // change from step to step, and the live one serves
  const ObstTiles live = c.tiles[0];
  const int cap = live.capacity;
  const size_t tb = (size_t)cap * BS2;
  const bool keepObst = sf.kind != CUP2D_SHAPE_DISK;
  const size_t segK = keepObst ? segN : 0;
  DevShape* shSnap = B.get<DevShape>(segK);
  int* tlSnap = B.get<int>((size_t)cap * segK);
  double* tSnap[6];
  for (int q = 0; q < 6; q++) tSnap[q] = B.get<double>(tb * segK);   // chi, udx, udy, sD, sdx, sdy
  double* chiSnap = B.get<double>(n * segK);
  if (!shSnap || !tlSnap || !chiSnap) return adj_fail(ctx, CUP2D_ENOMEM, "adjoint obstacle snapshots");
  for (double* q : tSnap) if (!q) return adj_fail(ctx, CUP2D_ENOMEM, "adjoint obstacle snapshots");
  auto tilesAt = [&](int j) {
    if (!keepObst) return live;
    ObstTiles t = live;
    t.tiles = tlSnap + (size_t)j * cap;
    t.chi = tSnap[0] + j * tb; t.udx = tSnap[1] + j * tb; t.udy = tSnap[2] + j * tb;
    t.sD = tSnap[3] + j * tb; t.sdx = tSnap[4] + j * tb; t.sdy = tSnap[5] + j * tb;
    t.dist = nullptr; t.slot = nullptr;
    return t;
  };
  ACK(cudaMemsetAsync(lu, 0, nb, c.stream));
  ACK(cudaMemsetAsync(lv, 0, nb, c.stream));
  ACK(cudaMemsetAsync(obv + 1, 0, sizeof(double) * 11, c.stream));
  ACK(cudaEventRecord(e2, c.stream));
  double* lx = obv + 1;                      // the body-velocity adjoint (see above)
  double* lxPrev = obv + 4;
  double* lb = obv + 8;
  const int tctas = tile_ctas(c, cap);
  for (int s = nseg - 1; s >= 0; s--) {
    const int i0 = s * every, i1 = std::min(nsteps, i0 + every);
    ALOAD(s);
    ACK(cudaMemcpyAsync(su, c.u(), nb, cudaMemcpyDeviceToDevice, c.stream));
    ACK(cudaMemcpyAsync(sv, c.v(), nb, cudaMemcpyDeviceToDevice, c.stream));
    for (int i = i0; i < i1; i++) {
      const size_t o = (size_t)(i - i0) * n;
      ARC(step(dts[i], sT + o, sF + o, gait ? su1 + o : nullptr, gait ? sv1 + o : nullptr));
      // what the step leaves, in one launch
      CopyList L{};
      auto add = [&](const void* src, void* dst, size_t bytes) {
        L.src[L.n] = static_cast<const unsigned*>(src);
        L.dst[L.n] = static_cast<unsigned*>(dst);
        L.words[L.n] = bytes / 4;
        L.n++;
      };
      add(c.u(), pu + o, nb);
      add(c.v(), pv + o, nb);
      if (gait) add(c.pres, sp + o, nb);
      if (keepObst) {
        const int j = i - i0;
        const ObstTiles t = tilesAt(j);
        add(c.dshapes, shSnap + j, sizeof(DevShape));
        add(live.tiles, t.tiles, sizeof(int) * cap);
        const double* src[6] = {live.chi, live.udx, live.udy, live.sD, live.sdx, live.sdy};
        double* dst[6] = {t.chi, t.udx, t.udy, t.sD, t.sdx, t.sdy};
        for (int q = 0; q < 6; q++) add(src[q], dst[q], sizeof(double) * tb);
        add(c.chi, chiSnap + o, nb);
      }
      k_copy_many<<<2 * c.sms, 256, 0, c.stream>>>(L);
      ACK(cudaGetLastError());
    }
    for (int i = i1 - 1; i >= i0; i--) {
      const size_t o = (size_t)(i - i0) * n;
      const double dt = dts[i];
      const DevShape* shI = keepObst ? shSnap + (i - i0) : c.dshapes;   // the step's obstacle state
      const ObstTiles tI = tilesAt(i - i0);
      const double* chiI = keepObst ? chiSnap + o : c.chi;
      // the objective's terms of u^(i+1), p^(i+1) and the body velocity
      if (energy) k_adj_probe<<<probeGrid, 256, 0, c.stream>>>(g, bx, pu + o, pv + o, wE, nullptr, lu, lv);
      if (force)
        k_adj_force<<<tctas, dim3(32, 32), 0, c.stream>>>(g, shI, 0, tI, wFx, wFy, wTs[i], 0, lu, lv, nullptr);
      if (bodyTerm) k_adj_add3<<<1, 1, 0, c.stream>>>(lx, wB[0], wB[1], wB[2]);
      if (gait) {
        const size_t og = (size_t)i * n;
        k_adj_geo_pen<<<tctas, dim3(32, 32), 0, c.stream>>>(g, shI, 0, tI, chiI, su1 + o, sv1 + o, sp + o,
            -0.5 * dt / g.h, pu + o, pv + o, lu, lv, wFx, wFy, wTs[i], gG[0] + og, gG[1] + og, gG[2] + og,
            gG[3] + og, gG[4] + og, gCom + 2 * (size_t)i);
      }
      // penalization
      k_adj_pen<<<tctas, dim3(32, 32), 0, c.stream>>>(g, shI, 0, tI, chiI, lu, lv, lx);
      if (freeBody) {
        // the body velocity of the step came from the momentum integrals of
        // the pressure-corrected velocity
        k_adj_solve<<<1, 1, 0, c.stream>>>(shI, 0, lx, lb);
        k_adj_momenta<<<tctas, dim3(32, 32), 0, c.stream>>>(g, shI, 0, tI, lb, lu, lv);
      }
      // pressure correction: lambda_p, the force's pressure term, then the convolution
      k_adj_grad_T<<<grid2, blk2, 0, c.stream>>>(g, -0.5 * dt / g.h, lu, lv, l1);
      if (force)
        k_adj_force<<<tctas, dim3(32, 32), 0, c.stream>>>(g, shI, 0, tI, wFx, wFy, wTs[i], 1, nullptr, nullptr, l1);
      ACK(cudaGetLastError());
      {
        double* const R = c.rhs;
        double* const P = c.pres;
        c.rhs = l1; c.pres = l2; c.solveNoFade = true;
        poisson_solve(c);
        c.rhs = R; c.pres = P; c.solveNoFade = false;
      }
      // the fade, then the obstacle terms, both in place on l2 (over the
      // strip blocks and the shape's tiles)
      ACK(cudaMemsetAsync(acc, 0, sizeof(double) * 8, c.stream));
      k_adj_fade_sums<<<grid2, blk2, 0, c.stream>>>(g, sF + o, l2, acc);
      k_adj_fade_apply<<<grid2, blk2, 0, c.stream>>>(g, sF + o, l2, acc);
      ACK(cudaMemsetAsync(acc, 0, sizeof(double) * 8, c.stream));
      k_adj_obst_sums<<<tctas, dim3(32, 32), 0, c.stream>>>(g, shI, 0, tI, chiI, sT + o, l2, acc);
      if (gait)
        k_adj_geo_obst<<<tctas, dim3(32, 32), 0, c.stream>>>(g, shI, 0, tI, chiI, sT + o, l2, acc,
                                                            gG[0] + (size_t)i * n);
      k_adj_obst_apply<<<tctas, dim3(32, 32), 0, c.stream>>>(g, shI, 0, tI, chiI, sT + o, l2, acc);
      // the divergence, added to lambda of u1
      k_adj_div_T<<<grid2, blk2, 0, c.stream>>>(g, 0.5 * g.h / dt, l2, lu, lv);
      // advDiff about u^i
      ACK(cudaMemsetAsync(acc, 0, sizeof(double) * 8, c.stream));
      k_adj_adv_gamma<<<std::min(148, (2 * (g.nx + g.ny) + 255) / 256), 256, 0, c.stream>>>(g, lu, lv, acc);
      // (a free body: its previous velocity set the lab velocity of this
      // step; a forced one: its held velocity, accumulated)
      const double* un0 = i == i0 ? su : pu + o - n;     // u^n of the step
      const double* vn0 = i == i0 ? sv : pv + o - n;
      k_adj_advdiff<<<grid2, blk2, 0, c.stream>>>(g, adv_coef_host(c, dt, U0s[i], U1s[i]), un0, vn0,
                                                 lu, lv, acc, tu, tv, freeBody ? lxPrev : lx);
      ACK(cudaGetLastError());
      std::swap(lu, tu);
      std::swap(lv, tv);
      if (freeBody) {
        ACK(cudaMemcpyAsync(lx, lxPrev, sizeof(double) * 3, cudaMemcpyDeviceToDevice, c.stream));
        ACK(cudaMemsetAsync(lxPrev, 0, sizeof(double) * 3, c.stream));
      }
    }
  }
  ACK(cudaEventRecord(e1, c.stream));
  if (grad_u) ACK(cudaMemcpyAsync(grad_u, lu, nb, cudaMemcpyDeviceToHost, c.stream));
  if (grad_v) ACK(cudaMemcpyAsync(grad_v, lv, nb, cudaMemcpyDeviceToHost, c.stream));
  if (grad_body) ACK(cudaMemcpyAsync(grad_body, lx, sizeof(double) * 3, cudaMemcpyDeviceToHost, c.stream));
  ACK(cudaStreamSynchronize(c.stream));
  float bms = 0;
  ACK(cudaEventElapsedTime(&bms, e2, e1));
  if (ms) ms[1] = bms;
  if (gait) {
    // d(geometry)/dtheta by central differences of the placement alone: from
    // the run's first checkpoint, each perturbed gait replays the steps'
    // PutObjectsOnGrid (and the step end: time, the next midline) with the
    // frozen dt, and <g, geometry> is summed over the steps
    double theta[CUP2D_GAIT_PARAMS];
    ARC(cup2d_fish_gait_get(ctx, 0, theta));
    const int np = CUP2D_GAIT_PARAMS;
    const double eps = obj->gait_step > 0 ? obj->gait_step : 1e-7;
    for (int q = 0; q < CUP2D_GAIT_PARAMS; q++) grad_gait[q] = 0;
    // one replay: from the first checkpoint, with gait th, on context x
    // (acc: its contraction, a device double of x's)
    auto replay = [&](cup2d_ctx* x, const double* th, double* accx, double* out) -> int {
      Ctx& cx = x->c;
      if (cudaSetDevice(cx.device) != cudaSuccess) return CUP2D_ECUDA;
      int rc = cup2d_fish_gait_set(x, 0, theta);        // the checkpoints' gait
      if (!rc) rc = cup2d_checkpoint_load(x, ck[0], ckBytes);
      if (!rc) rc = cup2d_fish_gait_set(x, 0, th);
      if (rc) return rc;
      if (cudaMemsetAsync(accx, 0, sizeof(double), cx.stream) != cudaSuccess) return CUP2D_ECUDA;
      for (int i = 0; i < nsteps && !rc; i++) {
        rc = cup2d_put_objects(x, dts[i]);
        if (rc) break;
        const size_t og = (size_t)i * n;
        k_adj_geo_dot<<<tctas, dim3(32, 32), 0, cx.stream>>>(g, cx.dshapes, 0, cx.tiles[0], cx.chi, gG[0] + og,
                                                            gG[1] + og, gG[2] + og, gG[3] + og, gG[4] + og,
                                                            gCom + 2 * (size_t)i, accx);
        if (cudaGetLastError() != cudaSuccess) return CUP2D_ECUDA;
        rc = cup2d_end_step(x);
      }
      if (rc) return rc;
      if (cudaMemcpyAsync(out, accx, sizeof(double), cudaMemcpyDeviceToHost, cx.stream) != cudaSuccess ||
          cudaStreamSynchronize(cx.stream) != cudaSuccess) return CUP2D_ECUDA;
      return CUP2D_OK;
    };
    const int nrep = 2 * np;
    std::vector<double> Cpm(nrep, 0.0);
    std::vector<std::array<double, CUP2D_GAIT_PARAMS>> ths(nrep);
    for (int j = 0; j < nrep; j++) {
      std::copy(theta, theta + CUP2D_GAIT_PARAMS, ths[j].begin());
      ths[j][j / 2] += j % 2 == 0 ? eps : -eps;
    }
    // side by side on contexts of this configuration, one host thread each
    // (the replays are latency-bound: the midline and the frame are
    // one-CTA kernels), else one after another on this context
    double* accs = B.get<double>(nrep);
    const bool side = accs && gait_shadows(ctx, nrep);   // (made on first use, not timed)
    // host clock: the replays run on other contexts' streams
    const auto t0 = std::chrono::steady_clock::now();
    if (side) {
      std::vector<int> rcs(nrep, CUP2D_OK);
      std::vector<std::thread> pool;
      for (int j = 0; j < nrep; j++)
        pool.emplace_back([&, j] { rcs[j] = replay(c.gaitShadows[j], ths[j].data(), accs + j, &Cpm[j]); });
      for (std::thread& t : pool) t.join();
      for (int j = 0; j < nrep; j++)
        if (rcs[j]) return adj_fail(ctx, rcs[j], std::string("gait replay: ") + c.gaitShadows[j]->c.err);
    } else {
      for (int j = 0; j < nrep; j++) {
        const int rc = replay(ctx, ths[j].data(), acc, &Cpm[j]);
        if (rc) return rc;
      }
    }
    for (int q = 0; q < np; q++) grad_gait[q] = (Cpm[2 * q] - Cpm[2 * q + 1]) / (2 * eps);
    if (ms) ms[2] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    ARC(cup2d_fish_gait_set(ctx, 0, theta));
  }
  ALOAD(nseg);
  return CUP2D_OK;
}

} // extern "C"
