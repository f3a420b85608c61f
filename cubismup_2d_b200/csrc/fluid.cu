// Dense grid kernels of the timestep: findMaxU + dt, advDiff, the outflow
// correction, the pressure RHS divergence, the fade reductions of cub2rhs,
// the pressure correction, IC and ApplyObjVel.
//
// Every kernel maps one CTA to one 32x32 reference block (blockDim 32x8,
// 4 rows per thread): a warp reads one 256-byte fp64 row segment.  advDiff
// stages its tile with a two-cell halo by TMA; the others take the 5-point
// halo from L1/L2 (neighbour rows are read by the CTA itself, neighbour
// columns by the adjacent CTA), so DRAM sees each plane once.
// Arithmetic is written in the reference's operation order and the library
// is compiled without FMA contraction, so a stage fed the same inputs as the
// reference reproduces it bit for bit (reductions excepted: their order
// differs).
#include <cmath>
#include "context.hpp"
#include "step_begin.cuh"
#include "tma.cuh"

namespace cup2d {

namespace {

__global__ void __launch_bounds__(512)
k_max_u_dt(GridDesc g, Scalars* sc, const DevShape* sh, int nsh,
           const double* __restrict__ u, const double* __restrict__ v,
           double* partials, unsigned* counter)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_MAXU);
  __shared__ double red[64];
  max_u_dt_cta(g, sc, sh, nsh, u, v, partials, counter, red);
}

__global__ void k_set_dt(Scalars* sc, double dt) { pdl_begin(); CUP2D_TRACE_SCOPE(TR_SETDT); sc->dt = dt; }

// End of a step (Simulation.cpp:289-290): t += dt, step += 1, then the next step's
// calcMaxTimestep from the maximum k_pcorr<true> and k_forces formed on the final velocity
// (max is exact in any order: dtNext equals what k_max_u_dt would form).
__global__ void k_end_step_dt(GridDesc g, Scalars* sc, const DevShape* sh, int nsh, double* dtOut,
                              unsigned long long* seqOut, unsigned long long seqVal)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_ENDSTEP);
  const double m = sc->maxNext;
  sc->time += sc->dt;
  sc->step += 1;
  const double dtn = dt_from_max_u(g, sc, sh, nsh, m);
  sc->dtNext = dtn;
  sc->maxUNext = m;
  sc->dtNextValid = 1;
  if (dtOut) *dtOut = dtn;                    // to mapped host memory
  signal_host(seqOut, seqVal);
}

// End of an operator-by-operator step: findMaxU on the final velocity (its
// last CTA), then t += dt, step += 1 and the next step's calcMaxTimestep --
// a graph step's findMaxU parts and k_end_step_dt in one launch.
__global__ void __launch_bounds__(512)
k_end_step_max(GridDesc g, Scalars* sc, const DevShape* sh, int nsh, const double* __restrict__ u,
               const double* __restrict__ v, double* partials, unsigned* counter, double* dtOut,
               unsigned long long* seqOut, unsigned long long seqVal)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_ENDSTEP);
  __shared__ double red[64];
  double m;
  if (!max_u_cta(g, sc, u, v, partials, counter, red, &m)) return;
  sc->time += sc->dt;
  sc->step += 1;
  const double dtn = dt_from_max_u(g, sc, sh, nsh, m);
  sc->dtNext = dtn;
  sc->maxUNext = m;
  sc->dtNextValid = 1;
  if (dtOut) *dtOut = dtn;                    // to mapped host memory
  signal_host(seqOut, seqVal);
}

// calcMaxTimestep of a state whose dt the last step end already formed
// (dtNextValid; nothing has changed the state since): the same values
// k_max_u_dt would write (Simulation.cpp:254-277), taken from dtNext.
__global__ void k_take_dt_next(GridDesc g, Scalars* sc) {
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_SETDT);
  const double dt = sc->dtNext;
  sc->dt = dt;
  sc->maxU = sc->maxUNext;
  if (g.dlm > 0) sc->lambda = g.dlm / dt;
}

// ---- advDiff (advDiff.cpp:14-116) -------------------------------------------
// The step's coefficients dfac = (nu/h)(dt/h), afac = -0.5 dt/h and the
// inflow fades 1 - r^2/100 of r = max/min(U, 0)/max(|U|, eps): seven
// quotients (eleven divisions), each evaluated by its own lane of the warp
// and shared by shuffles -- the same operations as evaluating all of them in
// every thread.  Every lane of the warp calls it.
struct AdvCoef { double afac, dfac, fadeW, fadeS, fadeE, fadeN, U0, U1; };
__device__ __forceinline__ AdvCoef adv_coef(const GridDesc& g, const Scalars* sc) {
  const double dt = sc->dt, h = g.h;
  AdvCoef k;
  k.U0 = sc->uinfx; k.U1 = sc->uinfy;
  double qa = 1.0, qb = 1.0;
  {
    const double norUinf = fmax(fmax(fabs(k.U0), fabs(k.U1)), EPSd);
    switch (lin_tid() & 31) {
      case 0: qa = -0.5 * dt; qb = h; break;
      case 1: qa = g.nu; qb = h; break;
      case 2: qa = dt; qb = h; break;
      case 3: qa = fmax(k.U0, 0.0); qb = norUinf; break;     // W
      case 4: qa = fmax(k.U1, 0.0); qb = norUinf; break;     // S
      case 5: qa = fmin(k.U0, 0.0); qb = norUinf; break;     // E
      case 6: qa = fmin(k.U1, 0.0); qb = norUinf; break;     // N
      default: break;
    }
  }
  const double q = qa / qb, fq = 1 - q * q / 100;
  k.afac = __shfl_sync(0xffffffffu, q, 0);
  k.dfac = __shfl_sync(0xffffffffu, q, 1) * __shfl_sync(0xffffffffu, q, 2);
  k.fadeW = __shfl_sync(0xffffffffu, fq, 3); k.fadeS = __shfl_sync(0xffffffffu, fq, 4);
  k.fadeE = __shfl_sync(0xffffffffu, fq, 5); k.fadeN = __shfl_sync(0xffffffffu, fq, 6);
  return k;
}

// advDiff.cpp:57-87 for cell (gx, gy): the new velocity before the outflow
// correction.  Ghosts: neighbour cells, or at the domain edge the
// zero-gradient copy scaled by the inflow fade of advDiff.cpp:50-55,68-71.
__device__ __forceinline__ void adv_cell(const GridDesc& g, const AdvCoef& k, const double* __restrict__ u,
                                         const double* __restrict__ v, int gx, int gy,
                                         double& unew, double& vnew) {
  const int nx = g.nx, ny = g.ny;
  const size_t c = (size_t)gy * nx + gx;
  const double ucc = u[c], vcc = v[c];
  double ulx, vlx, upx, vpx, uly, vly, upy, vpy;
  if (gx > 0) { ulx = u[c - 1]; vlx = v[c - 1]; } else { ulx = ucc * k.fadeW; vlx = vcc * k.fadeW; }
  if (gx < nx - 1) { upx = u[c + 1]; vpx = v[c + 1]; } else { upx = ucc * k.fadeE; vpx = vcc * k.fadeE; }
  if (gy > 0) { uly = u[c - nx]; vly = v[c - nx]; } else { uly = ucc * k.fadeS; vly = vcc * k.fadeS; }
  if (gy < ny - 1) { upy = u[c + nx]; vpy = v[c + nx]; } else { upy = ucc * k.fadeN; vpy = vcc * k.fadeN; }
  const double dUadv = (ucc + k.U0) * (upx - ulx) + (vcc + k.U1) * (upy - uly);
  const double dUdif = upx + upy + ulx + uly - 4 * ucc;
  const double dVadv = (ucc + k.U0) * (vpx - vlx) + (vcc + k.U1) * (vpy - vly);
  const double dVdif = vpx + vpy + vlx + vly - 4 * vcc;
  unew = ucc + (k.afac * dUadv + k.dfac * dUdif);
  vnew = vcc + (k.afac * dVadv + k.dfac * dVdif);
}

// advDiff.cpp:89-106: the net outflow of the new velocity through the domain
// boundary and its correction per boundary cell.  The boundary cells' new
// values depend on the old velocity only, so they are formed here, before
// the update, with the update's own arithmetic (adv_cell).  Item k walks
// the west column (-u), the east column (+u), the south row (-v) and the
// north row (+v); the CTA sums, then the last CTA sums those in block order.
__global__ void __launch_bounds__(256)
k_outflow_flux(GridDesc g, const Scalars* sc, const double* __restrict__ u, const double* __restrict__ v,
               double* partials, unsigned* counter, Scalars* scw)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_ADVDIFF);
  __shared__ double red[32];
  const AdvCoef kc = adv_coef(g, sc);
  if (blockIdx.x == 0 && threadIdx.x == 0) {            // for the update kernel after this one
    scw->advCoef[0] = kc.afac; scw->advCoef[1] = kc.dfac;
    scw->advCoef[2] = kc.fadeW; scw->advCoef[3] = kc.fadeS;
    scw->advCoef[4] = kc.fadeE; scw->advCoef[5] = kc.fadeN;
    scw->facDiv = 0.5 * g.h / sc->dt;
  }
  const int nx = g.nx, ny = g.ny, nitems = 2 * (nx + ny);
  double IF = 0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nitems; q += gridDim.x * blockDim.x) {
    int gx, gy, comp;
    double sgn;
    if (q < ny) { gx = 0; gy = q; comp = 0; sgn = -1; }
    else if (q < 2 * ny) { gx = nx - 1; gy = q - ny; comp = 0; sgn = 1; }
    else if (q < 2 * ny + nx) { gx = q - 2 * ny; gy = 0; comp = 1; sgn = -1; }
    else { gx = q - 2 * ny - nx; gy = ny - 1; comp = 1; sgn = 1; }
    double un, vn;
    adv_cell(g, kc, u, v, gx, gy, un, vn);
    const double f = comp == 0 ? un : vn;
    if (sgn < 0) IF -= f; else IF += f;
  }
  double s1[1] = {IF};
  block_sum<1>(s1, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = s1[0];
  if (!last_block_done(counter, gridDim.x)) return;
  double t1[1] = {0.0};
  for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) t1[0] += __ldcg(&partials[i]);
  block_sum<1>(t1, red);
  if (threadIdx.x == 0)                                   // advDiff.cpp:105
    scw->outflowCorr = t1[0] / (2 * (BS * g.bpdy - 0) + 2 * (BS * g.bpdx - 0));
}

// adv_cell on the staged tile: U, V hold the block's cells and a two-cell
// halo (tile position (lx + 2, ly + 2) for block cell (lx, ly)); the domain
// edge tests use the global cell (gx, gy), as adv_cell does
// EDGE = false: a cell whose four neighbours are all inside the domain (no
// ghost tests); COMP: both components (2), or only u (0) or v (1).  The
// same expressions in every case.
template <bool EDGE = true, int COMP = 2>
__device__ __forceinline__ void adv_cell_tile(const GridDesc& g, const AdvCoef& k, const double* U,
                                              const double* V, int lx, int ly, int gx, int gy,
                                              double& unew, double& vnew) {
  const int t = (ly + 2) * ADV_HT + lx + 2;
  const double ucc = U[t], vcc = V[t];
  double ulx, vlx, upx, vpx, uly, vly, upy, vpy;
  if (!EDGE || gx > 0) { ulx = U[t - 1]; vlx = V[t - 1]; } else { ulx = ucc * k.fadeW; vlx = vcc * k.fadeW; }
  if (!EDGE || gx < g.nx - 1) { upx = U[t + 1]; vpx = V[t + 1]; } else { upx = ucc * k.fadeE; vpx = vcc * k.fadeE; }
  if (!EDGE || gy > 0) { uly = U[t - ADV_HT]; vly = V[t - ADV_HT]; } else { uly = ucc * k.fadeS; vly = vcc * k.fadeS; }
  if (!EDGE || gy < g.ny - 1) { upy = U[t + ADV_HT]; vpy = V[t + ADV_HT]; } else { upy = ucc * k.fadeN; vpy = vcc * k.fadeN; }
  if (COMP != 1) {
    const double dUadv = (ucc + k.U0) * (upx - ulx) + (vcc + k.U1) * (upy - uly);
    const double dUdif = upx + upy + ulx + uly - 4 * ucc;
    unew = ucc + (k.afac * dUadv + k.dfac * dUdif);
  }
  if (COMP != 0) {
    const double dVadv = (ucc + k.U0) * (vpx - vlx) + (vcc + k.U1) * (vpy - vly);
    const double dVdif = vpx + vpy + vlx + vly - 4 * vcc;
    vnew = vcc + (k.afac * dVadv + k.dfac * dVdif);
  }
}

// k_advdiff after its tiles landed: the update with the outflow
// correction, the halo of the new velocity, the divergence and the fade
// sums.  EDGE = false for a block away from the domain edge.
template <bool EDGE>
__device__ __forceinline__ void advdiff_tile_body(const GridDesc& g, const AdvCoef& kc, const double* tU,
                                                  const double* tV, double (*su)[BS + 2], double (*sv)[BS],
                                                  double corr, double facDiv, double* __restrict__ un,
                                                  double* __restrict__ vn, double* __restrict__ rhs,
                                                  const int* __restrict__ fadeSlot,
                                                  double* __restrict__ fadePartials) {
  const int bx = blockIdx.x, by = blockIdx.y, tx = threadIdx.x, ty = threadIdx.y, tid = lin_tid();
  const int nx = g.nx, ny = g.ny;
  const int gx = bx * BS + tx;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int iy = ty + 8 * r, gy = by * BS + iy;
    double unew, vnew;
    adv_cell_tile<EDGE>(g, kc, tU, tV, tx, iy, gx, gy, unew, vnew);
    if (EDGE) {
      if (gx == 0) unew = unew + corr;                   // advDiff.cpp:107-115
      if (gx == nx - 1) unew = unew - corr;
      if (gy == 0) vnew = vnew + corr;
      if (gy == ny - 1) vnew = vnew - corr;
    }
    const size_t c = (size_t)gy * nx + gx;
    un[c] = unew; vn[c] = vnew;
    su[iy][tx + 1] = unew; sv[iy + 1][tx] = vnew;
  }
  // halo: warps 0-3, one lane per cell (u west / east column, v south /
  // north row of the neighbouring blocks)
  if (ty < 4) {
    const int side = ty;
    const bool have = side == 0 ? bx > 0 : side == 1 ? bx < g.bpdx - 1 : side == 2 ? by > 0 : by < g.bpdy - 1;
    if (have) {
      const int lx = side == 0 ? -1 : side == 1 ? BS : tx;
      const int ly = side == 2 ? -1 : side == 3 ? BS : tx;
      double unew, vnew;
      if (side < 2) {                                  // only u of the west / east columns
        adv_cell_tile<EDGE, 0>(g, kc, tU, tV, lx, ly, bx * BS + lx, by * BS + ly, unew, vnew);
        su[tx][side == 0 ? 0 : BS + 1] = unew;
      } else {                                         // only v of the south / north rows
        adv_cell_tile<EDGE, 1>(g, kc, tU, tV, lx, ly, bx * BS + lx, by * BS + ly, unew, vnew);
        sv[side == 2 ? 0 : BS + 1][tx] = vnew;
      }
    }
  }
  __syncthreads();
  const bool touch = fade_touch(g, bx, by);
  double s[3] = {0, 0, 0};
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int iy = ty + 8 * r, gy = by * BS + iy;
    const double uW = !EDGE || gx > 0 ? su[iy][tx] : su[iy][tx + 1];
    const double uE = !EDGE || gx < nx - 1 ? su[iy][tx + 2] : su[iy][tx + 1];
    const double vS = !EDGE || gy > 0 ? sv[iy][tx] : sv[iy + 1][tx];
    const double vN = !EDGE || gy < ny - 1 ? sv[iy + 2][tx] : sv[iy + 1][tx];
    const double divVx = uE - uW, divVy = vN - vS;
    const double b = facDiv * (divVx + divVy);
    rhs[(size_t)gy * nx + gx] = b;
    if (touch) fade_accumulate(g, bx, by, tx, iy, b, s);
  }
  if (touch) {                                         // uniform over the CTA
    __shared__ double red[96];
    block_sum<3>(s, red);
    if (tid == 0) {
      const int q = fadeSlot[bx + g.bpdx * by];
      for (int k = 0; k < 3; k++) fadePartials[3 * q + k] = s[k];
    }
  }
}

// advDiff.cpp:57-116 with PressureSingle.cpp:112-128 in place, one CTA per
// 32x32 block: one thread loads the block's u and v with a two-cell halo by
// TMA (the halo beyond the domain reads as zero and is never used: edge
// cells take the reference's ghosts instead), the CTA forms the new
// velocity with the outflow correction of k_outflow_flux on the boundary
// cells (u on the west / east columns, v on the south / north rows), keeps
// it in shared memory with the new u one column and the new v one row
// beyond the block (formed here too: they are never on the boundary
// column or row whose correction they would need; at the domain edge the
// zero-gradient ghost is the cell itself), and writes the divergence RHS
// and the strip blocks' fade sums.  Thread (tx, ty) of 32 x 8 takes rows
// ty + 8 r, the order of every producer of the fade sums.  The tile
// barrier's wait is bounded: a load that never lands raises ST_TIMEOUT.
__global__ void __launch_bounds__(256, 4)
k_advdiff(const __grid_constant__ CUtensorMap tmU, const __grid_constant__ CUtensorMap tmV,
          GridDesc g, Scalars* sc, unsigned txBytes,
          double* __restrict__ un, double* __restrict__ vn,
          double* __restrict__ rhs, const int* __restrict__ fadeSlot, double* __restrict__ fadePartials)
{
  __shared__ __align__(128) double tU[ADV_HT * ADV_HT];
  __shared__ __align__(128) double tV[ADV_HT * ADV_HT];
  __shared__ __align__(8) unsigned long long bar;
  __shared__ double su[BS][BS + 2];
  __shared__ double sv[BS + 2][BS];
  const int tid = lin_tid();
  if (tid == 0) mbar_init(&bar, 1);
  __syncthreads();
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_ADVDIFF);
  const int bx = blockIdx.x, by = blockIdx.y, tx = threadIdx.x, ty = threadIdx.y;
  if (tid == 0) {
    mbar_arrive_expect_tx(&bar, txBytes);
    tma_load_2d(tU, &tmU, bx * BS - 2, by * BS - 2, &bar);
    tma_load_2d(tV, &tmV, bx * BS - 2, by * BS - 2, &bar);
  }
  // the step's coefficients, as k_outflow_flux (launched before every
  // update) formed them, read while the tiles are in flight
  AdvCoef kc;
  kc.afac = sc->advCoef[0]; kc.dfac = sc->advCoef[1];
  kc.fadeW = sc->advCoef[2]; kc.fadeS = sc->advCoef[3];
  kc.fadeE = sc->advCoef[4]; kc.fadeN = sc->advCoef[5];
  kc.U0 = sc->uinfx; kc.U1 = sc->uinfy;
  const double corr = sc->outflowCorr;
  const double facDiv = sc->facDiv;
  const int nx = g.nx, ny = g.ny;
  const int gx = bx * BS + tx;
  // one thread waits for the tiles (the others at the CTA barrier, where
  // they take no issue slots); its acquire of the barrier's phase and the
  // CTA barrier make the tiles visible to every thread
  bool landed = true;
  if (tid == 0) landed = mbar_wait_bounded(&bar, 0, TMA_WAIT_NS);
  if (__syncthreads_or(!landed)) {
    // the loads did not land: report, give them the same time again (the
    // CTA's shared memory stays while thread 0 waits), leave
    if (tid == 0) {
      atomicOr(&sc->status, ST_TIMEOUT);
      mbar_wait_bounded(&bar, 0, TMA_WAIT_NS);
    }
    return;
  }
  // blocks away from the domain edge: no ghost, outflow or one-sided tests
  if (bx > 0 && by > 0 && bx < g.bpdx - 1 && by < g.bpdy - 1)
    advdiff_tile_body<false>(g, kc, tU, tV, su, sv, corr, facDiv, un, vn, rhs, fadeSlot, fadePartials);
  else
    advdiff_tile_body<true>(g, kc, tU, tV, su, sv, corr, facDiv, un, vn, rhs, fadeSlot, fadePartials);
}

// PressureSingle.cpp:112-128: tmp = (h / 2dt) * div_2h(u); zero-gradient ghosts
__global__ void __launch_bounds__(256)
k_rhs_div(GridDesc g, const Scalars* sc, const double* __restrict__ u,
          const double* __restrict__ v, double* __restrict__ rhs,
          const int* __restrict__ fadeSlot, double* __restrict__ fadePartials)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_RHSDIV);
  const double h = g.h, facDiv = 0.5 * h / sc->dt;
  const int nx = g.nx, ny = g.ny;
  const int bx = blockIdx.x, by = blockIdx.y;
  const int gx = bx * BS + threadIdx.x;
  const bool touch = fade_touch(g, bx, by);
  if (!touch && bx > 0 && by > 0 && bx < g.bpdx - 1 && by < g.bpdy - 1) {
    // a block away from the domain edge and the fade band (uniform over the
    // CTA): no ghosts and no fade sums.  Two cells per thread with 16-byte
    // loads; a half-warp covers one tile row, and each lane takes its x
    // neighbours from the adjacent lanes (the half-row's ends load theirs).
    // The same expression per cell as below.
    const int p = threadIdx.x & 15, half = threadIdx.x >> 4;
    const int gx0 = bx * BS + 2 * p;
#pragma unroll
    for (int r = 0; r < 2; r++) {
      const int gy = by * BS + 2 * threadIdx.y + half + 16 * r;
      const size_t c = (size_t)gy * nx + gx0;
      const double2 uc = *reinterpret_cast<const double2*>(u + c);
      const double2 vS = *reinterpret_cast<const double2*>(v + c - nx);
      const double2 vN = *reinterpret_cast<const double2*>(v + c + nx);
      double uW = __shfl_up_sync(0xffffffffu, uc.y, 1, 16);     // u[c - 1]
      double uE = __shfl_down_sync(0xffffffffu, uc.x, 1, 16);   // u[c + 2]
      if (p == 0) uW = u[c - 1];
      if (p == 15) uE = u[c + 2];
      const double b0 = facDiv * ((uc.y - uW) + (vN.x - vS.x));
      const double b1 = facDiv * ((uE - uc.x) + (vN.y - vS.y));
      *reinterpret_cast<double2*>(rhs + c) = make_double2(b0, b1);
    }
    return;
  }
  double s[3] = {0, 0, 0};
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int iy = threadIdx.y + 8 * r, gy = by * BS + iy;
    const size_t c = (size_t)gy * nx + gx;
    const double uW = u[gx > 0 ? c - 1 : c], uE = u[gx < nx - 1 ? c + 1 : c];
    const double vS = v[gy > 0 ? c - nx : c], vN = v[gy < ny - 1 ? c + nx : c];
    const double divVx = uE - uW, divVy = vN - vS;
    const double b = facDiv * (divVx + divVy);
    rhs[c] = b;
    if (touch) fade_accumulate(g, bx, by, threadIdx.x, iy, b, s);
  }
  // a strip block's fade sums of the RHS as it leaves the divergence; the
  // obstacle terms rewrite those of their own tiles
  if (touch) {
    __shared__ double red[96];
    block_sum<3>(s, red);
    if (lin_tid() == 0) {
      const int q = fadeSlot[bx + g.bpdx * by];
      for (int k = 0; k < 3; k++) fadePartials[3 * q + k] = s[k];
    }
  }
}

// cub2rhs's strip sums (PoissonSolver.cpp:61-100) of a plane as it is, for
// a Poisson solve called on its own: the same per-block order as the RHS
// kernels' (32 x 8 threads, rows ty + 8r), written to the strip slots.
__global__ void __launch_bounds__(256)
k_fade_sums(GridDesc g, const double* __restrict__ rhs, const int* __restrict__ fadeSlot,
            double* __restrict__ fadePartials)
{
  pdl_begin();
  const int bx = blockIdx.x, by = blockIdx.y;
  if (!fade_touch(g, bx, by)) return;                  // uniform over the CTA
  const int gx = bx * BS + threadIdx.x;
  double s[3] = {0, 0, 0};
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int iy = threadIdx.y + 8 * r;
    fade_accumulate(g, bx, by, threadIdx.x, iy, rhs[(size_t)(by * BS + iy) * g.nx + gx], s);
  }
  __shared__ double red[96];
  block_sum<3>(s, red);
  if (lin_tid() == 0) {
    const int q = fadeSlot[bx + g.bpdx * by];
    for (int k = 0; k < 3; k++) fadePartials[3 * q + k] = s[k];
  }
}

// PressureIterator_unif::updatePressureRHS (PressureIterator_unif.cpp:22-49):
// tmp = (h/2dt) (div V - chi div UDEF) on the penalized velocity and the
// grid's deformation velocity, zero-gradient ghosts for both (the same
// VectorLab), with the fade sums of the strip blocks as k_rhs_div forms them.
__global__ void __launch_bounds__(256)
k_rhs_iter(GridDesc g, const Scalars* sc, const double* __restrict__ u, const double* __restrict__ v,
           const double* __restrict__ udx, const double* __restrict__ udy, const double* __restrict__ chi,
           double* __restrict__ rhs, const int* __restrict__ fadeSlot, double* __restrict__ fadePartials)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_RHSDIV);
  const double h = g.h, facDiv = 0.5 * h / sc->dt;
  const int nx = g.nx, ny = g.ny;
  const int bx = blockIdx.x, by = blockIdx.y;
  const int gx = bx * BS + threadIdx.x;
  const bool touch = fade_touch(g, bx, by);
  double s[3] = {0, 0, 0};
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int iy = threadIdx.y + 8 * r, gy = by * BS + iy;
    const size_t c = (size_t)gy * nx + gx;
    const size_t cW = gx > 0 ? c - 1 : c, cE = gx < nx - 1 ? c + 1 : c;
    const size_t cS = gy > 0 ? c - nx : c, cN = gy < ny - 1 ? c + nx : c;
    const double divVx = u[cE] - u[cW], divVy = v[cN] - v[cS];
    const double divUSx = udx[cE] - udx[cW], divUSy = udy[cN] - udy[cS];
    const double b = facDiv * (divVx + divVy - chi[c] * (divUSx + divUSy));
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

// fadeSlot[b] = rank of block b among the strip blocks (block order), or -1;
// fadeSlot[nblocks] = their number.  Once per grid, one thread.
__global__ void k_fade_slots(GridDesc g, int* fadeSlot)
{
  int n = 0;
  for (int b = 0; b < g.nblocks; b++) fadeSlot[b] = fade_touch(g, b % g.bpdx, b / g.bpdx) ? n++ : -1;
  fadeSlot[g.nblocks] = n;
}

// PressureSingle.cpp:216-241: V += -(dt/2h) grad_2h P; zero-gradient P ghosts.
// Reads the velocity written by advDiff (ui, vi) and writes the current one.
// MAXNEXT (graph steps): the next step's findMaxU (Helpers.cpp:136-176) is
// formed on the step's final velocity in two parts meeting in sc->maxNext by
// exact atomic max: here over the blocks no shape has a tile in (the
// penalization leaves them as they are), and by the force pass over the
// tiles once they are penalized.
template <bool MAXNEXT>
__global__ void __launch_bounds__(256)
k_pcorr(GridDesc g, Scalars* sc, AllTiles T, int nsh, const double* __restrict__ p,
        const double* __restrict__ ui, const double* __restrict__ vi,
        double* __restrict__ uo, double* __restrict__ vo)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_PCORR);
  const double pFac = -0.5 * sc->dt / g.h;
  const double UINF = sc->uinfx, VINF = sc->uinfy;
  const int nx = g.nx, ny = g.ny;
  const int gx = blockIdx.x * BS + threadIdx.x;
  double m = 0.0;
  int bad = 0;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int gy = blockIdx.y * BS + threadIdx.y + 8 * r;
    const size_t c = (size_t)gy * nx + gx;
    const double pW = p[gx > 0 ? c - 1 : c], pE = p[gx < nx - 1 ? c + 1 : c];
    const double pS = p[gy > 0 ? c - nx : c], pN = p[gy < ny - 1 ? c + nx : c];
    const double un = ui[c] + pFac * (pE - pW), vn = vi[c] + pFac * (pN - pS);
    uo[c] = un;
    vo[c] = vn;
    if (MAXNEXT) {
      m = fmax(m, cell_speed(un, vn, UINF, VINF));
      bad |= !isfinite(un) || !isfinite(vn);
    }
  }
  if (!MAXNEXT) return;
  const int b = blockIdx.x + g.bpdx * blockIdx.y;
  bool tile = false;
  for (int k = 0; k < nsh; k++) tile |= T.t[k].slot[b] >= 0;
  if (tile) return;                                    // uniform over the CTA
  __shared__ double red[32];
  m = block_max(m, red);
  const int anyBad = __syncthreads_or(bad);
  if (lin_tid() == 0) {
    atomic_max_nonneg(&sc->maxNext, m);
    if (anyBad) atomicOr(&sc->status, ST_NAN);
  }
}

__global__ void k_ic(size_t n, double* u, double* v, double* chi, double* pres,
                     double* rhs, double* sdf, double* udx, double* udy)
{
  pdl_begin();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    u[i] = 0; v[i] = 0; chi[i] = 0; pres[i] = 0; rhs[i] = 0;
    sdf[i] = -1; udx[i] = 0; udy[i] = 0;
  }
}

// Helpers.cpp:290-307: u <- u (1 - chi) + udef chi
__global__ void k_apply_obj_vel(size_t n, double* u, double* v, const double* chi,
                                const double* udx, const double* udy)
{
  pdl_begin();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double X = chi[i];
    u[i] = u[i] * (1 - X) + udx[i] * X;
    v[i] = v[i] * (1 - X) + udy[i] * X;
  }
}

inline int reduce_grid(const Ctx& c) {
  int n = (int)((c.ncells() + 255) / 256);
  return n < 148 * 8 ? n : 148 * 8;
}
inline int max_grid(const Ctx& c) {
  int n = (int)((c.ncells() / 2 + 511) / 512);
  return n < 148 * 2 ? n : 148 * 2;
}

} // namespace

void launch_max_u_dt(Ctx& c) {
  const int nb = max_grid(c);
  launch_k(k_max_u_dt, nb, 512, 0, c.stream, c.g, c.dsc, c.dshapes, c.nshapes, c.u(), c.v(),
                                        c.partials, c.counters + CNT_MAXU);
  CUP2D_LAUNCHED(c);
}

void launch_set_dt(Ctx& c, double dt) {
  launch_k(k_set_dt, 1, 1, 0, c.stream, c.dsc, dt);
  CUP2D_LAUNCHED(c);
}

void launch_end_step_max(Ctx& c, double* dtOut, unsigned long long* seqOut, unsigned long long seqVal) {
  launch_k(k_end_step_max, max_grid(c), 512, 0, c.stream, c.g, c.dsc, (const DevShape*)c.dshapes, c.nshapes,
           (const double*)c.u(), (const double*)c.v(), c.partials, c.counters + CNT_MAXU, dtOut, seqOut, seqVal);
  CUP2D_LAUNCHED(c);
}

void launch_take_dt_next(Ctx& c) {
  launch_k(k_take_dt_next, 1, 1, 0, c.stream, c.g, c.dsc);
  CUP2D_LAUNCHED(c);
}

void launch_end_step_dt(Ctx& c, double* dtOut, unsigned long long* seqOut, unsigned long long seqVal) {
  launch_k(k_end_step_dt, 1, 1, 0, c.stream, c.g, c.dsc, (const DevShape*)c.dshapes, c.nshapes, dtOut,
           seqOut, seqVal);
  CUP2D_LAUNCHED(c);
}

void launch_outflow_flux(Ctx& c) {
  const int items = 2 * (c.g.nx + c.g.ny);
  int grid = (items + 255) / 256;
  if (grid > c.sms) grid = c.sms;
  launch_k(k_outflow_flux, grid, 256, 0, c.stream, c.g, (const Scalars*)c.dsc, (const double*)c.u(),
           (const double*)c.v(), c.partials, c.counters + CNT_ADV, c.dsc);
  CUP2D_LAUNCHED(c);
}

void launch_advdiff_rhs_div(Ctx& c) {
  dim3 grid(c.g.bpdx, c.g.bpdy), block(32, 8);
  launch_k(k_advdiff, grid, block, 0, c.stream, c.tmVel[c.cur][0], c.tmVel[c.cur][1], c.g, c.dsc, c.advTx,
           c.uo(), c.vo(), c.rhs, (const int*)c.fadeSlot, fade_partials(c));
  CUP2D_LAUNCHED(c);
  c.cur = 1 - c.cur;
}

// timing helpers: return the velocity to the buffer it came from (no launch)
void launch_advdiff_undo(Ctx& c) { c.cur = 1 - c.cur; }
void launch_pcorr_undo(Ctx& c) { c.cur = 1 - c.cur; }

void launch_fade_sums(Ctx& c) {
  launch_k(k_fade_sums, dim3(c.g.bpdx, c.g.bpdy), dim3(32, 8), 0, c.stream, c.g, (const double*)c.rhs,
           (const int*)c.fadeSlot, fade_partials(c));
  CUP2D_LAUNCHED(c);
}

void launch_rhs_div(Ctx& c) {
  dim3 grid(c.g.bpdx, c.g.bpdy), block(32, 8);
  launch_k(k_rhs_div, grid, block, 0, c.stream, c.g, c.dsc, c.u(), c.v(), c.rhs, (const int*)c.fadeSlot,
           fade_partials(c));
  CUP2D_LAUNCHED(c);
}

int build_fade_slots(Ctx& c) {
  k_fade_slots<<<1, 1, 0, c.stream>>>(c.g, c.fadeSlot);
  int n = -1;
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(&n, c.fadeSlot + c.g.nblocks, sizeof(int), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
      cudaStreamSynchronize(c.stream) != cudaSuccess) return -1;
  return n;
}

void launch_rhs_iter(Ctx& c) {
  dim3 grid(c.g.bpdx, c.g.bpdy), block(32, 8);
  launch_k(k_rhs_iter, grid, block, 0, c.stream, c.g, (const Scalars*)c.dsc, (const double*)c.u(),
           (const double*)c.v(), (const double*)c.udefx, (const double*)c.udefy, (const double*)c.chi,
           c.rhs, (const int*)c.fadeSlot, fade_partials(c));
  CUP2D_LAUNCHED(c);
}

void launch_pcorr_from(Ctx& c, const double* ui, const double* vi, double* uo, double* vo) {
  dim3 grid(c.g.bpdx, c.g.bpdy), block(32, 8);
  launch_k(k_pcorr<false>, grid, block, 0, c.stream, c.g, c.dsc, AllTiles{}, 0, (const double*)c.pres, ui, vi,
           uo, vo);
  CUP2D_LAUNCHED(c);
}

void launch_pcorr(Ctx& c, bool maxNext) {
  dim3 grid(c.g.bpdx, c.g.bpdy), block(32, 8);
  if (maxNext)
    launch_k(k_pcorr<true>, grid, block, 0, c.stream, c.g, c.dsc, all_tiles(c), c.nshapes, (const double*)c.pres,
             (const double*)c.u(), (const double*)c.v(), c.uo(), c.vo());
  else
    launch_k(k_pcorr<false>, grid, block, 0, c.stream, c.g, c.dsc, AllTiles{}, 0, (const double*)c.pres,
             (const double*)c.u(), (const double*)c.v(), c.uo(), c.vo());
  CUP2D_LAUNCHED(c);
  c.cur = 1 - c.cur;
}

void launch_ic(Ctx& c) {
  launch_k(k_ic, reduce_grid(c), 256, 0, c.stream, c.ncells(), c.u(), c.v(), c.chi, c.pres, c.rhs,
                                              c.sdf, c.udefx, c.udefy);
  CUP2D_LAUNCHED(c);
}

void launch_apply_obj_vel(Ctx& c) {
  launch_k(k_apply_obj_vel, reduce_grid(c), 256, 0, c.stream, c.ncells(), c.u(), c.v(), c.chi,
                                                         c.udefx, c.udefy);
  CUP2D_LAUNCHED(c);
}

} // namespace cup2d

#ifdef CUP2D_TRACE
namespace cup2d { void trace_bind_fluid(unsigned long long* p) { trace_bind_this_unit(p); } }
#endif
