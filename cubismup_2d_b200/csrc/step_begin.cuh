// Start of a step, shared by the stand-alone kernels (calcMaxTimestep,
// PutObjectsOnGrid's motion update) and the fused step-begin kernel of the
// step graph.
#pragma once
#include "internal.cuh"
#include "rigid_body.cuh"

namespace cup2d {

// Small device regions the start of a step reads with dependent loads (the
// scalars, the shapes, the fish midline arrays): the step-begin kernel
// prefetches them into L2 first, one region per CTA.
constexpr int MAX_PREFETCH = 8;
struct PrefetchList {
  const char* p[MAX_PREFETCH];
  size_t bytes[MAX_PREFETCH];
  int n;
};

__device__ __forceinline__ void prefetch_region(const PrefetchList& pf, int r) {
  if (r >= pf.n) return;
  const char* base = pf.p[r];
  for (size_t o = (size_t)lin_tid() * 128; o < pf.bytes[r]; o += (size_t)lin_nthreads() * 128)
    asm volatile("prefetch.global.L2 [%0];" :: "l"(base + o));
}

// Helpers.cpp:160-166: the velocity magnitude findMaxU maximises for one cell
__device__ __forceinline__ double cell_speed(double u, double v, double UINF, double VINF) {
  return fmax(fmax(fabs(u + UINF), fabs(v + VINF)), fmax(fabs(u), fabs(v)));
}

// Simulation::calcMaxTimestep (Simulation.cpp:254-277) from the maximum
// speed; one thread.
__device__ __forceinline__ double dt_from_max_u(const GridDesc& g, const Scalars* sc, const DevShape* sh,
                                                int nsh, double maxU) {
  const double h = g.h;
  const double dtFourier = h * h / g.nu, dtCFL = maxU < 2.2e-16 ? 1 : h / maxU;
  double maxUb = 0;                                   // SimulationData::maxRelSpeed
  for (int k = 0; k < nsh; k++) {
    const double su = sh[k].s.u, sv = sh[k].s.v;
    maxUb = fmax(maxUb, sqrt(su * su + sv * sv));     // Shape::getMaxVel
  }
  const double dtBody = maxUb < 2.2e-16 ? 1 : h / maxUb;
  double mn = dtCFL;
  if (dtFourier < mn) mn = dtFourier;
  if (dtBody < mn) mn = dtBody;
  double dt = g.CFL * mn;
  if (sc->step < 100) dt = sc->rampCFL[sc->step] * mn;
  return dt;
}

// Helpers.cpp:136-176 (findMaxU) over a 1D grid: per-CTA maxima, met by the
// last CTA (max is exact in any order).  Returns true in thread 0 of that
// CTA, with the maximum in *mmax.  red must hold 64 doubles.
__device__ __forceinline__ bool max_u_cta(const GridDesc& g, Scalars* sc,
                                          const double* __restrict__ u, const double* __restrict__ v,
                                          double* partials, unsigned* counter, double* red, double* mmax)
{
  const double UINF = sc->uinfx, VINF = sc->uinfy;
  double m = 0.0; int bad = 0;
  const size_t n2 = (size_t)g.nx * g.ny / 2;        // Nx is a multiple of 32
  const double2* u2 = reinterpret_cast<const double2*>(u);
  const double2* v2 = reinterpret_cast<const double2*>(v);
  // Helpers.cpp:160-166: max of |u+uinf|, |v+vinf|, |u|, |v| (four
  // iterations' loads issued before their maxima, for bytes in flight)
  auto take = [&](double2 a2, double2 b2) {
    m = fmax(m, cell_speed(a2.x, b2.x, UINF, VINF));
    m = fmax(m, cell_speed(a2.y, b2.y, UINF, VINF));
    bad |= !isfinite(a2.x) || !isfinite(b2.x) || !isfinite(a2.y) || !isfinite(b2.y);
  };
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  // the last pass's loads are predicated rather than issued one at a
  // time, so that the tail keeps four of them in flight too
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n2; i += 4 * stride) {
    double2 a2[4], b2[4];
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (i + q * stride < n2) { a2[q] = u2[i + q * stride]; b2[q] = v2[i + q * stride]; }
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (i + q * stride < n2) take(a2[q], b2[q]);
  }
  m = block_max(m, red);
  const int anyBad = __syncthreads_or(bad);
  if (lin_tid() == 0) {
    partials[blockIdx.x] = m;
    if (anyBad) atomicOr(&sc->status, ST_NAN);
  }
  if (!last_block_done(counter, gridDim.x)) return false;
  double mm = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) mm = fmax(mm, __ldcg(&partials[i]));
  mm = block_max(mm, red);
  if (threadIdx.x != 0) return false;
  *mmax = mm;
  return true;
}

// findMaxU + Simulation::calcMaxTimestep (Simulation.cpp:254-277): the last
// CTA forms dt.  Returns true in thread 0 of the CTA that set sc->dt.
__device__ __forceinline__ bool max_u_dt_cta(const GridDesc& g, Scalars* sc, const DevShape* sh, int nsh,
                                             const double* __restrict__ u, const double* __restrict__ v,
                                             double* partials, unsigned* counter, double* red)
{
  double mm;
  if (!max_u_cta(g, sc, u, v, partials, counter, red, &mm)) return false;
  const double dt = dt_from_max_u(g, sc, sh, nsh, mm);
  sc->dt = dt;
  sc->maxU = mm;
  if (g.dlm > 0) sc->lambda = g.dlm / dt;
  return true;
}

// The PID controllers of StefanFish::create (StefanFish.cpp:264-364), run
// after every body has moved and before the midline of this step is formed:
// exponential averages of the lateral offset, the angle and the angular
// velocity, then the curvature correction (-pid: the angle; -pidpos: the
// position, also through the tail period).
__device__ __forceinline__ void fish_pid(const Scalars* sc, DevShape& S)
{
  FishCtl& C = S.ctl;
  const ShapeCfg& f = S.cfg;
  const double Tperiod = f.Tperiod, length = f.length;
  const double DT = sc->dt / Tperiod, time = sc->time;
  const double xDiff = (S.s.com[0] - f.origC[0]) / length;
  const double yDiff = (S.s.com[1] - f.origC[1]) / length;
  const double angDiff = S.s.orientation - f.origAng;
  const double relU = (S.s.u + sc->uinfx) / length;
  const double relV = (S.s.v + sc->uinfy) / length;
  const double angVel = S.s.omega, lastAngVel = C.lastAvel;
  const double aVelMidP = (angVel + lastAngVel) * Tperiod / 2;
  const double aVelDiff = (angVel - lastAngVel) * Tperiod / sc->dt;
  C.lastAvel = angVel;
  const double velDAavg = (angDiff - C.avgDangle) / Tperiod + DT * angVel;
  const double velDYavg = (yDiff - C.avgDeltaY) / Tperiod + DT * relV;
  const double velAVavg = 10 * ((aVelMidP - C.avgAngVel) / Tperiod + DT * aVelDiff);
  C.avgDangle = (1.0 - DT) * C.avgDangle + DT * angDiff;
  C.avgDeltaY = (1.0 - DT) * C.avgDeltaY + DT * yDiff;
  C.avgAngVel = (1 - 10 * DT) * C.avgAngVel + 10 * DT * aVelMidP;
  const double avgDangle = C.avgDangle, avgDeltaY = C.avgDeltaY;
  const double absPy = fabs(yDiff), absIy = fabs(avgDeltaY);
  const double velAbsPy = yDiff > 0 ? relV : -relV;
  const double velAbsIy = avgDeltaY > 0 ? velDYavg : -velDYavg;
  if (f.pidpos && sc->dt > 0) {
    const double IangPdy = (avgDangle * yDiff < 0) ? avgDangle * absPy : 0;
    const double PangIdy = (angDiff * avgDeltaY < 0) ? angDiff * absIy : 0;
    const double IangIdy = (avgDangle * avgDeltaY < 0) ? avgDangle * absIy : 0;
    const double velIangPdy = velAbsPy * avgDangle + absPy * velDAavg;
    const double velPangIdy = velAbsIy * angDiff + absIy * angVel;
    const double velIangIdy = velAbsIy * avgDangle + absIy * velDAavg;
    const double coefIangPdy = avgDangle * yDiff < 0 ? 1 : 0;
    const double coefPangIdy = angDiff * avgDeltaY < 0 ? 1 : 0;
    const double coefIangIdy = avgDangle * avgDeltaY < 0 ? 1 : 0;
    const double valIangPdy = coefIangPdy * IangPdy, difIangPdy = coefIangPdy * velIangPdy;
    const double valPangIdy = coefPangIdy * PangIdy, difPangIdy = coefPangIdy * velPangIdy;
    const double valIangIdy = coefIangIdy * IangIdy, difIangIdy = coefIangIdy * velIangIdy;
    const double periodFac = 1.0 - xDiff, periodVel = -relU;
    C.pidFac = valIangPdy + valPangIdy + valIangIdy;      // correctTrajectory
    C.pidDif = difIangPdy + difPangIdy + difIangIdy;
    // correctTailPeriod (StefanFish.cpp:92-106)
    const double lastArg = (C.lastTime - C.time0) / C.periodPIDval + C.timeshift;
    C.time0 = C.lastTime;
    C.timeshift = lastArg;
    C.periodPIDval = Tperiod * periodFac;
    C.periodPIDdif = Tperiod * periodVel;
    C.lastTime = time;
    C.TperiodPID = 1;
  } else if (f.pid && sc->dt > 0) {
    const double avgAngVel = C.avgAngVel, absAngVel = fabs(avgAngVel);
    const double absAvelDiff = avgAngVel > 0 ? velAVavg : -velAVavg;
    const double coefInst = angDiff * avgAngVel > 0 ? 0.01 : 1, coefAvg = 0.1;
    const double termInst = angDiff * absAngVel;
    const double diffInst = angDiff * absAvelDiff + angVel * absAngVel;
    C.pidFac = coefInst * termInst + coefAvg * avgDangle;
    C.pidDif = coefInst * diffInst + coefAvg * velDAavg;
  }
}

// PutObjectsOnGrid.cpp:201-220 (one thread): lab velocity from fixed
// bodies, then Shape::updatePosition; a body whose centre leaves the domain
// raises ST_DOMAIN (the reference exits).  Then the PID controllers of the
// swimmers that have them (StefanFish::create runs after every body moved).
__device__ __forceinline__ void bodies_motion(const GridDesc& g, Scalars* sc, DevShape* sh, int nsh)
{
  const double dt = sc->dt;
  int nSum[2] = {0, 0}; double uSum[2] = {0, 0};
  for (int k = 0; k < nsh; k++) {                       // Shape::updateLabVelocity
    if (sh[k].cfg.bFixedx) { nSum[0]++; uSum[0] -= sh[k].s.u; }
    if (sh[k].cfg.bFixedy) { nSum[1]++; uSum[1] -= sh[k].s.v; }
  }
  if (nSum[0] > 0) sc->uinfx = uSum[0] / nSum[0];
  if (nSum[1] > 0) sc->uinfy = uSum[1] / nSum[1];
  for (int k = 0; k < nsh; k++) {
    DevShape& S = sh[k];
    shape_update_position(S, dt, sc->uinfx, sc->uinfy);
    const double p0 = S.s.center[0], p1 = S.s.center[1];
    if (p0 < 0 || p0 > g.ext[0] || p1 < 0 || p1 > g.ext[1]) atomicOr(&sc->status, ST_DOMAIN);
    S.ntilesPrev = S.ntiles;
    if (S.cfg.kind == CUP2D_SHAPE_DISK) {               // FillBlocks_Cylinder bbox
      const double safety = 2 * g.h, R = S.cfg.radius;
      S.bbox[0][0] = p0 - R - safety; S.bbox[0][1] = p0 + R + safety;
      S.bbox[1][0] = p1 - R - safety; S.bbox[1][1] = p1 + R + safety;
    }
  }
  for (int k = 0; k < nsh; k++)
    if (sh[k].cfg.pid || sh[k].cfg.pidpos) fish_pid(sc, sh[k]);
}

// Reset the grid cells of last step's tiles of every shape, chi = 0
// (PutObjectsOnGrid.cpp:193) and sdf = -1 (:194), and drop their slot
// mapping; CTA `cta` of `ncta` takes tiles cta, cta + ncta, ...
__device__ __forceinline__ void clear_old_tiles(const GridDesc& g, const DevShape* sh, int nsh,
                                                const ObstTiles* T, double* chi, double* sdf,
                                                int cta, int ncta)
{
  const int tid = lin_tid(), nt = lin_nthreads();
  for (int k = 0; k < nsh; k++) {
    const ObstTiles& t = T[k];
    for (int s = cta; s < sh[k].ntiles; s += ncta) {
      const int b = t.tiles[s];
      const int bx = b % g.bpdx, by = b / g.bpdx;
      for (int i = tid; i < BS2; i += nt) {
        const size_t c = (size_t)(by * BS + i / BS) * g.nx + bx * BS + (i % BS);
        chi[c] = 0; sdf[c] = -1;
      }
      if (tid == 0) t.slot[b] = -1;
    }
  }
}

} // namespace cup2d
