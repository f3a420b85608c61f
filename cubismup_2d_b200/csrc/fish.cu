// Fish on the device: Fish::create (Fish.cpp:20-178) in three kernels.
//
// k_fish_midline (one CTA per fish): the midline at time t for the two
//   midline models of the reference -- StefanFish's
//   CurvatureFish::computeMidline (StefanFish.cpp:154-206: curvature
//   scheduler ramp, travelling curvature wave, Frenet integration
//   FishUtilities.h:15-79) and CarlingFish's AmplitudeFish::computeMidline
//   (CarlingFish.cpp:16-88) -- then integrateLinearMomentum,
//   changeToCoMFrameLinear and integrateAngularMomentum
//   (FishLibrary.cpp:86-159).  None of this depends on the flow or on the
//   body's position, only on t, so the pipeline computes the midline of step
//   n+1 on a side branch while step n runs (double buffer by step parity).
//   The Frenet recurrence is serial in s; it runs on one thread with its
//   inputs and outputs in shared memory.
// k_fish_frame (one CTA per fish): changeToCoMFrameAngular with the current
//   theta_internal (FishLibrary.cpp:161-176) and the AreaSegment boxes in the
//   computational frame (Fish.cpp:118-150, FishLibrary.cpp:295-342).
// k_fish_raster (4 CTAs per obstacle tile, one per 16x16 cells):
//   PutFishOnBlocks (FishLibrary.cpp:403-638).  The reference scatters every
//   surface / interior point of every intersecting segment onto the block;
//   here each CTA walks the points of the block's segments in the
//   reference's loop order (segment, s index, side or width offset), keeps
//   those whose support reaches its 16x16 cells, and every cell applies them
//   in that order, so its "keep the
//   nearest" updates (ties included) and its hat-kernel sums see exactly the
//   reference's sequence.
#include <cmath>
#include "context.hpp"
#include "fish.cuh"

namespace cup2d {

namespace {

constexpr double EPSd = 2.220446049250313e-16;

__device__ __forceinline__ double sq(double x) { return x * x; }

// IF2D_Interpolation1D::cubicInterpolation (FishUtilities.h:132-145)
__device__ __forceinline__ void cubic_interp(double x0, double x1, double x, double y0, double y1,
                                             double dy0, double dy1, double& y, double& dy)
{
  const double xrel = (x - x0);
  const double deltax = (x1 - x0);
  const double a = (dy0 + dy1) / (deltax * deltax) - 2 * (y1 - y0) / (deltax * deltax * deltax);
  const double b = (-2 * dy0 - dy1) / deltax + 3 * (y1 - y0) / (deltax * deltax);
  const double c = dy0;
  const double d = y0;
  y = a * xrel * xrel * xrel + b * xrel * xrel + c * xrel + d;
  dy = 3 * a * xrel * xrel + 2 * b * xrel + c;
}

// mode 0: midline at sc->time into buffer (step & 1);
// mode 1: midline at sc->time + sc->dt (the next step) into buffer ((step + 1) & 1);
// mode 2: mode 1 at the start of a graph step, before the step has set its
//   dt: runs only if that dt was carried from the previous step
//   (dtNextValid; the step copies dtNext into dt), and records in
//   sc->midlineEarly whether it ran.  Reads only the shape's configuration,
//   time, step and dtNext, which nothing changes before the step's end;
// mode 3: mode 1 unless mode 2 ran;
// mode 4: mode 0 unless buffer (step & 1) already holds the midline of
//   sc->time (the integrals keep the time they were formed at; a fresh
//   buffer holds NaN), i.e. unless an earlier launch formed it ahead.
__global__ void __launch_bounds__(512)
k_fish_midline(Scalars* sc, const DevShape* sh, int k, FishArrays F, int mode)
{
  pdl_begin();
  const int tid = threadIdx.x;
  if (mode == 2) {
    const int ok = sc->dtNextValid;
    if (tid == 0) sc->midlineEarly = ok;
    if (!ok) return;
  }
  if (mode == 3 && sc->midlineEarly) return;
  if (mode == 4 && F.integ[8 * (sc->step & 1) + 7] == sc->time) return;
  CUP2D_TRACE_SCOPE(TR_MIDLINE);
  CUP2D_TRACE_MARK(TRACE_ITEMS - 3, 0);
  extern __shared__ double smem[];
  __shared__ double red[32 * 5];
  __shared__ double bc[4];
  const DevShape& S = sh[k];
  const int Nm = F.nm, nt = blockDim.x;
  const bool now = mode == 0 || mode == 4;              // this step's midline
  const double t = now ? sc->time : sc->time + (mode == 2 ? sc->dtNext : sc->dt);
  const int p = now ? sc->step & 1 : (sc->step + 1) & 1;
  const double L = S.cfg.length, T = S.cfg.Tperiod;
  double* rS = smem;          double* width = rS + Nm;
  double* rK = width + Nm;    double* vK = rK + Nm;
  double* rX = vK + Nm;       double* rY = rX + Nm;
  double* vX = rY + Nm;       double* vY = vX + Nm;
  double* norX = vY + Nm;     double* norY = norX + Nm;
  double* vNorX = norY + Nm;  double* vNorY = vNorX + Nm;
  for (int i = tid; i < Nm; i += nt) { rS[i] = F.rS[i]; width[i] = F.width[i]; }
  __syncthreads();
  CUP2D_TRACE_MARK(TRACE_ITEMS - 3, 1);

  if (S.cfg.kind != CUP2D_SHAPE_CARLINGFISH) {
    // curvature scheduler: after transition(0, 0, T, zeros, values) the start
    // state and slope are zero and the end state is p1f (StefanFish: the
    // spline of its control values; the envelope swimmer: its envelope)
    // (StefanFish.cpp:166-206).  The RL bending wave rB, vB of the learn-wave
    // scheduler (zero without actions), the tail period and its phase, and
    // the PID terms come from the actuation state (cup2d_fish_act).
    const FishCtl& C = S.ctl;
    const double waveLength = 1, amp = S.cfg.ampFac, phaseShift = S.cfg.phaseShift;
    const double periodPIDval = C.periodPIDval, time0 = C.time0, timeshift = C.timeshift;
    const double diffT = C.TperiodPID ? 1 - (t - time0) * C.periodPIDdif / periodPIDval : 1;
    const double darg = 2 * M_PI / periodPIDval * diffT;
    const double arg0 = 2 * M_PI * ((t - time0) / periodPIDval + timeshift) + M_PI * phaseShift;
    const double fac = C.pidFac, dif = C.pidDif;
    // ParameterSchedulerLearnWave<7>::gimmeValues (FishUtilities.h:320-366)
    // at nodes -.5, -.25, 0, .25, .5, .75, 1 (StefanFish.cpp:163-164)
    const double _1oL = 1. / L, _1oT = 1. / periodPIDval;
    for (int i = tid; i < Nm; i += nt) {
      double rC, vC;
      if (t > T) { rC = F.p1f[i]; vC = 0; }
      else cubic_interp(0.0, T, t, 0.0, F.p1f[i], 0.0, 0.0, rC, vC);
      double rB = 0, vB = 0;
      {
        const double c = rS[i] * _1oL - (t - C.bendT0) * _1oT;   // travelling wave coordinate
        if (c < -.5) {
          cubic_interp(c, -.5, c, C.bend[0], C.bend[0], 0.0, 0.0, rB, vB);
        } else if (c > 1.) {
          cubic_interp(1., c, c, C.bend[6], C.bend[6], 0.0, 0.0, rB, vB);
        } else {
#pragma unroll
          for (int j = 1; j < 7; ++j) {                 // the last interval holding c wins
            const double xa = .25 * (j - 1) - .5, xb = .25 * j - .5;
            if (c >= xa && c <= xb) {
              cubic_interp(xa, xb, c, C.bend[j - 1], C.bend[j], 0.0, 0.0, rB, vB);
              vB = -vB * _1oT;
            }
          }
        }
      }
      const double arg = arg0 - 2 * M_PI * rS[i] / L / waveLength;
      rK[i] = amp * rC * (sin(arg) + rB + fac);
      vK[i] = amp * (vC * (sin(arg) + rB + fac) + rC * (cos(arg) * darg + vB + dif));
    }
    __syncthreads();
  CUP2D_TRACE_MARK(TRACE_ITEMS - 3, 2);
    if (tid == 0) {                                     // IF2D_Frenet2D::solve
      const double* curv = rK; const double* curv_dt = vK;
      rX[0] = 0.0; rY[0] = 0.0;
      double nX = 0.0, nY = 1.0;                        // norX[i-1], norY[i-1]
      double ksiX = 1.0, ksiY = 0.0;
      vX[0] = 0.0; vY[0] = 0.0;
      double vnX = 0.0, vnY = 0.0;                      // vNorX[i-1], vNorY[i-1]
      double vKsiX = 0.0, vKsiY = 0.0;
      double rx = 0.0, ry = 0.0, vx = 0.0, vy = 0.0;
      norX[0] = nX; norY[0] = nY; vNorX[0] = vnX; vNorY[0] = vnY;
      double sPrev = rS[0];
      // the next point's inputs are read one iteration ahead, off the
      // recurrence's chain
      double cN = curv[0], cdN = curv_dt[0], sN = rS[1];
#pragma unroll 2
      for (int i = 1; i < Nm; i++) {
        const double c = cN, cd = cdN, sNow = sN;
        if (i + 1 < Nm) { cN = curv[i]; cdN = curv_dt[i]; sN = rS[i + 1]; }
        const double dksiX = c * nX;
        const double dksiY = c * nY;
        const double dnuX = -c * ksiX;
        const double dnuY = -c * ksiY;
        const double dvKsiX = cd * nX + c * vnX;
        const double dvKsiY = cd * nY + c * vnY;
        const double dvNuX = -cd * ksiX - c * vKsiX;
        const double dvNuY = -cd * ksiY - c * vKsiY;
        const double ds = sNow - sPrev;
        rx = rx + ds * ksiX;
        ry = ry + ds * ksiY;
        nX = nX + ds * dnuX;
        nY = nY + ds * dnuY;
        ksiX += ds * dksiX;
        ksiY += ds * dksiY;
        vx = vx + ds * vKsiX;
        vy = vy + ds * vKsiY;
        vnX = vnX + ds * dvNuX;
        vnY = vnY + ds * dvNuY;
        vKsiX += ds * dvKsiX;
        vKsiY += ds * dvKsiY;
        const double d1 = ksiX * ksiX + ksiY * ksiY;
        const double d2 = nX * nX + nY * nY;
        // 1/sqrt(d) as the reference rounds it: the correctly rounded square
        // root, then the correctly rounded reciprocal (both factors first, so
        // the two sequences overlap)
        const double nf1 = __drcp_rn(__dsqrt_rn(d1)), nf2 = __drcp_rn(__dsqrt_rn(d2));
        if (d1 > EPSd) { ksiX *= nf1; ksiY *= nf1; }
        if (d2 > EPSd) { nX *= nf2; nY *= nf2; }
        rX[i] = rx; rY[i] = ry; vX[i] = vx; vY[i] = vy;
        norX[i] = nX; norY[i] = nY; vNorX[i] = vnX; vNorY[i] = vnY;
        sPrev = sNow;
      }
    }
    __syncthreads();
  CUP2D_TRACE_MARK(TRACE_ITEMS - 3, 3);
  } else {
    // AmplitudeFish::computeMidline (CarlingFish.cpp:70-107)
    const double phaseShift = S.cfg.phaseShift;
    const double rampFac = t < T ? sin(0.5 * M_PI * t / T) : 1.0;
    const double rampFacVel = t < T ? 0.5 * M_PI / T * cos(0.5 * M_PI * t / T) : 0.0;
    auto latPos = [&](double s) {
      const double arg = 2 * M_PI * (s / L - t / T + phaseShift);
      return 4. / 33. * (s + 0.03125 * L) * sin(arg);
    };
    auto latVel = [&](double s) {
      const double arg = 2 * M_PI * (s / L - t / T + phaseShift);
      return -4. / 33. * (s + 0.03125 * L) * (2 * M_PI / T) * cos(arg);
    };
    for (int i = tid; i < Nm; i += nt) {
      rY[i] = rampFac * latPos(rS[i]);
      vY[i] = rampFac * latVel(rS[i]) + rampFacVel * latPos(rS[i]);
    }
    __syncthreads();
    for (int i = 1 + tid; i < Nm; i += nt) {
      const double dy = rY[i] - rY[i - 1], ds = rS[i] - rS[i - 1];
      const double dx = sqrt(ds * ds - dy * dy);
      const double dVy = vY[i] - vY[i - 1];
      const double dVx = -dy / dx * dVy;
      rK[i] = dx; vK[i] = dVx;                          // increments, summed below
      norX[i - 1] = -dy / ds; norY[i - 1] = dx / ds;
      vNorX[i - 1] = -dVy / ds; vNorY[i - 1] = dVx / ds;
    }
    __syncthreads();
    if (tid == 0) {
      rX[0] = 0.0; vX[0] = 0.0;
      for (int i = 1; i < Nm; i++) { rX[i] = rK[i] + rX[i - 1]; vX[i] = vK[i] + vX[i - 1]; }
      norX[Nm - 1] = norX[Nm - 2]; norY[Nm - 1] = norY[Nm - 2];
      vNorX[Nm - 1] = vNorX[Nm - 2]; vNorY[Nm - 1] = vNorY[Nm - 2];
    }
    __syncthreads();
  }

  // FishData::computeSurface (FishLibrary.cpp:178-194): the skin in the
  // midline's own frame, kept with this buffer
  {
    const FishMidline& M = F.mid[p];
    for (int i = tid; i < Nm; i += nt) {
      double n0 = norX[i], n1 = norY[i];
      const double mod = sqrt(n0 * n0 + n1 * n1);
      n0 /= mod; n1 /= mod;
      M.lX[i] = rX[i] - width[i] * n0; M.lY[i] = rY[i] - width[i] * n1;
      M.uX[i] = rX[i] + width[i] * n0; M.uY[i] = rY[i] + width[i] * n1;
    }
  }

  // FishData::_d_ds / _integrationFac* (FishLibrary.h:79-95)
  auto d_ds = [&](int idx, const double* vals) -> double {
    if (idx == 0) return (vals[idx + 1] - vals[idx]) / (rS[idx + 1] - rS[idx]);
    else if (idx == Nm - 1) return (vals[idx] - vals[idx - 1]) / (rS[idx] - rS[idx - 1]);
    else return ((vals[idx + 1] - vals[idx]) / (rS[idx + 1] - rS[idx]) +
                 (vals[idx] - vals[idx - 1]) / (rS[idx] - rS[idx - 1])) / 2;
  };
  auto dsOf = [&](int i) -> double {
    return (i == 0) ? rS[1] - rS[0] : ((i == Nm - 1) ? rS[Nm - 1] - rS[Nm - 2] : rS[i + 1] - rS[i - 1]);
  };
  double* integ = F.integ + 8 * p;
  {                                                     // integrateLinearMomentum
    double a[5] = {0, 0, 0, 0, 0};
    for (int i = tid; i < Nm; i += nt) {
      const double ds = dsOf(i);
      const double fac1 = 2 * width[i];
      const double fac2 = 2 * F.w3[i] * (d_ds(i, norX) * norY[i] - d_ds(i, norY) * norX[i]) / 3;
      a[0] += fac1 * ds / 2;
      a[1] += (rX[i] * fac1 + norX[i] * fac2) * ds / 2;
      a[2] += (rY[i] * fac1 + norY[i] * fac2) * ds / 2;
      a[3] += (vX[i] * fac1 + vNorX[i] * fac2) * ds / 2;
      a[4] += (vY[i] * fac1 + vNorY[i] * fac2) * ds / 2;
    }
    block_sum<5>(a, red);
    if (tid == 0) {
      const double area = a[0];
      integ[0] = area;
      integ[1] = a[1] / area; integ[2] = a[2] / area;
      integ[3] = a[3] / area; integ[4] = a[4] / area;
      bc[0] = integ[1]; bc[1] = integ[2]; bc[2] = integ[3]; bc[3] = integ[4];
    }
    __syncthreads();
  CUP2D_TRACE_MARK(TRACE_ITEMS - 3, 4);
  }
  for (int i = tid; i < Nm; i += nt) {                  // changeToCoMFrameLinear
    rX[i] -= bc[0]; rY[i] -= bc[1]; vX[i] -= bc[2]; vY[i] -= bc[3];
  }
  __syncthreads();
  CUP2D_TRACE_MARK(TRACE_ITEMS - 3, 5);
  {                                                     // integrateAngularMomentum
    double a[2] = {0, 0};
    for (int i = tid; i < Nm; i += nt) {
      const double ds = dsOf(i);
      const double w3 = F.w3[i];                        // pow(width, 3), formed at set-up
      const double fac1 = 2 * width[i];
      const double fac2 = 2 * w3 * (d_ds(i, norX) * norY[i] - d_ds(i, norY) * norX[i]) / 3;
      const double fac3 = 2 * w3 / 3;
      const double tmp_M = (rX[i] * vY[i] - rY[i] * vX[i]) * fac1
        + (rX[i] * vNorY[i] - rY[i] * vNorX[i] + vY[i] * norX[i] - vX[i] * norY[i]) * fac2
        + (norX[i] * vNorY[i] - norY[i] * vNorX[i]) * fac3;
      const double tmp_J = (rX[i] * rX[i] + rY[i] * rY[i]) * fac1
        + 2 * (rX[i] * norX[i] + rY[i] * norY[i]) * fac2 + fac3;
      a[0] += tmp_M * ds / 2;
      a[1] += tmp_J * ds / 2;
    }
    block_sum<2>(a, red);
    if (tid == 0) { integ[5] = a[1]; integ[6] = a[0] / a[1]; integ[7] = t; }
  }
  const FishMidline& M = F.mid[p];
  for (int i = tid; i < Nm; i += nt) {
    M.rX[i] = rX[i]; M.rY[i] = rY[i]; M.vX[i] = vX[i]; M.vY[i] = vY[i];
    M.norX[i] = norX[i]; M.norY[i] = norY[i]; M.vNorX[i] = vNorX[i]; M.vNorY[i] = vNorY[i];
  }
}

// 1024 threads of at most 64 registers take a whole SM's register file, so
// no other kernel's CTA shares (and slows) the SM of this latency-bound CTA.
__global__ void __launch_bounds__(1024)
k_fish_frame(GridDesc g, Scalars* sc, DevShape* sh, int k, FishArrays F, ObstTiles t)
{
  extern __shared__ double fsm[];                      // the frame midline, staged
  __shared__ double bc[3];
  DevShape& S = sh[k];
  const int Nm = F.nm, tid = threadIdx.x, nt = blockDim.x;
  double* rX = fsm;           double* rY = rX + Nm;
  double* vX = rY + Nm;       double* vY = vX + Nm;
  double* norX = vY + Nm;     double* norY = norX + Nm;
  double* vNorX = norY + Nm;  double* vNorY = vNorX + Nm;
  double* width = vNorY + Nm; double* rS = width + Nm;
  Segment* segS = reinterpret_cast<Segment*>(rS + Nm);  // this step's segments, also kept on chip
  // Before the wait: only what earlier steps wrote -- the step parity (set
  // at the previous step's end), this step's midline (computed during the
  // previous step, or by a kernel the predecessor already waited for), the
  // width and the arclength -- staged while the kernel before runs.
  const int p = sc->step & 1;
  const double* integ = F.integ + 8 * p;
  const FishMidline& M = F.mid[p];
#pragma unroll 1
  for (int i = tid; i < Nm; i += nt) {
    width[i] = F.width[i]; rS[i] = F.rS[i];
    rX[i] = M.rX[i]; rY[i] = M.rY[i]; vX[i] = M.vX[i]; vY[i] = M.vY[i];
  }
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_FRAME);
  CUP2D_TRACE_MARK(TRACE_ITEMS - 1, 0);
  // the body's motion of this step (written by step_begin), loaded now so
  // that the reads overlap the rotation and normal phases instead of
  // stalling the segment chain behind a barrier
  const double cosO = S.cosO, sinO = S.sinO, cen0 = S.s.center[0], cen1 = S.s.center[1];
  if (tid == 0) {                                       // Fish.cpp:87-93 bookkeeping
    S.f.midBuf = p;
    S.f.area_internal = integ[0];
    S.f.CoM_internal[0] = integ[1]; S.f.CoM_internal[1] = integ[2];
    S.f.vCoM_internal[0] = integ[3]; S.f.vCoM_internal[1] = integ[4];
    S.f.angvel_internal_prev = S.f.angvel_internal;
    S.f.J_internal = integ[5];
    S.f.angvel_internal = integ[6];
    bc[0] = S.f.cosTh; bc[1] = S.f.sinTh; bc[2] = integ[6];   // theta_internal, angvel
  }
  __syncthreads();
  CUP2D_TRACE_MARK(TRACE_ITEMS - 1, 1);
  const FishMidline& R = F.frame;
  {                                                     // changeToCoMFrameAngular
    const double vAin = bc[2];
    const double R00 = bc[0], R01 = -bc[1], R10 = bc[1], R11 = bc[0];   // rotation by theta_internal
#pragma unroll 1
    for (int i = tid; i < Nm; i += nt) {                // in place: thread i reads and writes entry i
      const double px = rX[i], py = rY[i];
      const double qx = vX[i] + vAin * py, qy = vY[i] - vAin * px;
      const double a = R00 * px + R01 * py, b = R10 * px + R11 * py;
      const double c = R00 * qx + R01 * qy, d = R10 * qx + R11 * qy;
      rX[i] = a; rY[i] = b; vX[i] = c; vY[i] = d;
      R.rX[i] = a; R.rY[i] = b; R.vX[i] = c; R.vY[i] = d;
    }
    __syncthreads();
  CUP2D_TRACE_MARK(TRACE_ITEMS - 1, 2);
#pragma unroll 1
    for (int i = tid; i < Nm; i += nt) {                // _computeMidlineNormals
      const int j = i < Nm - 1 ? i : Nm - 2;            // the last copies its neighbour
      const double ds = rS[j + 1] - rS[j];
      const double tX = rX[j + 1] - rX[j], tY = rY[j + 1] - rY[j];
      const double tVX = vX[j + 1] - vX[j], tVY = vY[j + 1] - vY[j];
      const double a = -tY / ds, b = tX / ds, c = -tVY / ds, d = tVX / ds;
      norX[i] = a; norY[i] = b; vNorX[i] = c; vNorY[i] = d;
      R.norX[i] = a; R.norY[i] = b; R.vNorX[i] = c; R.vNorY[i] = d;
    }
    __syncthreads();
  CUP2D_TRACE_MARK(TRACE_ITEMS - 1, 3);
  }
  // AreaSegments (Fish.cpp:118-150) in the computational frame: 16 lanes per
  // segment take its midline points (the bounding box is a min / max, exact
  // in any order), then lane 0 of the group finishes the segment.
  const int Nseg = F.nseg;
  const double R00 = cosO, R01 = -sinO, R10 = sinO, R11 = cosO;   // rotation by the orientation
  const double h = g.h;
  __shared__ double box[4];
  const int g16 = tid >> 4, l16 = tid & 15;
#pragma unroll 1
  for (int i0 = 0; i0 < Nseg; i0 += nt / 16) {
    const int i = i0 + g16;
    int idx = 0, next_idx = -1;
    if (i < Nseg) { next_idx = (i + 1) * (Nm - 1) / Nseg; idx = i * (Nm - 1) / Nseg; }
    double bb[2][2] = {{1e9, -1e9}, {1e9, -1e9}};
#pragma unroll 1
    for (int ss = idx + l16; ss <= next_idx; ss += 16) {
      const double xB0 = rX[ss] - norX[ss] * width[ss], xB1 = rX[ss] + norX[ss] * width[ss];
      const double yB0 = rY[ss] - norY[ss] * width[ss], yB1 = rY[ss] + norY[ss] * width[ss];
      const double maxX = fmax(xB0, xB1), minX = fmin(xB0, xB1);
      const double maxY = fmax(yB0, yB1), minY = fmin(yB0, yB1);
      bb[0][0] = fmin(bb[0][0], minX); bb[0][1] = fmax(bb[0][1], maxX);
      bb[1][0] = fmin(bb[1][0], minY); bb[1][1] = fmax(bb[1][1], maxY);
    }
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
      bb[0][0] = fmin(bb[0][0], __shfl_xor_sync(0xffffffffu, bb[0][0], o));
      bb[0][1] = fmax(bb[0][1], __shfl_xor_sync(0xffffffffu, bb[0][1], o));
      bb[1][0] = fmin(bb[1][0], __shfl_xor_sync(0xffffffffu, bb[1][0], o));
      bb[1][1] = fmax(bb[1][1], __shfl_xor_sync(0xffffffffu, bb[1][1], o));
    }
    CUP2D_TRACE_MARK_AFTER(TRACE_ITEMS - 2, 0, bb[1][1]);
    if (i < Nseg && l16 == 0) {
      const double safe = 2 * g.h;
      Segment sg;
      sg.first = idx; sg.second = next_idx;
      sg.w[0] = (bb[0][1] - bb[0][0]) / 2 + safe; sg.w[1] = (bb[1][1] - bb[1][0]) / 2 + safe;
      const double c0 = (bb[0][1] + bb[0][0]) / 2, c1 = (bb[1][1] + bb[1][0]) / 2;
      // AreaSegment::changeToComputationalFrame (FishLibrary.cpp:295-342)
      const double nI0 = R00 * 1 + R01 * 0, nI1 = R10 * 1 + R11 * 0;
      const double nJ0 = R00 * 0 + R01 * 1, nJ1 = R10 * 0 + R11 * 1;
      sg.c[0] = R00 * c0 + R01 * c1 + cen0;
      sg.c[1] = R10 * c0 + R11 * c1 + cen1;
      const double magI = sqrt(nI0 * nI0 + nI1 * nI1), magJ = sqrt(nJ0 * nJ0 + nJ1 * nJ1);
      const double invMagI = 1 / magI, invMagJ = 1 / magJ;
      CUP2D_TRACE_MARK_AFTER(TRACE_ITEMS - 2, 1, invMagI + invMagJ);
      sg.normalI[0] = fabs(nI0) * invMagI; sg.normalI[1] = fabs(nI1) * invMagI;
      sg.normalJ[0] = fabs(nJ0) * invMagJ; sg.normalJ[1] = fabs(nJ1) * invMagJ;
      const double wX[2] = {sg.w[0] * sg.normalI[0], sg.w[0] * sg.normalI[1]};
      const double wY[2] = {sg.w[1] * sg.normalJ[0], sg.w[1] * sg.normalJ[1]};
      for (int d = 0; d < 2; d++) {
        sg.boxLab[d][0] = sg.c[d] - wX[d] - wY[d];
        sg.boxLab[d][1] = sg.c[d] + wX[d] + wY[d];
        sg.boxObj[d][0] = sg.c[d] - sg.w[d];
        sg.boxObj[d][1] = sg.c[d] + sg.w[d];
      }
      F.seg[i] = sg;
      segS[i] = sg;
      CUP2D_TRACE_MARK(TRACE_ITEMS - 2, 2);
    }
  }
  __syncthreads();
  CUP2D_TRACE_MARK(TRACE_ITEMS - 1, 4);
  if (tid < 32) {                                       // one warp: bounding box of boxLab
    double lo0 = 1e300, hi0 = -1e300, lo1 = 1e300, hi1 = -1e300;
#pragma unroll 1
    for (int i = tid; i < Nseg; i += 32) {
      const Segment& sg = segS[i];
      lo0 = fmin(lo0, sg.boxLab[0][0]); hi0 = fmax(hi0, sg.boxLab[0][1]);
      lo1 = fmin(lo1, sg.boxLab[1][0]); hi1 = fmax(hi1, sg.boxLab[1][1]);
    }
    for (int o = 16; o > 0; o >>= 1) {
      lo0 = fmin(lo0, __shfl_xor_sync(0xffffffffu, lo0, o)); hi0 = fmax(hi0, __shfl_xor_sync(0xffffffffu, hi0, o));
      lo1 = fmin(lo1, __shfl_xor_sync(0xffffffffu, lo1, o)); hi1 = fmax(hi1, __shfl_xor_sync(0xffffffffu, hi1, o));
    }
    if (tid == 0) { box[0] = lo0; box[1] = hi0; box[2] = lo1; box[3] = hi1; S.nseg = Nseg; }
  }
  CUP2D_TRACE_MARK(TRACE_ITEMS - 1, 5);
  // the obstacle tiles: blocks any segment intersects (Fish.cpp:158-173),
  // searched inside the segments' bounding box only
  __syncthreads();
  CUP2D_TRACE_MARK(TRACE_ITEMS - 1, 6);
  CUP2D_TRACE_SCOPE(TR_SELECT);
  int bx0, bx1, by0, by1;
  block_range(box[0], box[1], h, 2 * h, bx0, bx1);
  block_range(box[2], box[3], h, 2 * h, by0, by1);
  clip_rect(g, bx0, bx1, by0, by1);
  const int W = bx1 - bx0 + 1, H = by1 - by0 + 1, ncand = (W > 0 && H > 0) ? W * H : 0;
  CUP2D_TRACE_MARK(TRACE_ITEMS - 2, 3);
  // candidates in chunks of one per thread, in increasing block order; the
  // (candidate, segment) pairs of a chunk are spread over the threads
  __shared__ unsigned char hit[1024];
  __shared__ int wcnt[32];
  __shared__ int base;
  const int lane = tid & 31, wid = tid >> 5, nwarps = nt >> 5;
  if (tid == 0) base = 0;
#pragma unroll 1
  for (int c0 = 0; c0 < ncand; c0 += nt) {
    const int nq = min(nt, ncand - c0);
    if (tid < nq) hit[tid] = 0;
    __syncthreads();
    // group g16 takes segments g16, g16 + nt/16, ... and tests each against
    // the blocks of its own box (block_range keeps a block of margin, so no
    // block the segment can touch is left out)
#pragma unroll 1
    for (int si = g16; si < Nseg; si += nt / 16) {
      const Segment& sg = segS[si];
      int sx0, sx1, sy0, sy1;
      block_range(sg.boxLab[0][0], sg.boxLab[0][1], h, 2 * h, sx0, sx1);
      block_range(sg.boxLab[1][0], sg.boxLab[1][1], h, 2 * h, sy0, sy1);
      sx0 = max(sx0, bx0); sx1 = min(sx1, bx1); sy0 = max(sy0, by0); sy1 = min(sy1, by1);
      const int sw = sx1 - sx0 + 1, sh = sy1 - sy0 + 1, nblk = (sw > 0 && sh > 0) ? sw * sh : 0;
#pragma unroll 1
      for (int j = l16; j < nblk; j += 16) {
        const int bx = sx0 + j % sw, by = sy0 + j / sw;
        const int cq = (by - by0) * W + (bx - bx0) - c0;
        if (cq < 0 || cq >= nq || hit[cq]) continue;
        const double start[2] = {cell_x(g, bx, 0), cell_y(g, by, 0)};
        const double end[2] = {cell_x(g, bx, BS - 1), cell_y(g, by, BS - 1)};
        if (segment_hits_block(sg, start, end, 2 * h)) hit[cq] = 1;
      }
    }
    __syncthreads();
    CUP2D_TRACE_MARK(TRACE_ITEMS - 2, 4);
    const bool f = tid < nq && hit[tid];
    const unsigned m = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wcnt[wid] = __popc(m);
    __syncthreads();
    // exclusive offset of this warp and the chunk's total: a scan of the
    // warp counts over the lanes
    int incl = lane < nwarps ? wcnt[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int pre = __shfl_sync(0xffffffffu, incl, wid > 0 ? wid - 1 : 0);
    const int off = wid > 0 ? pre : 0;
    const int tot = __shfl_sync(0xffffffffu, incl, nwarps - 1);
    const int pos = base + off + __popc(m & ((1u << lane) - 1u));
    if (f) {
      const int q = c0 + tid, b = (by0 + q / W) * g.bpdx + bx0 + q % W;
      if (pos < t.capacity) { t.tiles[pos] = b; t.slot[b] = pos; }
      else atomicOr(&sc->status, ST_CAPACITY);
    }
    __syncthreads();
    CUP2D_TRACE_MARK(TRACE_ITEMS - 2, 5);
    if (tid == 0) base += tot;
  }
  __syncthreads();
  CUP2D_TRACE_MARK(TRACE_ITEMS - 2, 6);
  if (tid == 0) S.ntiles = base < t.capacity ? base : t.capacity;
}

struct SurfPt { double myP[2], pP[2], pM[2], ud[2]; int iap[2], ss; };
struct IntPt { double ud[2], w[2][2]; int iap[2]; };

constexpr int SUB = 16;                     // cells per sub-tile edge
constexpr int NSUB = (BS / SUB) * (BS / SUB);
constexpr int RT = SUB * SUB;               // threads per CTA (one per cell)
constexpr int NWARP = RT / 32;
constexpr int CH = 4;                       // candidate points per thread and chunk
constexpr int CAP = RT * CH;                // points per chunk
constexpr int MAX_SEG_PER_TILE = 256;
constexpr int WU = 4;                       // list entries a cell evaluates at a time

// order-preserving compaction over the CTA's warps; returns the count
__device__ __forceinline__ int compact_slot(bool keep, int* wc, int& pos) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const unsigned m = __ballot_sync(0xffffffffu, keep);
  if (lane == 0) wc[wid] = __popc(m);
  __syncthreads();
  int off = 0, tot = 0;
  for (int w = 0; w < NWARP; w++) { if (w < wid) off += wc[w]; tot += wc[w]; }
  pos = off + __popc(m & ((1u << lane) - 1u));
  return tot;
}

// The same for CH candidates per thread, candidate r of thread t being
// number r*RT + t of the chunk: positions follow that order.  One barrier.
__device__ __forceinline__ int compact_chunk(const bool (&keep)[CH], int (*wc)[NWARP], int (&pos)[CH]) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  unsigned m[CH];
#pragma unroll
  for (int r = 0; r < CH; r++) {
    m[r] = __ballot_sync(0xffffffffu, keep[r]);
    if (lane == 0) wc[r][wid] = __popc(m[r]);
  }
  __syncthreads();
  int base = 0;
#pragma unroll
  for (int r = 0; r < CH; r++) {
    int off = 0, tot = 0;
    for (int w = 0; w < NWARP; w++) { if (w < wid) off += wc[r][w]; tot += wc[r][w]; }
    pos[r] = base + off + __popc(m[r] & ((1u << lane) - 1u));
    base += tot;
  }
  return base;
}

// index of the list entry whose range [start[i], start[i+1]) holds q
__device__ __forceinline__ int find_range(const int* start, int n, int q) {
  int lo = 0, hi = n;            // start[0] = 0 <= q < start[n]
  while (hi - lo > 1) { const int mid = (lo + hi) >> 1; if (start[mid] <= q) lo = mid; else hi = mid; }
  return lo;
}

// Half-row lists: warp w owns the sub-tile rows 2w (lanes 0-15) and 2w+1
// (lanes 16-31), each split into two halves of 8 columns, i.e. four lists
// (list 2*row + half).  The warp walks the chunk's kept points in order, 32
// at a time, and appends (ballot + popc, so order is kept) those whose
// support covers the list's row and reaches its half.  Every cell then
// visits only its half-row's points, in the reference's order, and skips
// those whose columns miss it.
constexpr int NLIST = 2 * SUB;

__device__ __forceinline__ void rows_build(unsigned short* rowIdx, int* rowN, const uchar4* supp, int nc) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int n[4] = {0, 0, 0, 0};
  for (int p0 = 0; p0 < nc; p0 += 32) {
    const int p = p0 + lane;
    bool in[4] = {false, false, false, false};
    if (p < nc) {
      const uchar4 sp = supp[p];          // x lo, x hi, y lo, y hi relative to the sub-tile
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int r = 2 * w + (q >> 1), h0 = 8 * (q & 1);
        in[q] = sp.z <= r && r < sp.w && sp.x < h0 + 8 && h0 < sp.y;
      }
    }
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const unsigned m = __ballot_sync(0xffffffffu, in[q]);
      if (in[q]) rowIdx[(4 * w + q) * CAP + n[q] + __popc(m & lt)] = (unsigned short)p;
      n[q] += __popc(m);
    }
  }
  if (lane < 4) rowN[4 * w + lane] = lane == 0 ? n[0] : lane == 1 ? n[1] : lane == 2 ? n[2] : n[3];
  __syncwarp();
}

// constructSurface's point (FishLibrary.cpp:470-486) of midline index ss on
// side (0: signp = -1, 1: +1) in the computational frame: rotation by the
// orientation (R) and, with TRANS, translation by the centre (pos); without
// it, on the velocity arrays, the point's deformation velocity.  The
// expressions of the reference, so the values are those it scatters.
template <bool TRANS>
__device__ __forceinline__ double2 surf_point(const double* x, const double* y, const double* nx,
                                              const double* ny, const double* width, int ss, int side,
                                              double R00, double R01, double R10, double R11,
                                              double pos0, double pos1) {
  const int signp = side ? 1 : -1;
  const double m0 = x[ss] + width[ss] * signp * nx[ss];
  const double m1 = y[ss] + width[ss] * signp * ny[ss];
  if (TRANS) return make_double2(R00 * m0 + R01 * m1 + pos0, R10 * m0 + R11 * m1 + pos1);
  return make_double2(R00 * m0 + R01 * m1, R10 * m0 + R11 * m1);
}
// constructInternl's point (FishLibrary.cpp:597-610) of midline index ss at
// width offset offsetW = iw h, likewise
template <bool TRANS>
__device__ __forceinline__ double2 int_point(const double* x, const double* y, const double* nx,
                                             const double* ny, int ss, double offsetW,
                                             double R00, double R01, double R10, double R11,
                                             double pos0, double pos1) {
  const double m0 = x[ss] + offsetW * nx[ss], m1 = y[ss] + offsetW * ny[ss];
  if (TRANS) return make_double2(R00 * m0 + R01 * m1 + pos0, R10 * m0 + R11 * m1 + pos1);
  return make_double2(R00 * m0 + R01 * m1, R10 * m0 + R11 * m1);
}

// dynamic shared memory of the raster: the frame midline (x, y, normal,
// velocity, normal velocity) and the width (RSTAGE Nm doubles), the chunk's
// points, their supports and the row lists
constexpr int RSTAGE = 9;
inline size_t raster_smem(int Nm) {
  const size_t pts = CAP * (sizeof(SurfPt) > sizeof(IntPt) ? sizeof(SurfPt) : sizeof(IntPt));
  return sizeof(double) * RSTAGE * (size_t)Nm + pts + sizeof(uchar4) * CAP + sizeof(unsigned short) * NLIST * CAP;
}

__global__ void __launch_bounds__(RT)
k_fish_raster(GridDesc g, const DevShape* sh, int k, ObstTiles t, FishArrays F, double* sdfg)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_RASTER);
  __shared__ int segFst[MAX_SEG_PER_TILE];       // first s index of the segment's points (>= 1)
  __shared__ int segIntBase[MAX_SEG_PER_TILE];   // its first interior point
  __shared__ int segSurfCnt[MAX_SEG_PER_TILE], segIntCnt[MAX_SEG_PER_TILE];
  __shared__ int surfStart[MAX_SEG_PER_TILE + 1];
  __shared__ int intStart[MAX_SEG_PER_TILE + 1];
  __shared__ int nSegList;
  __shared__ int wc[NWARP];
  __shared__ int wcc[CH][NWARP];
  __shared__ int rowN[NLIST];
  extern __shared__ double msm[];
  const DevShape& S = sh[k];
  const int nwork = S.ntiles * NSUB;
  if ((int)blockIdx.x >= nwork) return;
  const int tid = threadIdx.x;
  const int Nm = F.nm;
  double* rX = msm; double* rY = msm + Nm; double* width = msm + 2 * Nm;
  double* norX = msm + 3 * Nm; double* norY = msm + 4 * Nm;
  double* vX = msm + 5 * Nm; double* vY = msm + 6 * Nm;
  double* vNorX = msm + 7 * Nm; double* vNorY = msm + 8 * Nm;
  SurfPt* ptsS = reinterpret_cast<SurfPt*>(msm + RSTAGE * Nm);
  IntPt* ptsI = reinterpret_cast<IntPt*>(msm + RSTAGE * Nm);
  uchar4* supp = reinterpret_cast<uchar4*>(reinterpret_cast<char*>(msm + RSTAGE * Nm) +
                                           CAP * (sizeof(SurfPt) > sizeof(IntPt) ? sizeof(SurfPt) : sizeof(IntPt)));
  unsigned short* rowIdx = reinterpret_cast<unsigned short*>(supp + CAP);
  for (int i = tid; i < Nm; i += RT) {
    rX[i] = F.frame.rX[i]; rY[i] = F.frame.rY[i]; width[i] = F.width[i];
    norX[i] = F.frame.norX[i]; norY[i] = F.frame.norY[i];
    vX[i] = F.frame.vX[i]; vY[i] = F.frame.vY[i];
    vNorX[i] = F.frame.vNorX[i]; vNorY[i] = F.frame.vNorY[i];
  }
  const double h = g.h, invh = 1.0 / h;
  const double R00 = S.cosO, R01 = -S.sinO, R10 = S.sinO, R11 = S.cosO;   // rotation by the orientation
  const double pos0 = S.s.center[0], pos1 = S.s.center[1];
  for (int wi = blockIdx.x; wi < nwork; wi += gridDim.x) {
  const int s = wi / NSUB, sub = wi % NSUB;
  CUP2D_TRACE_MARK(wi, 0);
  const int b = t.tiles[s], bx = b % g.bpdx, by = b / g.bpdx;
  const int sx0 = (sub % (BS / SUB)) * SUB, sy0 = (sub / (BS / SUB)) * SUB;
  const int ix = sx0 + tid % SUB, iy = sy0 + tid / SUB;
  const int row = iy - sy0, col = ix - sx0;
  const double org0 = cell_x(g, bx, 0), org1 = cell_y(g, by, 0);

  // ordered list of the segments intersecting this block (Fish.cpp:167-173),
  // each with its point ranges of constructSurface / constructInternl
  if (tid == 0) nSegList = 0;
  __syncthreads();
  {
    const double start[2] = {org0, org1};
    const double end[2] = {cell_x(g, bx, BS - 1), cell_y(g, by, BS - 1)};
    for (int s0 = 0; s0 < S.nseg; s0 += RT) {
      const int q = s0 + tid;
      bool f = false;
      int fst = 0, sc = 0, ib = 0, ic = 0;
      if (q < S.nseg) {
        const Segment& sg = F.seg[q];
        f = segment_hits_block(sg, start, end, 2 * h);
        if (f) {
          fst = max(sg.first, 1);
          const int lst = min(sg.second, Nm - 2);
          sc = max(0, (lst - fst + 1) * 2);
          ib = F.off[fst];
          ic = max(0, F.off[lst + 1] - ib);
        }
      }
      int pos;
      const int tot = compact_slot(f, wc, pos);
      const int at = nSegList + pos;
      if (f && at < MAX_SEG_PER_TILE) { segFst[at] = fst; segIntBase[at] = ib; segSurfCnt[at] = sc; segIntCnt[at] = ic; }
      __syncthreads();
      if (tid == 0) nSegList += tot;
      __syncthreads();
    }
  }
  const int nsl = nSegList < MAX_SEG_PER_TILE ? nSegList : MAX_SEG_PER_TILE;
  if (tid == 0) {
    surfStart[0] = 0; intStart[0] = 0;
    for (int i = 0; i < nsl; i++) {
      surfStart[i + 1] = surfStart[i] + segSurfCnt[i];
      intStart[i + 1] = intStart[i] + segIntCnt[i];
    }
  }
  __syncthreads();
  const int totSurf = surfStart[nsl], totInt = intStart[nsl];
  CUP2D_TRACE_MARK(wi, 1);
  const double px = cell_x(g, bx, ix), py = cell_y(g, by, iy);   // info.pos(p, sx, sy)

  // constructSurface (FishLibrary.cpp:438-573).  A point changes the cell
  // only if its nearest-of-three squared distance dist1 = min(dist0, distP,
  // distM) is below |dist|, and then |dist| becomes dist1 (sign2d is +-1):
  // the cell ends with the first point, in the reference's order, attaining
  // the strict running minimum, so the sign, weight and velocity are
  // evaluated once, for that point.
  double dist = -1, chi = 0, ud0 = 0, ud1 = 0;
  double best = 1.0;                                    // |dist| of the initial -1
  for (int c0 = 0; c0 < totSurf; c0 += CAP) {
    // the keep test needs the point itself only; kept points load the rest
    // (neighbours, velocity) after the compaction
    int gs[CH];                                       // 2 ss + side of the candidate
    double2 my[CH];
    bool keep[CH];
    uchar4 sup[CH];
#pragma unroll
    for (int r = 0; r < CH; r++) {
      keep[r] = false;
      gs[r] = 0;
      const int q = c0 + r * RT + tid;
      if (q < totSurf) {
        const int si = find_range(surfStart, nsl, q);
        const int rr = q - surfStart[si];
        const int ss = segFst[si] + rr / 2, side = rr & 1;
        gs[r] = 2 * ss + side;
        my[r] = surf_point<true>(rX, rY, norX, norY, width, ss, side, R00, R01, R10, R11, pos0, pos1);
      }
    }
#pragma unroll
    for (int r = 0; r < CH; r++) {
      const int q = c0 + r * RT + tid;
      if (q < totSurf) {
        const int iap0 = (int)floor((my[r].x - org0) * invh), iap1 = (int)floor((my[r].y - org1) * invh);
        // support [iap-1, iap+3) clipped to the block, intersected with this sub-tile
        const int xlo = max(max(0, iap0 - 1), sx0), xhi = min(min(iap0 + 3, BS), sx0 + SUB);
        const int ylo = max(max(0, iap1 - 1), sy0), yhi = min(min(iap1 + 3, BS), sy0 + SUB);
        keep[r] = xlo < xhi && ylo < yhi;
        sup[r] = make_uchar4(xlo - sx0, xhi - sx0, ylo - sy0, yhi - sy0);
      }
    }
    int pos[CH];
    const int nc = compact_chunk(keep, wcc, pos);
#pragma unroll
    for (int r = 0; r < CH; r++)
      if (keep[r]) {
        SurfPt& Pr = ptsS[pos[r]];
        const int ss = gs[r] >> 1, side = gs[r] & 1;
        const double2 pp = surf_point<true>(rX, rY, norX, norY, width, ss + 1, side, R00, R01, R10, R11, pos0, pos1);
        const double2 pm = surf_point<true>(rX, rY, norX, norY, width, ss - 1, side, R00, R01, R10, R11, pos0, pos1);
        const double2 uu = surf_point<false>(vX, vY, vNorX, vNorY, width, ss, side, R00, R01, R10, R11, 0.0, 0.0);
        Pr.ss = ss;
        Pr.myP[0] = my[r].x; Pr.myP[1] = my[r].y;
        Pr.pP[0] = pp.x; Pr.pP[1] = pp.y; Pr.pM[0] = pm.x; Pr.pM[1] = pm.y;
        Pr.ud[0] = uu.x; Pr.ud[1] = uu.y;
        supp[pos[r]] = sup[r];
      }
    __syncthreads();
    CUP2D_TRACE_MARK(wi + 2048, 0);
    rows_build(rowIdx, rowN, supp, nc);
    CUP2D_TRACE_MARK(wi + 2048, 1);
    const int li = 2 * row + (col >> 3);                // this cell's half-row list
    const int n = rowN[li];
    const unsigned short* l = rowIdx + li * CAP;
    int winner = -1;
    // WU list entries at a time: their loads and distances are independent,
    // the running minimum then takes them in list order
    for (int e0 = 0; e0 < n; e0 += WU) {
      double d1[WU];
      int qs[WU];
      bool ok[WU];
#pragma unroll
      for (int u = 0; u < WU; u++) {
        const int e = e0 + u;
        qs[u] = l[e < n ? e : e0];
        const uchar4 sp = supp[qs[u]];
        ok[u] = e < n && col >= sp.x && col < sp.y;
        const SurfPt& Q = ptsS[qs[u]];
        const double dist0 = sq(px - Q.myP[0]) + sq(py - Q.myP[1]);
        const double distP = sq(px - Q.pP[0]) + sq(py - Q.pP[1]);
        const double distM = sq(px - Q.pM[0]) + sq(py - Q.pM[1]);
        d1[u] = fmin(fmin(dist0, distP), distM);
      }
#pragma unroll
      for (int u = 0; u < WU; u++)
        if (ok[u] && best > d1[u]) { best = d1[u]; winner = qs[u]; }
    }
    if (winner >= 0) {
      // evaluate the winner of this chunk now (its point data is in shared
      // memory only until the next chunk); a later chunk's winner replaces it
      const SurfPt& Q = ptsS[winner];
      const double dist0 = sq(px - Q.myP[0]) + sq(py - Q.myP[1]);
      const double distP = sq(px - Q.pP[0]) + sq(py - Q.pP[1]);
      const double distM = sq(px - Q.pM[0]) + sq(py - Q.pM[1]);
      // changeFromComputationalFrame (FishLibrary.h:194-200)
      const double q0 = px - pos0, q1 = py - pos1;
      const double p0 = R00 * q0 + R10 * q1, p1 = R01 * q0 + R11 * q1;
      const int ss = Q.ss;
      int close_s = ss, secnd_s = ss + (distP < distM ? 1 : -1);
      double dist1 = dist0, dist2 = distP < distM ? distP : distM;
      if (distP < dist0 || distM < dist0) {
        dist1 = dist2; dist2 = dist0;
        close_s = secnd_s; secnd_s = ss;
      }
      const double dSsq = sq(rX[close_s] - rX[secnd_s]) + sq(rY[close_s] - rY[secnd_s]);
      const double cnt2ML = sq(width[close_s]);
      const double nxt2ML = sq(width[secnd_s]);
      const double safeW = fmax(width[close_s], width[secnd_s]) + 2 * h;
      const double grd2ML = sq(p0 - rX[close_s]) + sq(p1 - rY[close_s]);
      const double diffH = fabs(width[close_s] - width[secnd_s]);
      double sign2d = 0;
      if (dSsq > diffH * diffH || grd2ML > safeW * safeW) {
        sign2d = grd2ML > cnt2ML ? -1 : 1;
      } else {
        const double corr = 2 * sqrt(cnt2ML * nxt2ML);
        const double Rsq = (cnt2ML + nxt2ML - corr + dSsq) * (cnt2ML + nxt2ML + corr + dSsq) / 4 / dSsq;
        const double maxAx = fmax(cnt2ML, nxt2ML);
        const int idAx1 = cnt2ML > nxt2ML ? close_s : secnd_s;
        const int idAx2 = idAx1 == close_s ? secnd_s : close_s;
        const double d = sqrt((Rsq - maxAx) / dSsq);
        const double xC0 = rX[idAx1] + (rX[idAx1] - rX[idAx2]) * d;
        const double xC1 = rY[idAx1] + (rY[idAx1] - rY[idAx2]) * d;
        const double grd2Core = sq(p0 - xC0) + sq(p1 - xC1);
        sign2d = grd2Core > Rsq ? -1 : 1;
      }
      const double W = 1 - sqrt(dist1) * (invh / 3);
      ud0 = W * Q.ud[0]; ud1 = W * Q.ud[1];
      dist = sign2d * dist1;
      chi = W;
    }
    __syncthreads();
  }

  CUP2D_TRACE_MARK(wi, 2);
  // constructInternl (FishLibrary.cpp:575-638)
  for (int c0 = 0; c0 < totInt; c0 += CAP) {
    int2 sw[CH];                                      // (ss, iw) of the candidate
    double2 xw[CH];
    bool keep[CH];
    uchar4 sup[CH];
#pragma unroll
    for (int r = 0; r < CH; r++) {
      keep[r] = false;
      sw[r] = make_int2(0, 0);
      const int q = c0 + r * RT + tid;
      if (q < totInt) {
        const int si = find_range(intStart, nsl, q);
        sw[r] = F.ipIdx[segIntBase[si] + (q - intStart[si])];
      }
    }
#pragma unroll
    for (int r = 0; r < CH; r++)
      if (c0 + r * RT + tid < totInt)
        xw[r] = int_point<true>(rX, rY, norX, norY, sw[r].x, sw[r].y * h, R00, R01, R10, R11, pos0, pos1);
#pragma unroll
    for (int r = 0; r < CH; r++) {
      const int q = c0 + r * RT + tid;
      if (q < totInt) {
        const int iap0 = (int)floor((xw[r].x - org0) * invh), iap1 = (int)floor((xw[r].y - org1) * invh);
        const int xlo = max(max(0, iap0), sx0), xhi = min(min(iap0 + 2, BS), sx0 + SUB);
        const int ylo = max(max(0, iap1), sy0), yhi = min(min(iap1 + 2, BS), sy0 + SUB);
        keep[r] = xlo < xhi && ylo < yhi;
        sup[r] = make_uchar4(xlo - sx0, xhi - sx0, ylo - sy0, yhi - sy0);
      }
    }
    int pos[CH];
    const int nc = compact_chunk(keep, wcc, pos);
#pragma unroll
    for (int r = 0; r < CH; r++)
      if (keep[r]) {
        IntPt& Pr = ptsI[pos[r]];
        const double2 u = int_point<false>(vX, vY, vNorX, vNorY, sw[r].x, sw[r].y * h, R00, R01, R10, R11, 0.0, 0.0);
        const double xp0 = (xw[r].x - org0) * invh, xp1 = (xw[r].y - org1) * invh;
        const double ap0 = floor(xp0), ap1 = floor(xp1);
        Pr.iap[0] = (int)ap0; Pr.iap[1] = (int)ap1;
        Pr.ud[0] = u.x; Pr.ud[1] = u.y;
        Pr.w[0][0] = 1 - fabs(xp0 - ap0); Pr.w[0][1] = 1 - fabs(xp0 - (ap0 + 1));
        Pr.w[1][0] = 1 - fabs(xp1 - ap1); Pr.w[1][1] = 1 - fabs(xp1 - (ap1 + 1));
        supp[pos[r]] = sup[r];
      }
    __syncthreads();
    rows_build(rowIdx, rowN, supp, nc);
    CUP2D_TRACE_MARK(wi + 2048, 2);
    const int li = 2 * row + (col >> 3);                // this cell's half-row list
    const int n = rowN[li];
    const unsigned short* l = rowIdx + li * CAP;
    for (int e0 = 0; e0 < n; e0 += WU) {
      double w[WU], a0[WU], a1[WU];
      bool ok[WU];
#pragma unroll
      for (int u = 0; u < WU; u++) {
        const int e = e0 + u;
        const int qi = l[e < n ? e : e0];
        const uchar4 sp = supp[qi];
        ok[u] = e < n && col >= sp.x && col < sp.y;
        const IntPt& Q = ptsI[qi];
        // a kept entry's cell lies in its 2x2 support (sx, sy in {0, 1})
        const int sx = ok[u] ? ix - Q.iap[0] : 0, sy = ok[u] ? iy - Q.iap[1] : 0;
        w[u] = Q.w[1][sy] * Q.w[0][sx];
        a0[u] = Q.ud[0]; a1[u] = Q.ud[1];
      }
#pragma unroll
      for (int u = 0; u < WU; u++)
        if (ok[u]) {
          ud0 += w[u] * a0[u];
          ud1 += w[u] * a1[u];
          chi += w[u];
          if (fabs(dist + 1) < EPSd) dist = 1;
        }
    }
    __syncthreads();
  }

  CUP2D_TRACE_MARK(wi, 3);
  // signedDistanceSqrt (FishLibrary.cpp:419-436)
  const double normfac = chi > EPSd ? chi : 1;
  ud0 /= normfac; ud1 /= normfac;
  dist = dist >= 0 ? sqrt(dist) : -sqrt(-dist);
  const size_t o = (size_t)s * BS2 + iy * BS + ix;
  t.dist[o] = dist; t.chi[o] = 0; t.udx[o] = ud0; t.udy[o] = ud1;
  atomic_max_double(&sdfg[(size_t)(by * BS + iy) * g.nx + bx * BS + ix], dist);
  __syncthreads();                                      // shared state is reused by the next item
  CUP2D_TRACE_MARK(wi, 4);
#ifdef CUP2D_TRACE
  if (threadIdx.x == 0 && wi < TRACE_ITEMS && g_trace) {   // counts of the trace build
    g_trace[2 * TR_N + 8 * wi + 5] = totSurf; g_trace[2 * TR_N + 8 * wi + 6] = totInt;
    g_trace[2 * TR_N + 8 * wi + 7] = nsl;
  }
#endif
  }
}

size_t midline_smem(int Nm) { return sizeof(double) * 12 * (size_t)Nm; }
size_t frame_smem(int Nm, int nseg) { return sizeof(double) * 10 * (size_t)Nm + sizeof(Segment) * (size_t)nseg; }

} // namespace


bool fish_fits_on_chip(int Nm, int nseg, int device) {
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess) return false;
  cudaFuncAttributes a{};
  const size_t need[3] = {midline_smem(Nm), frame_smem(Nm, nseg), raster_smem(Nm)};
  const void* fn[3] = {(const void*)k_fish_midline, (const void*)k_fish_frame, (const void*)k_fish_raster};
  for (int i = 0; i < 3; i++) {
    if (cudaFuncGetAttributes(&a, fn[i]) != cudaSuccess) return false;
    if (need[i] + a.sharedSizeBytes > (size_t)optin) return false;
  }
  return true;
}

// pow(width, 3) of each midline point (FishLibrary.cpp integrals), formed
// once on the device with the same pow the per-step integrals used
__global__ void k_fish_w3(FishArrays F) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F.nm; i += gridDim.x * blockDim.x)
    F.w3[i] = pow(F.width[i], 3.0);
}

cudaError_t fish_width_cubes(const FishArrays& F, cudaStream_t st) {
  k_fish_w3<<<(F.nm + 255) / 256, 256, 0, st>>>(F);
  return cudaGetLastError();
}

cudaError_t fish_setup_kernels() {
  cudaError_t e = allow_max_dynamic_smem((const void*)k_fish_midline);
  if (e == cudaSuccess) e = allow_max_dynamic_smem((const void*)k_fish_frame);
  if (e == cudaSuccess) e = allow_max_dynamic_smem((const void*)k_fish_raster);
  return e;
}

void launch_fish_midline(Ctx& c, int k, cudaStream_t stream, int mode) {
  launch_k(k_fish_midline, 1, 512, midline_smem(c.fish[k].nm), stream, c.dsc, c.dshapes, k, c.fish[k], mode);
  CUP2D_LAUNCHED(c);
}

void launch_fish_place(Ctx& c, int k) {
  launch_k(k_fish_frame, 1, 1024, frame_smem(c.fish[k].nm, c.fish[k].nseg), c.stream, c.g, c.dsc, c.dshapes, k, c.fish[k], c.tiles[k]);
  CUP2D_LAUNCHED(c);
}

void launch_fish_raster(Ctx& c, int k) {
  // two resident CTAs per SM at most (registers); each loops over
  // (tile, sub-tile) items
  const int items = c.tiles[k].capacity * NSUB, grid = items < 2 * c.sms ? items : 2 * c.sms;
  launch_k(k_fish_raster, grid, RT, raster_smem(c.fish[k].nm), c.stream, c.g, c.dshapes, k, c.tiles[k],
                                                                c.fish[k], c.sdf);
  CUP2D_LAUNCHED(c);
}

} // namespace cup2d

#ifdef CUP2D_TRACE
namespace cup2d { void trace_bind_fish(unsigned long long* p) { trace_bind_this_unit(p); } }
#endif
