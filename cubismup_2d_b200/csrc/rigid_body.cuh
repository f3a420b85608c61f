// Rigid-body updates of one shape, evaluated by a single device thread:
// Shape::updatePosition (Shape.cpp:67-105), Shape::updateVelocity with its
// 3x3 LU solve (Shape.cpp:25-59) and Disk::updateVelocity's ramp
// (ShapesSimple.cpp:83-87).
#pragma once
#include "internal.cuh"

namespace cup2d {

// Gaussian elimination with partial pivoting (first row with the largest
// |a_ij| of the column, Golub & Van Loan Alg. 3.4.1), then the permuted
// forward / back substitutions as running inner products.  The oracle's GSL
// stand-in (oracle/shim/gsl/gsl_linalg.h) performs the identical sequence.
__device__ __forceinline__ void lu_solve3(double A[3][3], const double b[3], double x[3]) {
  int p[3] = {0, 1, 2};
  for (int j = 0; j < 2; j++) {
    double vmax = fabs(A[j][j]);
    int piv = j;
    for (int i = j + 1; i < 3; i++) {
      const double aij = fabs(A[i][j]);
      if (aij > vmax) { vmax = aij; piv = i; }
    }
    if (piv != j) {
      for (int k = 0; k < 3; k++) { const double t = A[j][k]; A[j][k] = A[piv][k]; A[piv][k] = t; }
      const int tp = p[j]; p[j] = p[piv]; p[piv] = tp;
    }
    const double ajj = A[j][j];
    if (ajj != 0.0) {
      for (int i = j + 1; i < 3; i++) {
        const double lij = A[i][j] / ajj;
        A[i][j] = lij;
        for (int k = j + 1; k < 3; k++) A[i][k] = A[i][k] - lij * A[j][k];
      }
    }
  }
  for (int i = 0; i < 3; i++) x[i] = b[p[i]];
  for (int i = 0; i < 3; i++) {
    double s = x[i];
    for (int j = 0; j < i; j++) s = s - A[i][j] * x[j];
    x[i] = s;
  }
  for (int ii = 2; ii >= 0; ii--) {
    double s = x[ii];
    for (int j = ii + 1; j < 3; j++) s = s - A[ii][j] * x[j];
    x[ii] = s / A[ii][ii];
  }
}

__device__ __forceinline__ void shape_update_velocity(DevShape& S, const double dt, const double time) {
  cup2d_shape_state& s = S.s;
  const ShapeCfg& c = S.cfg;
  double A[3][3] = {{s.penalM, 0, -s.penalDY}, {0, s.penalM, s.penalDX}, {-s.penalDY, s.penalDX, s.penalJ}};
  // appliedForceX/Y and appliedTorque are never set on this path (Shape.h:55-57)
  double b[3] = {s.fluidMomX + dt * 0.0, s.fluidMomY + dt * 0.0, s.fluidAngMom + dt * 0.0};
  if (c.bForcedx && time < c.timeForced) { A[0][1] = 0; A[0][2] = 0; b[0] = s.penalM * c.forcedu; }
  if (c.bForcedy && time < c.timeForced) { A[1][0] = 0; A[1][2] = 0; b[1] = s.penalM * c.forcedv; }
  if (c.bBlockang && time < c.timeForced) { A[2][0] = 0; A[2][1] = 0; b[2] = s.penalJ * c.forcedomega; }
  double x[3];
  lu_solve3(A, b, x);
  // Shape.cpp:56 tests bForcedy for u as well: kept as in the reference
  if (!c.bForcedy || time > c.timeForced) s.u = x[0];
  if (!c.bForcedy || time > c.timeForced) s.v = x[1];
  if (!c.bBlockang || time > c.timeForced) s.omega = x[2];
  if (c.kind == CUP2D_SHAPE_DISK && c.tAccel > 0) {
    if (c.bForcedx && time < c.tAccel) s.u = (time / c.tAccel) * c.forcedu;
    if (c.bForcedy && time < c.tAccel) s.v = (time / c.tAccel) * c.forcedv;
  }
}

__device__ __forceinline__ void shape_update_position(DevShape& S, const double dt,
                                                      const double uinfx, const double uinfy) {
  cup2d_shape_state& s = S.s;
  s.com[0] += dt * (s.u + uinfx);
  s.com[1] += dt * (s.v + uinfy);
  s.lab_com[0] += dt * s.u;
  s.lab_com[1] += dt * s.v;
  s.orientation += dt * s.omega;
  s.orientation = s.orientation > M_PI ? s.orientation - 2 * M_PI : s.orientation;
  s.orientation = s.orientation < -M_PI ? s.orientation + 2 * M_PI : s.orientation;
  const double cosang = cos(s.orientation), sinang = sin(s.orientation);
  S.cosO = cosang; S.sinO = sinang;             // reused by the kernels of this step
  s.center[0] = s.com[0] + cosang * s.d_gm[0] - sinang * s.d_gm[1];
  s.center[1] = s.com[1] + sinang * s.d_gm[0] + cosang * s.d_gm[1];
  if (S.cfg.kind != CUP2D_SHAPE_DISK) {         // Fish::updatePosition (Fish.cpp:180-185)
    S.f.theta_internal -= dt * S.f.angvel_internal;
    S.f.cosTh = cos(S.f.theta_internal);
    S.f.sinTh = sin(S.f.theta_internal);
  }
}

} // namespace cup2d
