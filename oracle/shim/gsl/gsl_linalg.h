// Oracle test infrastructure: project-written stand-in for the few GSL calls
// of Shape::updateVelocity (Shape.cpp:48-58): a 3x3 LU decomposition with
// partial pivoting and the matching triangular solves.  GSL is not installed.
//
// Algorithm: Gaussian elimination with partial pivoting, the pivot being the
// first row holding the largest |a_ij| of column j (Golub & Van Loan,
// "Matrix Computations", Alg. 3.4.1); the solve permutes b, then forward
// substitution with the unit lower factor, then back substitution with the
// upper factor, each as an inner product over the already-solved entries.
// The GPU path (cubismup_2d_b200/csrc/rigid_body.cuh) evaluates the same
// operation sequence.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdlib>

struct gsl_matrix { size_t size1, size2, tda; double* data; };
struct gsl_vector { size_t size, stride; double* data; int owner; };
struct gsl_matrix_view { gsl_matrix matrix; };
struct gsl_vector_view { gsl_vector vector; };
struct gsl_permutation { size_t size; size_t* data; };

inline gsl_matrix_view gsl_matrix_view_array(double* base, size_t n1, size_t n2) {
  gsl_matrix_view v; v.matrix.size1 = n1; v.matrix.size2 = n2; v.matrix.tda = n2; v.matrix.data = base;
  return v;
}
inline gsl_vector_view gsl_vector_view_array(double* base, size_t n) {
  gsl_vector_view v; v.vector.size = n; v.vector.stride = 1; v.vector.data = base; v.vector.owner = 0;
  return v;
}
// The reference never frees these two (Shape.cpp:50-52); the shim keeps that
// behaviour rather than changing the caller.
inline gsl_vector* gsl_vector_alloc(size_t n) {
  gsl_vector* v = new gsl_vector; v->size = n; v->stride = 1; v->data = new double[n](); v->owner = 1;
  return v;
}
inline gsl_permutation* gsl_permutation_alloc(size_t n) {
  gsl_permutation* p = new gsl_permutation; p->size = n; p->data = new size_t[n];
  for (size_t i = 0; i < n; i++) p->data[i] = i;
  return p;
}
inline double gsl_vector_get(const gsl_vector* v, size_t i) { return v->data[i * v->stride]; }

inline int gsl_linalg_LU_decomp(gsl_matrix* A, gsl_permutation* p, int* signum) {
  const size_t N = A->size1;
  double* a = A->data;
  const size_t t = A->tda;
  *signum = 1;
  for (size_t i = 0; i < N; i++) p->data[i] = i;
  for (size_t j = 0; j + 1 < N; j++) {
    double vmax = std::fabs(a[j * t + j]);
    size_t piv = j;
    for (size_t i = j + 1; i < N; i++) {
      const double aij = std::fabs(a[i * t + j]);
      if (aij > vmax) { vmax = aij; piv = i; }
    }
    if (piv != j) {
      for (size_t k = 0; k < N; k++) { const double tmp = a[j * t + k]; a[j * t + k] = a[piv * t + k]; a[piv * t + k] = tmp; }
      const size_t tp = p->data[j]; p->data[j] = p->data[piv]; p->data[piv] = tp;
      *signum = -*signum;
    }
    const double ajj = a[j * t + j];
    if (ajj != 0.0) {
      for (size_t i = j + 1; i < N; i++) {
        const double lij = a[i * t + j] / ajj;
        a[i * t + j] = lij;
        for (size_t k = j + 1; k < N; k++) a[i * t + k] = a[i * t + k] - lij * a[j * t + k];
      }
    }
  }
  return 0;
}

inline int gsl_linalg_LU_solve(const gsl_matrix* LU, const gsl_permutation* p, const gsl_vector* b, gsl_vector* x) {
  const size_t N = LU->size1, t = LU->tda;
  const double* a = LU->data;
  for (size_t i = 0; i < N; i++) x->data[i] = b->data[p->data[i] * b->stride];
  for (size_t i = 0; i < N; i++) {          // unit lower
    double s = x->data[i];
    for (size_t j = 0; j < i; j++) s = s - a[i * t + j] * x->data[j];
    x->data[i] = s;
  }
  for (size_t ii = N; ii-- > 0;) {          // upper
    double s = x->data[ii];
    for (size_t j = ii + 1; j < N; j++) s = s - a[ii * t + j] * x->data[j];
    x->data[ii] = s / a[ii * t + ii];
  }
  return 0;
}
