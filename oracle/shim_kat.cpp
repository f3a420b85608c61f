// Oracle test infrastructure: C entry points for the known-answer tests of
// the project-written stand-ins the reference is compiled against (the
// FFTW-API FFT and DCT, the GSL 3x3 LU).  tests/test_oracle_cpu.py checks them
// against numpy/scipy before any parity result that depends on them is
// trusted.  Nothing in the product links this.
#include <cstdlib>
#include <cstring>
#include <fftw3.h>
#include <gsl/gsl_linalg.h>

extern "C" {

// 2D real-to-complex of an n0 x n1 row-major array (FFTW layout: n0 x (n1/2+1))
void kat_dft_r2c_2d(int n0, int n1, const double* in, double* out) {
  double* a = fftw_alloc_real((size_t)n0 * n1);
  fftw_complex* b = (fftw_complex*)fftw_alloc_real((size_t)n0 * (n1 / 2 + 1) * 2);
  std::memcpy(a, in, sizeof(double) * n0 * n1);
  fftw_plan p = fftw_plan_dft_r2c_2d(n0, n1, a, b, FFTW_MEASURE);
  fftw_execute(p);
  std::memcpy(out, b, sizeof(fftw_complex) * n0 * (n1 / 2 + 1));
  fftw_destroy_plan(p); fftw_free(a); fftw_free(b);
}

// its unnormalised inverse
void kat_dft_c2r_2d(int n0, int n1, const double* in, double* out) {
  fftw_complex* a = (fftw_complex*)fftw_alloc_real((size_t)n0 * (n1 / 2 + 1) * 2);
  double* b = fftw_alloc_real((size_t)n0 * n1);
  std::memcpy(a, in, sizeof(fftw_complex) * n0 * (n1 / 2 + 1));
  fftw_plan p = fftw_plan_dft_c2r_2d(n0, n1, a, b, FFTW_MEASURE);
  fftw_execute(p);
  std::memcpy(out, b, sizeof(double) * n0 * n1);
  fftw_destroy_plan(p); fftw_free(a); fftw_free(b);
}

// 2D real-to-real with kinds 0 = REDFT10, 1 = REDFT01 on both axes
void kat_r2r_2d(int n0, int n1, int kind, const double* in, double* out) {
  double* a = fftw_alloc_real((size_t)n0 * n1);
  double* b = fftw_alloc_real((size_t)n0 * n1);
  std::memcpy(a, in, sizeof(double) * n0 * n1);
  const fftw_r2r_kind k = kind == 0 ? FFTW_REDFT10 : FFTW_REDFT01;
  fftw_plan p = fftw_plan_r2r_2d(n0, n1, a, b, k, k, FFTW_MEASURE);
  fftw_execute(p);
  std::memcpy(out, b, sizeof(double) * n0 * n1);
  fftw_destroy_plan(p); fftw_free(a); fftw_free(b);
}

// x = A^-1 b through the GSL calls of Shape::updateVelocity (Shape.cpp:48-54)
int kat_lu_solve3(const double* A, const double* b, double* x) {
  double Ac[9];
  std::memcpy(Ac, A, sizeof(Ac));
  gsl_matrix_view Am = gsl_matrix_view_array(Ac, 3, 3);
  gsl_vector_view bv = gsl_vector_view_array(const_cast<double*>(b), 3);
  gsl_vector* xv = gsl_vector_alloc(3);
  gsl_permutation* perm = gsl_permutation_alloc(3);
  int s = 0;
  gsl_linalg_LU_decomp(&Am.matrix, perm, &s);
  const int rc = gsl_linalg_LU_solve(&Am.matrix, perm, &bv.vector, xv);
  for (int i = 0; i < 3; i++) x[i] = gsl_vector_get(xv, i);
  delete[] xv->data; delete xv;                // the stand-in's allocations
  delete[] perm->data; delete perm;
  return rc;
}

}
