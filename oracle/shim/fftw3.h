// Oracle test infrastructure: a project-written stand-in for the FFTW3 API
// subset called by the reference's Poisson solvers
// (Poisson/FFTW_freespace.cpp:25,48,84-95,123; Poisson/FFTW_periodic.h:115-157;
//  Poisson/FFTW_dirichlet.h:79-121).  FFTW is not installed on this machine.
//
// Semantics follow FFTW's documented definitions (unnormalised transforms):
//  r2c_2d : X[k0][k1] = sum_{j0,j1} x[j0][j1] e^{-2 pi i (j0 k0/n0 + j1 k1/n1)},
//           output n0 x (n1/2+1) complex; in-place real rows padded to
//           2*(n1/2+1) reals;
//  c2r_2d : the inverse with e^{+2 pi i ...}, no 1/(n0 n1) factor;
//  REDFT10: Y_k = 2 sum_j x_j cos(pi (j+1/2) k / n)        (DCT-II)
//  REDFT01: Y_k = x_0 + 2 sum_{j>=1} x_j cos(pi j (k+1/2)/n) (DCT-III)
//  RODFT10/01 (DST-II/III) are declared but the reference never reaches them
//  on the timestep path (the factory at PoissonSolver.cpp:23-59 never builds
//  FFTW_neumann).
// The transforms are computed by fftw_shim.cpp (radix-2 for powers of two,
// Bluestein's chirp-z algorithm otherwise; DCTs through an FFT of length 4n).
#pragma once
#include <cstddef>

typedef double fftw_complex[2];
typedef float fftwf_complex[2];
typedef struct fftw_plan_s* fftw_plan;
typedef struct fftw_plan_s* fftwf_plan;
typedef int fftw_r2r_kind;

enum { FFTW_R2HC = 0, FFTW_HC2R = 1, FFTW_DHT = 2,
       FFTW_REDFT00 = 3, FFTW_REDFT01 = 4, FFTW_REDFT10 = 5, FFTW_REDFT11 = 6,
       FFTW_RODFT00 = 7, FFTW_RODFT01 = 8, FFTW_RODFT10 = 9, FFTW_RODFT11 = 10 };
#define FFTW_MEASURE 0u
#define FFTW_ESTIMATE (1u << 6)

int fftw_init_threads(void);
void fftw_plan_with_nthreads(int n);
void fftw_cleanup_threads(void);
double* fftw_alloc_real(size_t n);
void fftw_free(void* p);
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex* in, double* out, unsigned flags);
fftw_plan fftw_plan_r2r_2d(int n0, int n1, double* in, double* out,
                           fftw_r2r_kind k0, fftw_r2r_kind k1, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

int fftwf_init_threads(void);
void fftwf_plan_with_nthreads(int n);
void fftwf_cleanup_threads(void);
float* fftwf_alloc_real(size_t n);
void fftwf_free(void* p);
fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float* in, fftwf_complex* out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex* in, float* out, unsigned flags);
fftwf_plan fftwf_plan_r2r_2d(int n0, int n1, float* in, float* out,
                             fftw_r2r_kind k0, fftw_r2r_kind k1, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
