// Oracle test infrastructure: the transforms behind the project-written
// FFTW-API stand-in (fftw3.h).  Not FFTW: a plain double-precision FFT
// written for this project (iterative radix-2 for powers of two, Bluestein's
// chirp-z convolution for every other length, e.g. the odd 2N-1 padded
// sizes of Poisson/FFTW_freespace.h:25-27).  The DCT-II/III of the
// "dirichlet" solver (Poisson/FFTW_dirichlet.h:79-90) are evaluated as the
// real part of a length-4n complex FFT of the even extension.
#include "fftw3.h"
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {
using cplx = std::complex<double>;

// exp(-2 pi i k / n), k reduced modulo n first so the angle stays small.
inline cplx root(long long k, long long n) {
  k %= n; if (k < 0) k += n;
  const double a = -2.0 * M_PI * (double)k / (double)n;
  return cplx(std::cos(a), std::sin(a));
}

struct Dft1D
{
  int n = 0;
  bool pow2 = false;
  std::vector<cplx> tw;      // radix-2 twiddles
  int M = 0;                 // Bluestein convolution length
  std::vector<cplx> chirp;   // exp(-i pi k^2 / n)
  std::vector<cplx> bhat;    // FFT of conj chirp, wrapped
  Dft1D* sub = nullptr;

  explicit Dft1D(int n_) : n(n_) {
    pow2 = n > 0 && (n & (n - 1)) == 0;
    if (pow2) {
      tw.resize(n / 2 > 0 ? n / 2 : 1);
      for (int k = 0; k < n / 2; k++) tw[k] = root(k, n);
      return;
    }
    M = 1; while (M < 2 * n - 1) M <<= 1;
    sub = new Dft1D(M);
    chirp.resize(n);
    for (long long k = 0; k < n; k++) {
      const long long e = (k * k) % (2LL * n);          // exact k^2 mod 2n
      const double a = -M_PI * (double)e / (double)n;
      chirp[k] = cplx(std::cos(a), std::sin(a));
    }
    bhat.assign(M, cplx(0, 0));
    for (int k = 0; k < n; k++) {
      bhat[k] = std::conj(chirp[k]);
      if (k) bhat[M - k] = std::conj(chirp[k]);
    }
    sub->forward(bhat.data());
  }
  ~Dft1D() { delete sub; }

  // in-place forward transform, X_k = sum_j x_j exp(-2 pi i j k / n)
  void forward(cplx* x) const {
    if (n <= 1) return;
    if (pow2) {
      for (int i = 1, j = 0; i < n; i++) {       // bit reversal
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(x[i], x[j]);
      }
      for (int len = 2; len <= n; len <<= 1) {
        const int half = len / 2, step = n / len;
        for (int i = 0; i < n; i += len)
          for (int k = 0; k < half; k++) {
            const cplx w = tw[k * step];
            const cplx a = x[i + k], b = x[i + k + half] * w;
            x[i + k] = a + b;
            x[i + k + half] = a - b;
          }
      }
      return;
    }
    std::vector<cplx> a(M, cplx(0, 0));
    for (int k = 0; k < n; k++) a[k] = x[k] * chirp[k];
    sub->forward(a.data());
    for (int k = 0; k < M; k++) a[k] *= bhat[k];
    // inverse of length M through conjugation
    for (int k = 0; k < M; k++) a[k] = std::conj(a[k]);
    sub->forward(a.data());
    const double inv = 1.0 / M;
    for (int k = 0; k < n; k++) x[k] = std::conj(a[k]) * inv * chirp[k];
  }
  void backward(cplx* x) const {
    for (int k = 0; k < n; k++) x[k] = std::conj(x[k]);
    forward(x);
    for (int k = 0; k < n; k++) x[k] = std::conj(x[k]);
  }
};

enum PlanType { R2C = 0, C2R = 1, R2R = 2 };
} // namespace

struct fftw_plan_s
{
  int type = 0, n0 = 0, n1 = 0, k0 = 0, k1 = 0;
  bool single = false;
  void* in = nullptr;
  void* out = nullptr;
  Dft1D* d0 = nullptr;  // length for dimension 0 (or 4*n0 for r2r)
  Dft1D* d1 = nullptr;  // length for dimension 1 (or 4*n1 for r2r)
  ~fftw_plan_s() { delete d0; delete d1; }
};

namespace {

// y (length n, stride s) <- DCT/DST kind applied to x (same place), via d4n
void r2r_line(double* y, const int n, const long stride, const int kind, const Dft1D& d4n) {
  std::vector<cplx> w(4 * n, cplx(0, 0));
  std::vector<double> x(n);
  for (int j = 0; j < n; j++) x[j] = y[j * stride];
  if (kind == FFTW_REDFT10) {          // Y_k = 2 sum x_j cos(pi (j+1/2) k / n)
    for (int j = 0; j < n; j++) { w[2 * j + 1] = x[j]; w[4 * n - 2 * j - 1] = x[j]; }
    d4n.forward(w.data());
    for (int k = 0; k < n; k++) y[k * stride] = w[k].real();
  } else if (kind == FFTW_REDFT01) {   // Y_k = x_0 + 2 sum_{j>=1} x_j cos(pi j (k+1/2)/n)
    w[0] = x[0];
    for (int j = 1; j < n; j++) { w[j] = x[j]; w[4 * n - j] = x[j]; }
    d4n.forward(w.data());
    for (int k = 0; k < n; k++) y[k * stride] = w[2 * k + 1].real();
  } else if (kind == FFTW_RODFT10) {   // Y_k = 2 sum x_j sin(pi (j+1/2)(k+1)/n)
    for (int j = 0; j < n; j++) { w[2 * j + 1] = x[j]; w[4 * n - 2 * j - 1] = -x[j]; }
    d4n.forward(w.data());
    for (int k = 0; k < n; k++) y[k * stride] = -w[k + 1].imag();
  } else if (kind == FFTW_RODFT01) {   // Y_k = (-1)^k x_{n-1} + 2 sum_{j<n-1} x_j sin(pi (j+1)(k+1/2)/n)
    for (int j = 0; j < n; j++) {
      const double v = (j == n - 1) ? x[j] : 2 * x[j];
      // sum_j v_j sin(pi (j+1)(2k+1)/(2n)) = -Im sum_m u_m e^{-2 pi i m (2k+1)/(4n)}
      w[j + 1] += 0.5 * v; w[4 * n - j - 1] -= 0.5 * v;
    }
    d4n.forward(w.data());
    for (int k = 0; k < n; k++) y[k * stride] = -w[2 * k + 1].imag();
  } else {
    std::abort();
  }
}

void exec_double(fftw_plan_s* p, double* rin, double* rout) {
  const int n0 = p->n0, n1 = p->n1, nh = n1 / 2 + 1;
  if (p->type == R2C) {
    // rin: n0 rows of n1 reals with row stride 2*nh (in place) ; out complex n0 x nh
    cplx* out = reinterpret_cast<cplx*>(rout);
    const long istride = (rin == rout) ? 2L * nh : n1;
    #pragma omp parallel
    {
      std::vector<cplx> row(n1);
      #pragma omp for schedule(static)
      for (int j = 0; j < n0; j++) {
        for (int i = 0; i < n1; i++) row[i] = cplx(rin[j * istride + i], 0);
        p->d1->forward(row.data());
        for (int i = 0; i < nh; i++) out[(long)j * nh + i] = row[i];
      }
      std::vector<cplx> col(n0);
      #pragma omp for schedule(static)
      for (int i = 0; i < nh; i++) {
        for (int j = 0; j < n0; j++) col[j] = out[(long)j * nh + i];
        p->d0->forward(col.data());
        for (int j = 0; j < n0; j++) out[(long)j * nh + i] = col[j];
      }
    }
  } else if (p->type == C2R) {
    cplx* in = reinterpret_cast<cplx*>(rin);
    const long ostride = (rin == rout) ? 2L * nh : n1;
    #pragma omp parallel
    {
      std::vector<cplx> col(n0);
      #pragma omp for schedule(static)
      for (int i = 0; i < nh; i++) {
        for (int j = 0; j < n0; j++) col[j] = in[(long)j * nh + i];
        p->d0->backward(col.data());
        for (int j = 0; j < n0; j++) in[(long)j * nh + i] = col[j];
      }
      std::vector<cplx> row(n1);
      #pragma omp for schedule(static)
      for (int j = 0; j < n0; j++) {
        for (int i = 0; i < nh; i++) row[i] = in[(long)j * nh + i];
        for (int i = nh; i < n1; i++) row[i] = std::conj(row[n1 - i]);
        p->d1->backward(row.data());
        // rows are written after all of this row's inputs were read
        for (int i = 0; i < n1; i++) rout[j * ostride + i] = row[i].real();
      }
    }
  } else {
    if (rin != rout) std::memcpy(rout, rin, sizeof(double) * (size_t)n0 * n1);
    #pragma omp parallel for schedule(static)
    for (int j = 0; j < n0; j++) r2r_line(rout + (long)j * n1, n1, 1, p->k1, *p->d1);
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < n1; i++) r2r_line(rout + i, n0, n1, p->k0, *p->d0);
  }
}

fftw_plan_s* make_plan(int type, int n0, int n1, void* in, void* out, int k0, int k1, bool single) {
  fftw_plan_s* p = new fftw_plan_s();
  p->type = type; p->n0 = n0; p->n1 = n1; p->in = in; p->out = out;
  p->k0 = k0; p->k1 = k1; p->single = single;
  if (type == R2R) { p->d0 = new Dft1D(4 * n0); p->d1 = new Dft1D(4 * n1); }
  else { p->d0 = new Dft1D(n0); p->d1 = new Dft1D(n1); }
  return p;
}
} // namespace

extern "C++" {
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int) {}
void fftw_cleanup_threads(void) {}
static void* alloc64(size_t bytes) { void* p = nullptr; if (posix_memalign(&p, 64, bytes ? bytes : 64)) return nullptr; return p; }
double* fftw_alloc_real(size_t n) { return (double*)alloc64(n * sizeof(double)); }
void fftw_free(void* p) { std::free(p); }
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double* in, fftw_complex* out, unsigned) {
  return make_plan(R2C, n0, n1, in, out, 0, 0, false);
}
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex* in, double* out, unsigned) {
  return make_plan(C2R, n0, n1, in, out, 0, 0, false);
}
fftw_plan fftw_plan_r2r_2d(int n0, int n1, double* in, double* out, fftw_r2r_kind k0, fftw_r2r_kind k1, unsigned) {
  return make_plan(R2R, n0, n1, in, out, k0, k1, false);
}
void fftw_execute(const fftw_plan p) { exec_double(p, (double*)p->in, (double*)p->out); }
void fftw_destroy_plan(fftw_plan p) { delete p; }

// single precision entry points: computed in double, rounded on output
int fftwf_init_threads(void) { return 1; }
void fftwf_plan_with_nthreads(int) {}
void fftwf_cleanup_threads(void) {}
float* fftwf_alloc_real(size_t n) { return (float*)alloc64(n * sizeof(float)); }
void fftwf_free(void* p) { std::free(p); }
fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float* in, fftwf_complex* out, unsigned) {
  return make_plan(R2C, n0, n1, in, out, 0, 0, true);
}
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex* in, float* out, unsigned) {
  return make_plan(C2R, n0, n1, in, out, 0, 0, true);
}
fftwf_plan fftwf_plan_r2r_2d(int n0, int n1, float* in, float* out, fftw_r2r_kind k0, fftw_r2r_kind k1, unsigned) {
  return make_plan(R2R, n0, n1, in, out, k0, k1, true);
}
void fftwf_execute(const fftwf_plan p) {
  const size_t nreal = (p->type == R2R) ? (size_t)p->n0 * p->n1 : 2 * (size_t)p->n0 * (p->n1 / 2 + 1);
  std::vector<double> a(nreal), b(nreal);
  const float* fin = (const float*)p->in;
  for (size_t i = 0; i < nreal; i++) a[i] = fin[i];
  const bool inplace = p->in == p->out;
  exec_double(p, a.data(), inplace ? a.data() : b.data());
  const double* r = inplace ? a.data() : b.data();
  float* fout = (float*)p->out;
  for (size_t i = 0; i < nreal; i++) fout[i] = (float)r[i];
}
void fftwf_destroy_plan(fftwf_plan p) { delete p; }
}
