// Poisson solvers of PressureSingle (Poisson/PoissonSolver.cpp:23-59):
//  - free space (Poisson/FFTW_freespace.cpp): Hockney convolution of the
//    RHS with the sampled Green's function ln(h r)/(2 pi) on a zero-padded
//    grid, in three passes over HBM:
//      1. row pass  : fade (cub2rhs, PoissonSolver.cpp:61-141) on load, real
//                     FFT of length 2Nx of each of the Ny RHS rows (the
//                     zero half is never read), as a complex FFT of length
//                     Nx plus the even/odd split;
//      2. column pass: complex FFT of length 2Ny of each of the Nx+1
//                     spectrum columns (only Ny rows are non-zero), times
//                     the real kernel G^, inverse FFT, keep Ny rows;
//      3. row pass  : inverse real FFT, keep Nx outputs = the pressure.
//    The padded size is 2N instead of the reference's 2N-1: the cyclic
//    convolution over offsets |d| <= N-1 is the same linear convolution
//    either way (the extra offset N only ever multiplies zero padding), and
//    power-of-two lengths keep every FFT in shared memory.
//  - periodic (Poisson/FFTW_periodic.h:77-166): the same passes without
//    padding and with the spectral multiplier -1/|k|^2.
// FFTs are compile-time-length Stockham radix-4 (one radix-2 stage when
// log2 L is odd) in shared memory padded by one element per 16 against bank
// conflicts, twiddles from one host-computed table; one CTA transforms a few
// rows (or columns) with L/4 threads each.
#include <cmath>
#include <vector>
#include "context.hpp"

namespace cup2d {

struct Poisson {
  int type = CUP2D_POISSON_FREESPACE;
  int Lrow = 0;          // complex FFT length of the row passes (M/2)
  int Lcol = 0;          // complex FFT length of the column pass
  int nkx = 0;           // spectrum columns (Lrow + 1)
  double2* spec = nullptr;   // [Lcol rows][nkx] row-major spectrum
  double* ghat = nullptr;    // [Lcol/2 + 1][nkx] free-space kernel
  double2* tw = nullptr;     // exp(-2 pi i k / twLen)
  int twLen = 0;
  int rb = 1, cb = 1;        // rows / columns per CTA
};

namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 conjg(double2 a) { return make_double2(a.x, -a.y); }

__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }
template <int L> struct Len { static constexpr int SL = L + L / 16; };   // padded stride

// Stockham autosort FFT (radix-4 stages, plus one radix-2 stage first when
// log2 L is odd) of nseq sequences of length L stored at A + q*SL (padded
// indexing), B scratch.  Forward exp(-2 pi i jk/L), inverse exp(+...),
// unnormalised.  Returns the buffer holding the result.
template <int L, bool INV>
__device__ double2* fft4(double2* A, double2* B, int nseq, const double2* __restrict__ tw, int twLen)
{
  constexpr int SL = Len<L>::SL, Q = L / 4, H = L / 2;
  const int tid = threadIdx.x, nt = blockDim.x;
  int Ns = 1;
  if ((__builtin_ctz(L) & 1) == 1) {
    for (int idx = tid; idx < nseq * H; idx += nt) {
      const int q = idx / H, j = idx - q * H;
      const double2* a = A + q * SL;
      double2* b = B + q * SL;
      const double2 x0 = a[pad(j)], x1 = a[pad(j + H)];
      b[pad(2 * j)] = cadd(x0, x1);
      b[pad(2 * j + 1)] = csub(x0, x1);
    }
    __syncthreads();
    double2* T = A; A = B; B = T;
    Ns = 2;
  }
  for (; Ns < L; Ns <<= 2) {
    const int twStep = twLen / (4 * Ns);
    for (int idx = tid; idx < nseq * Q; idx += nt) {
      const int q = idx / Q, j = idx - q * Q;
      const double2* a = A + q * SL;
      double2* b = B + q * SL;
      const int k = j & (Ns - 1);
      double2 x0 = a[pad(j)], x1 = a[pad(j + Q)], x2 = a[pad(j + 2 * Q)], x3 = a[pad(j + 3 * Q)];
      if (k) {
        double2 w1 = tw[k * twStep], w2 = tw[2 * k * twStep], w3 = tw[3 * k * twStep];
        if (INV) { w1.y = -w1.y; w2.y = -w2.y; w3.y = -w3.y; }
        x1 = cmul(w1, x1); x2 = cmul(w2, x2); x3 = cmul(w3, x3);
      }
      const double2 t0 = cadd(x0, x2), t1 = csub(x0, x2), t2 = cadd(x1, x3), t3 = csub(x1, x3);
      const int o = ((j - k) << 2) + k;
      b[pad(o)] = cadd(t0, t2);
      b[pad(o + 2 * Ns)] = csub(t0, t2);
      if (!INV) {
        b[pad(o + Ns)] = make_double2(t1.x + t3.y, t1.y - t3.x);       // t1 - i t3
        b[pad(o + 3 * Ns)] = make_double2(t1.x - t3.y, t1.y + t3.x);   // t1 + i t3
      } else {
        b[pad(o + Ns)] = make_double2(t1.x - t3.y, t1.y + t3.x);
        b[pad(o + 3 * Ns)] = make_double2(t1.x + t3.y, t1.y - t3.x);
      }
    }
    __syncthreads();
    double2* T = A; A = B; B = T;
  }
  return A;
}

struct FadeArgs {
  int enabled;
  const Scalars* sc;
  GridDesc g;
  double* writeback;     // rhs buffer receives the faded values (cub2rhs writes tmp)
};

// PoissonSolver::cub2rhs (PoissonSolver.cpp:101-125) for one cell
__device__ __forceinline__ double fade_cell(const GridDesc& g, int gx, int gy, double b, double corr) {
  const double EPSd = 2.220446049250313e-16;
  const double fadeLenX = g.fadeLenX, invFadeX = 1 / fmax(fadeLenX, EPSd);
  const double fadeLenY = g.fadeLenY, invFadeY = 1 / fmax(fadeLenY, EPSd);
  const double px = gx_pos(g, gx), py = gy_pos(g, gy);
  const double yt = invFadeY * fmax(0.0, fadeLenY - g.ext[1] + py);
  const double yb = invFadeY * fmax(0.0, fadeLenY - py);
  const double xt = invFadeX * fmax(0.0, fadeLenX - g.ext[0] + px);
  const double xb = invFadeX * fmax(0.0, fadeLenX - px);
  const double fadeArg = fmin(fmax(fmax(yt, yb), fmax(xt, xb)), 1.0);
  const double f2 = fadeArg * fadeArg;
  const double fadeRHS = b * f2;
  const double fadeCorrection = corr * (corr > 0 ? fmax(fadeRHS, 0.0) : -fmin(fadeRHS, 0.0));
  return b * (1 - f2) + fadeCorrection;
}

// inMode 0: rows of `in`; 1: the free-space Green's function on the padded
// grid (FFTW_freespace.cpp:108-119) computed on the fly.
template <int L>
__global__ void __launch_bounds__(1024)
k_rows_r2c(const double* in, int inStride, int nrows, int ncolsIn, int inMode,
           double2* __restrict__ out, int outStride, int rb,
           const double2* __restrict__ tw, int twLen, FadeArgs fa, double h, int Nx, int Ny)
{
  constexpr int SL = Len<L>::SL;
  extern __shared__ double2 sm[];
  double2* A = sm;
  double2* B = sm + rb * SL;
  const int row0 = blockIdx.x * rb;
  const int nb = min(rb, nrows - row0);
  const double corr = fa.enabled ? fa.sc->fadeCorr : 0.0;
  // fade band: cells within fadeLen (+2 cells margin) of an edge
  const int bandX = fa.enabled ? (int)(fa.g.fadeLenX / fa.g.h) + 2 : 0;
  const int bandY = fa.enabled ? (int)(fa.g.fadeLenY / fa.g.h) + 2 : 0;
  for (int idx = threadIdx.x; idx < nb * L; idx += blockDim.x) {
    const int r = idx / L, n = idx - r * L, row = row0 + r;
    double x[2];
    if (inMode == 0 && 2 * n + 1 < ncolsIn) {
      const double2 v2 = *reinterpret_cast<const double2*>(in + (size_t)row * inStride + 2 * n);
      x[0] = v2.x; x[1] = v2.y;
      if (fa.enabled) {
        const bool rowBand = row < bandY || row >= fa.g.ny - bandY;
        for (int q = 0; q < 2; q++) {
          const int col = 2 * n + q;
          if (rowBand || col < bandX || col >= fa.g.nx - bandX) {
            x[q] = fade_cell(fa.g, col, row, x[q], corr);
            fa.writeback[(size_t)row * inStride + col] = x[q];
          }
        }
      }
    } else {
      for (int q = 0; q < 2; q++) {
        const int col = 2 * n + q;
        double val = 0;
        if (col < ncolsIn && inMode == 1) {
          const int MX = 2 * Nx, MY = 2 * Ny;
          const double fac = 1 / (2 * M_PI);
          if (row == 0 && col == 0) {
            val = fac / 2 * (2 * log(h / sqrt(M_PI)) - 1);
          } else {
            const double yi = row >= Ny ? MY - row : row;
            const double xi = col >= Nx ? MX - col : col;
            const double rr = sqrt(xi * xi + yi * yi);
            val = fac * log(h * rr);
          }
        } else if (col < ncolsIn) {
          val = in[(size_t)row * inStride + col];
        }
        x[q] = val;
      }
    }
    A[r * SL + pad(n)] = make_double2(x[0], x[1]);
  }
  __syncthreads();
  double2* Z = fft4<L, false>(A, B, nb, tw, twLen);
  // even/odd split: X[k] = Fe[k] + W^k Fo[k], W = exp(-i pi / L), k in [0, L]
  const int twStep = twLen / (2 * L);
  for (int idx = threadIdx.x; idx < nb * (L + 1); idx += blockDim.x) {
    const int r = idx / (L + 1), k = idx - r * (L + 1);
    const double2 Zk = Z[r * SL + pad(k == L ? 0 : k)];
    const double2 Zc = conjg(Z[r * SL + pad(k == 0 ? 0 : L - k)]);
    const double2 Fe = make_double2(0.5 * (Zk.x + Zc.x), 0.5 * (Zk.y + Zc.y));
    const double2 d = csub(Zk, Zc);
    const double2 Fo = make_double2(0.5 * d.y, -0.5 * d.x);   // (Zk - Zc) / (2i)
    const double2 X = cadd(Fe, cmul(tw[k * twStep], Fo));
    out[(size_t)(row0 + r) * outStride + k] = X;
  }
}

// mode 0: forward, x G^ (real, symmetric in ky), inverse, keep nrowsOut rows
// mode 1: forward; write Re * norm for ky <= L/2 into ghat (kernel set-up)
// mode 2: forward, periodic multiplier -1/|k|^2 / (MX MY), inverse
template <int L>
__global__ void __launch_bounds__(1024)
k_cols(double2* __restrict__ data, int stride, int ncols, int nrowsIn, int nrowsOut, int cb,
       double* __restrict__ ghat, int mode, const double2* __restrict__ tw, int twLen, double norm,
       int MXp, int MYp)
{
  constexpr int SL = Len<L>::SL;
  extern __shared__ double2 sm[];
  double2* A = sm;
  double2* B = sm + cb * SL;
  const int c0 = blockIdx.x * cb;
  const int nb = min(cb, ncols - c0);
  for (int idx = threadIdx.x; idx < nb * L; idx += blockDim.x) {
    const int r = idx / nb, j = idx - r * nb;     // consecutive threads: consecutive columns
    A[j * SL + pad(r)] = r < nrowsIn ? data[(size_t)r * stride + c0 + j] : make_double2(0, 0);
  }
  __syncthreads();
  double2* Z = fft4<L, false>(A, B, nb, tw, twLen);
  if (mode == 1) {
    for (int idx = threadIdx.x; idx < nb * nrowsOut; idx += blockDim.x) {
      const int r = idx / nb, j = idx - r * nb;
      ghat[(size_t)r * stride + c0 + j] = Z[j * SL + pad(r)].x * norm;
    }
    return;
  }
  for (int idx = threadIdx.x; idx < nb * L; idx += blockDim.x) {
    const int r = idx / nb, j = idx - r * nb;
    double f;
    if (mode == 0) {
      const int ky = r <= L / 2 ? r : L - r;
      f = ghat[(size_t)ky * stride + c0 + j];
    } else {
      // FFTW_periodic::_solve_spectral (FFTW_periodic.h:77-92)
      const int i = c0 + j;
      const int kx = i <= MXp / 2 ? i : MXp - i, ky = r <= MYp / 2 ? r : MYp - r;
      const double waveFactX = 2 * M_PI / MXp, waveFactY = 2 * M_PI / MYp;
      const double rkx = kx * waveFactX, rky = ky * waveFactY;
      const double kinv = -1 / (rkx * rkx + rky * rky);
      f = (i == 0 && r == 0) ? 0.0 : kinv * norm;
    }
    double2 z = Z[j * SL + pad(r)];
    if (mode == 2 && c0 + j == 0 && r == 0) z = make_double2(0, 0);
    Z[j * SL + pad(r)] = make_double2(z.x * f, z.y * f);
  }
  __syncthreads();
  double2* Bn = (Z == A) ? B : A;
  double2* Y = fft4<L, true>(Z, Bn, nb, tw, twLen);
  for (int idx = threadIdx.x; idx < nb * nrowsOut; idx += blockDim.x) {
    const int r = idx / nb, j = idx - r * nb;
    data[(size_t)r * stride + c0 + j] = Y[j * SL + pad(r)];
  }
}

// inverse real FFT of length 2L from X[0..L]; writes the first ncolsOut values
template <int L>
__global__ void __launch_bounds__(1024)
k_rows_c2r(const double2* __restrict__ in, int inStride, int nrows, double* __restrict__ out,
           int outStride, int ncolsOut, int rb, const double2* __restrict__ tw, int twLen)
{
  constexpr int SL = Len<L>::SL;
  extern __shared__ double2 sm[];
  double2* A = sm;
  double2* B = sm + rb * SL;
  const int row0 = blockIdx.x * rb;
  const int nb = min(rb, nrows - row0);
  const int twStep = twLen / (2 * L);
  for (int idx = threadIdx.x; idx < nb * L; idx += blockDim.x) {
    const int r = idx / L, k = idx - r * L;
    const double2* X = in + (size_t)(row0 + r) * inStride;
    double2 Xk = X[k], XL = X[L - k];
    if (k == 0) { Xk.y = 0; XL.y = 0; }         // c2r ignores Im X[0], Im X[L]
    const double2 Xc = conjg(XL);
    const double2 s = cadd(Xk, Xc), d = csub(Xk, Xc);
    const double2 wi = conjg(tw[k * twStep]);   // W^-k
    const double2 t = cmul(wi, d);
    A[r * SL + pad(k)] = make_double2(s.x - t.y, s.y + t.x);   // s + i t
  }
  __syncthreads();
  double2* z = fft4<L, true>(A, B, nb, tw, twLen);
  const int half = (ncolsOut + 1) / 2;
  for (int idx = threadIdx.x; idx < nb * half; idx += blockDim.x) {
    const int r = idx / half, n = idx - r * half;
    const double2 v = z[r * SL + pad(n)];
    double* o = out + (size_t)(row0 + r) * outStride;
    if (2 * n + 1 < ncolsOut) *reinterpret_cast<double2*>(o + 2 * n) = v;
    else o[2 * n] = v.x;
  }
}

inline bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// The opt-in limit is raised to the device maximum once per kernel, so a
// context with a smaller grid never lowers it under a larger one.
void set_smem(const void* f) {
  int dev = 0, maxOptin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxOptin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, maxOptin);
}

inline int batch_for(int L) { int b = 2048 / L; return b < 1 ? 1 : (b > 8 ? 8 : b); }
inline int threads_for(int L, int b) { int t = b * L / 4; return t < 64 ? 64 : (t > 1024 ? 1024 : t); }
template <int L> inline size_t smem_for(int b) { return sizeof(double2) * 2 * (size_t)b * Len<L>::SL; }

#define CUP2D_FFT_LENGTHS(X) X(64) X(128) X(256) X(512) X(1024) X(2048) X(4096)

void set_all_smem() {
#define X(L) set_smem((const void*)k_rows_r2c<L>); set_smem((const void*)k_rows_c2r<L>); \
             set_smem((const void*)k_cols<L>);
  CUP2D_FFT_LENGTHS(X)
#undef X
}

bool rows_r2c(int L, cudaStream_t st, const double* in, int inStride, int nrows, int ncolsIn, int inMode,
              double2* out, int outStride, const double2* tw, int twLen, FadeArgs fa, double h, int Nx, int Ny) {
  const int b = batch_for(L), grid = (nrows + b - 1) / b, thr = threads_for(L, b);
  switch (L) {
#define X(LL) case LL: k_rows_r2c<LL><<<grid, thr, smem_for<LL>(b), st>>>(in, inStride, nrows, ncolsIn, \
                  inMode, out, outStride, b, tw, twLen, fa, h, Nx, Ny); return true;
    CUP2D_FFT_LENGTHS(X)
#undef X
  }
  return false;
}

bool cols(int L, cudaStream_t st, double2* data, int stride, int ncols, int nrowsIn, int nrowsOut,
          double* ghat, int mode, const double2* tw, int twLen, double norm, int MXp, int MYp) {
  const int b = batch_for(L), grid = (ncols + b - 1) / b, thr = threads_for(L, b);
  switch (L) {
#define X(LL) case LL: k_cols<LL><<<grid, thr, smem_for<LL>(b), st>>>(data, stride, ncols, nrowsIn, \
                  nrowsOut, b, ghat, mode, tw, twLen, norm, MXp, MYp); return true;
    CUP2D_FFT_LENGTHS(X)
#undef X
  }
  return false;
}

bool rows_c2r(int L, cudaStream_t st, const double2* in, int inStride, int nrows, double* out, int outStride,
              int ncolsOut, const double2* tw, int twLen) {
  const int b = batch_for(L), grid = (nrows + b - 1) / b, thr = threads_for(L, b);
  switch (L) {
#define X(LL) case LL: k_rows_c2r<LL><<<grid, thr, smem_for<LL>(b), st>>>(in, inStride, nrows, out, \
                  outStride, ncolsOut, b, tw, twLen); return true;
    CUP2D_FFT_LENGTHS(X)
#undef X
  }
  return false;
}

} // namespace

Poisson* poisson_create(Ctx& c) {
  Poisson* P = new Poisson();
  P->type = c.cfg.poisson;
  const int Nx = c.g.nx, Ny = c.g.ny;
  if (P->type == CUP2D_POISSON_FREESPACE) {
    P->Lrow = Nx;          // real length 2Nx
    P->Lcol = 2 * Ny;
  } else if (P->type == CUP2D_POISSON_PERIODIC) {
    P->Lrow = Nx / 2;      // real length Nx
    P->Lcol = Ny;
  } else {
    delete P;
    return nullptr;        // cosine transform solver: not in this build
  }
  if (!is_pow2(P->Lrow) || !is_pow2(P->Lcol) || P->Lrow < 64 || P->Lcol < 64 ||
      P->Lrow > 4096 || P->Lcol > 4096) { delete P; return nullptr; }   // shared-memory limit
  P->nkx = P->Lrow + 1;
  P->twLen = 2 * (P->Lrow > P->Lcol ? P->Lrow : P->Lcol);
  std::vector<double2> tw(P->twLen);
  for (int k = 0; k < P->twLen; k++) {
    const long double a = -2.0L * 3.14159265358979323846264338327950288L * k / P->twLen;
    tw[k] = make_double2((double)cosl(a), (double)sinl(a));
  }
  if (cudaMalloc(&P->tw, sizeof(double2) * P->twLen) != cudaSuccess) { delete P; return nullptr; }
  cudaMemcpy(P->tw, tw.data(), sizeof(double2) * P->twLen, cudaMemcpyHostToDevice);
  const size_t specRows = (size_t)P->Lcol;
  if (cudaMalloc(&P->spec, sizeof(double2) * specRows * P->nkx) != cudaSuccess) { poisson_destroy(P); return nullptr; }
  set_all_smem();
  if (P->type == CUP2D_POISSON_FREESPACE) {
    // G^ = Re FFT[G] / (MX MY) on the (2Ny) x (2Nx) grid, kept for ky <= Ny
    if (cudaMalloc(&P->ghat, sizeof(double) * (P->Lcol / 2 + 1) * P->nkx) != cudaSuccess) { poisson_destroy(P); return nullptr; }
    FadeArgs fa{}; fa.enabled = 0;
    const int MYr = 2 * Ny;
    rows_r2c(P->Lrow, c.stream, nullptr, 0, MYr, 2 * Nx, 1, P->spec, P->nkx, P->tw, P->twLen, fa, c.g.h, Nx, Ny);
    CUP2D_LAUNCHED(c);
    const double norm = 1.0 / ((double)(2 * Nx) * (double)(2 * Ny));
    cols(P->Lcol, c.stream, P->spec, P->nkx, P->nkx, MYr, P->Lcol / 2 + 1, P->ghat, 1, P->tw, P->twLen, norm, 0, 0);
    CUP2D_LAUNCHED(c);
  }
  return P;
}

void poisson_destroy(Poisson* P) {
  if (!P) return;
  cudaFree(P->spec); cudaFree(P->ghat); cudaFree(P->tw);
  delete P;
}

// PoissonSolver::solve: cub2rhs (fade, reductions in launch_fade_sums), the
// transform passes, sol2cub (the inverse row pass writes pres directly).
void poisson_rows_fwd(Ctx& c) {
  Poisson* P = c.poisson;
  const int Nx = c.g.nx, Ny = c.g.ny;
  FadeArgs fa{1, c.dsc, c.g, c.rhs};
  rows_r2c(P->Lrow, c.stream, c.rhs, Nx, Ny, Nx, 0, P->spec, P->nkx, P->tw, P->twLen, fa, c.g.h, Nx, Ny);
  CUP2D_LAUNCHED(c);
}

void poisson_cols(Ctx& c) {
  Poisson* P = c.poisson;
  const int Nx = c.g.nx, Ny = c.g.ny;
  if (P->type == CUP2D_POISSON_FREESPACE) {
    cols(P->Lcol, c.stream, P->spec, P->nkx, P->nkx, Ny, Ny, P->ghat, 0, P->tw, P->twLen, 0.0, 0, 0);
  } else {
    const double norm = 1.0 / ((double)Nx * (double)Ny);
    cols(P->Lcol, c.stream, P->spec, P->nkx, P->nkx, Ny, Ny, nullptr, 2, P->tw, P->twLen, norm, Nx, Ny);
  }
  CUP2D_LAUNCHED(c);
}

void poisson_rows_inv(Ctx& c) {
  Poisson* P = c.poisson;
  const int Nx = c.g.nx, Ny = c.g.ny;
  rows_c2r(P->Lrow, c.stream, P->spec, P->nkx, Ny, c.pres, Nx, Nx, P->tw, P->twLen);
  CUP2D_LAUNCHED(c);
}

void poisson_solve(Ctx& c) {
  poisson_rows_fwd(c);
  poisson_cols(c);
  poisson_rows_inv(c);
}

} // namespace cup2d
