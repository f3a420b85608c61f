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
// FFTs are Stockham radix-2 in shared memory with twiddles from one
// host-computed table; one CTA transforms several rows (or columns) at once.
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

// Stockham autosort radix-2 FFT of nb sequences of length L (A -> result,
// B scratch), forward exp(-2 pi i jk/L) or inverse exp(+...), unnormalised.
__device__ double2* fft_stockham(double2* A, double2* B, int L, int nb, const double2* __restrict__ tw,
                                 int twLen, bool inverse)
{
  const int half = L >> 1, tid = threadIdx.x, nt = blockDim.x;
  for (int Ns = 1; Ns < L; Ns <<= 1) {
    const int twStep = twLen / (2 * Ns);
    for (int idx = tid; idx < nb * half; idx += nt) {
      const int seq = idx / half, j = idx - seq * half;
      const double2* a = A + seq * L;
      double2* b = B + seq * L;
      const int k = j & (Ns - 1);
      double2 w = tw[k * twStep];
      if (inverse) w.y = -w.y;
      const double2 x0 = a[j], t = cmul(w, a[j + half]);
      const int o = ((j - k) << 1) + k;
      b[o] = cadd(x0, t);
      b[o + Ns] = csub(x0, t);
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
__global__ void __launch_bounds__(512)
k_rows_r2c(const double* in, int inStride, int nrows, int ncolsIn, int inMode,
           double2* __restrict__ out, int outStride, int L, int rb,
           const double2* __restrict__ tw, int twLen, FadeArgs fa, double h, int Nx, int Ny)
{
  extern __shared__ double2 sm[];
  double2* A = sm;
  double2* B = sm + rb * L;
  const int row0 = blockIdx.x * rb;
  const int nb = min(rb, nrows - row0);
  const double corr = fa.enabled ? fa.sc->fadeCorr : 0.0;
  // fade band: cells within fadeLen (+2 cells margin) of an edge
  const int bandX = fa.enabled ? (int)(fa.g.fadeLenX / fa.g.h) + 2 : 0;
  const int bandY = fa.enabled ? (int)(fa.g.fadeLenY / fa.g.h) + 2 : 0;
  for (int idx = threadIdx.x; idx < nb * L; idx += blockDim.x) {
    const int r = idx / L, n = idx - r * L, row = row0 + r;
    double x[2];
    for (int q = 0; q < 2; q++) {
      const int col = 2 * n + q;
      double val = 0;
      if (col < ncolsIn) {
        if (inMode == 0) {
          val = in[(size_t)row * inStride + col];
          if (fa.enabled && (col < bandX || col >= fa.g.nx - bandX || row < bandY || row >= fa.g.ny - bandY)) {
            val = fade_cell(fa.g, col, row, val, corr);
            fa.writeback[(size_t)row * inStride + col] = val;
          }
        } else {
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
        }
      }
      x[q] = val;
    }
    A[r * L + n] = make_double2(x[0], x[1]);
  }
  __syncthreads();
  double2* Z = fft_stockham(A, B, L, nb, tw, twLen, false);
  // even/odd split: X[k] = Fe[k] + W^k Fo[k], W = exp(-i pi / L), k in [0, L]
  const int twStep = twLen / (2 * L);
  for (int idx = threadIdx.x; idx < nb * (L + 1); idx += blockDim.x) {
    const int r = idx / (L + 1), k = idx - r * (L + 1);
    const double2 Zk = Z[r * L + (k == L ? 0 : k)];
    const double2 Zc = conjg(Z[r * L + (k == 0 ? 0 : L - k)]);
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
__global__ void __launch_bounds__(512)
k_cols(double2* __restrict__ data, int stride, int ncols, int nrowsIn, int nrowsOut, int L, int cb,
       double* __restrict__ ghat, int mode, const double2* __restrict__ tw, int twLen, double norm,
       int MXp, int MYp)
{
  extern __shared__ double2 sm[];
  double2* A = sm;
  double2* B = sm + cb * L;
  const int c0 = blockIdx.x * cb;
  const int nb = min(cb, ncols - c0);
  for (int idx = threadIdx.x; idx < nb * L; idx += blockDim.x) {
    const int r = idx / nb, j = idx - r * nb;     // consecutive threads: consecutive columns
    A[j * L + r] = r < nrowsIn ? data[(size_t)r * stride + c0 + j] : make_double2(0, 0);
  }
  __syncthreads();
  double2* Z = fft_stockham(A, B, L, nb, tw, twLen, false);
  if (mode == 1) {
    for (int idx = threadIdx.x; idx < nb * nrowsOut; idx += blockDim.x) {
      const int r = idx / nb, j = idx - r * nb;
      ghat[(size_t)r * stride + c0 + j] = Z[j * L + r].x * norm;
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
    double2 z = Z[j * L + r];
    if (mode == 2 && c0 + j == 0 && r == 0) z = make_double2(0, 0);
    Z[j * L + r] = make_double2(z.x * f, z.y * f);
  }
  __syncthreads();
  double2* Bn = (Z == A) ? B : A;
  double2* Y = fft_stockham(Z, Bn, L, nb, tw, twLen, true);
  for (int idx = threadIdx.x; idx < nb * nrowsOut; idx += blockDim.x) {
    const int r = idx / nb, j = idx - r * nb;
    data[(size_t)r * stride + c0 + j] = Y[j * L + r];
  }
}

// inverse real FFT of length 2L from X[0..L]; writes the first ncolsOut values
__global__ void __launch_bounds__(512)
k_rows_c2r(const double2* __restrict__ in, int inStride, int nrows, double* __restrict__ out,
           int outStride, int ncolsOut, int L, int rb, const double2* __restrict__ tw, int twLen)
{
  extern __shared__ double2 sm[];
  double2* A = sm;
  double2* B = sm + rb * L;
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
    A[r * L + k] = make_double2(s.x - t.y, s.y + t.x);   // s + i t
  }
  __syncthreads();
  double2* z = fft_stockham(A, B, L, nb, tw, twLen, true);
  for (int idx = threadIdx.x; idx < nb * ((ncolsOut + 1) / 2); idx += blockDim.x) {
    const int r = idx / ((ncolsOut + 1) / 2), n = idx - r * ((ncolsOut + 1) / 2);
    const double2 v = z[r * L + n];
    double* o = out + (size_t)(row0 + r) * outStride;
    o[2 * n] = v.x;
    if (2 * n + 1 < ncolsOut) o[2 * n + 1] = v.y;
  }
}

inline bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// The opt-in limit is raised to the device maximum once per kernel, so a
// context with a smaller grid never lowers it under a larger one.
void set_smem(const void* f, size_t bytes) {
  int dev = 0, maxOptin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxOptin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  (void)bytes;
  cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, maxOptin);
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
  if (!is_pow2(P->Lrow) || !is_pow2(P->Lcol)) { delete P; return nullptr; }
  P->nkx = P->Lrow + 1;
  P->twLen = 2 * (P->Lrow > P->Lcol ? P->Lrow : P->Lcol);
  std::vector<double2> tw(P->twLen);
  for (int k = 0; k < P->twLen; k++) {
    // exp(-2 pi i k / n) from the first octant for accuracy
    const long double a = -2.0L * 3.14159265358979323846264338327950288L * k / P->twLen;
    tw[k] = make_double2((double)cosl(a), (double)sinl(a));
  }
  const int maxL = P->Lrow > P->Lcol ? P->Lrow : P->Lcol;
  P->rb = 4096 / P->Lrow; if (P->rb < 1) P->rb = 1; if (P->rb > 8) P->rb = 8;
  P->cb = 4096 / P->Lcol; if (P->cb < 1) P->cb = 1; if (P->cb > 8) P->cb = 8;
  (void)maxL;
  if (cudaMalloc(&P->tw, sizeof(double2) * P->twLen) != cudaSuccess) { delete P; return nullptr; }
  cudaMemcpy(P->tw, tw.data(), sizeof(double2) * P->twLen, cudaMemcpyHostToDevice);
  const size_t specRows = (size_t)P->Lcol;
  if (cudaMalloc(&P->spec, sizeof(double2) * specRows * P->nkx) != cudaSuccess) { delete P; return nullptr; }
  set_smem((const void*)k_rows_r2c, sizeof(double2) * 2 * P->rb * P->Lrow);
  set_smem((const void*)k_rows_c2r, sizeof(double2) * 2 * P->rb * P->Lrow);
  set_smem((const void*)k_cols, sizeof(double2) * 2 * P->cb * P->Lcol);
  if (P->type == CUP2D_POISSON_FREESPACE) {
    // G^ = Re FFT[G] / (MX MY) on the (2Ny) x (2Nx) grid, kept for ky <= Ny
    if (cudaMalloc(&P->ghat, sizeof(double) * (P->Lcol / 2 + 1) * P->nkx) != cudaSuccess) { delete P; return nullptr; }
    FadeArgs fa{}; fa.enabled = 0;
    const int MYr = 2 * Ny;
    k_rows_r2c<<<(MYr + P->rb - 1) / P->rb, 512, sizeof(double2) * 2 * P->rb * P->Lrow, c.stream>>>(
        nullptr, 0, MYr, 2 * Nx, 1, P->spec, P->nkx, P->Lrow, P->rb, P->tw, P->twLen, fa, c.g.h, Nx, Ny);
    CUP2D_LAUNCHED(c);
    const double norm = 1.0 / ((double)(2 * Nx) * (double)(2 * Ny));
    k_cols<<<(P->nkx + P->cb - 1) / P->cb, 512, sizeof(double2) * 2 * P->cb * P->Lcol, c.stream>>>(
        P->spec, P->nkx, P->nkx, MYr, P->Lcol / 2 + 1, P->Lcol, P->cb, P->ghat, 1, P->tw, P->twLen,
        norm, 0, 0);
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
  k_rows_r2c<<<(Ny + P->rb - 1) / P->rb, 512, sizeof(double2) * 2 * P->rb * P->Lrow, c.stream>>>(
      c.rhs, Nx, Ny, Nx, 0, P->spec, P->nkx, P->Lrow, P->rb, P->tw, P->twLen, fa, c.g.h, Nx, Ny);
  CUP2D_LAUNCHED(c);
}

void poisson_cols(Ctx& c) {
  Poisson* P = c.poisson;
  const int Nx = c.g.nx, Ny = c.g.ny;
  if (P->type == CUP2D_POISSON_FREESPACE) {
    k_cols<<<(P->nkx + P->cb - 1) / P->cb, 512, sizeof(double2) * 2 * P->cb * P->Lcol, c.stream>>>(
        P->spec, P->nkx, P->nkx, Ny, Ny, P->Lcol, P->cb, P->ghat, 0, P->tw, P->twLen, 0.0, 0, 0);
  } else {
    const double norm = 1.0 / ((double)Nx * (double)Ny);
    k_cols<<<(P->nkx + P->cb - 1) / P->cb, 512, sizeof(double2) * 2 * P->cb * P->Lcol, c.stream>>>(
        P->spec, P->nkx, P->nkx, Ny, Ny, P->Lcol, P->cb, nullptr, 2, P->tw, P->twLen, norm, Nx, Ny);
  }
  CUP2D_LAUNCHED(c);
}

void poisson_rows_inv(Ctx& c) {
  Poisson* P = c.poisson;
  const int Nx = c.g.nx, Ny = c.g.ny;
  k_rows_c2r<<<(Ny + P->rb - 1) / P->rb, 512, sizeof(double2) * 2 * P->rb * P->Lrow, c.stream>>>(
      P->spec, P->nkx, Ny, c.pres, Nx, Nx, P->Lrow, P->rb, P->tw, P->twLen);
  CUP2D_LAUNCHED(c);
}

void poisson_solve(Ctx& c) {
  poisson_rows_fwd(c);
  poisson_cols(c);
  poisson_rows_inv(c);
}

} // namespace cup2d
