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
#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>
#include "context.hpp"

namespace cup2d {

struct Poisson {
  int type = CUP2D_POISSON_FREESPACE;
  float* cosX = nullptr;     // cosine solver: float tables of FFTW_dirichlet.h:75-76
  float* cosY = nullptr;
  double tol = 0.1;          // FFTW_dirichlet.h:51
  int Lrow = 0;          // complex FFT length of the row passes (M/2)
  int Lcol = 0;          // complex FFT length of the column pass
  int nkx = 0;           // spectrum columns (Lrow + 1)
  double2* spec = nullptr;   // [Lcol rows][nkx] row-major spectrum
  double* ghat = nullptr;    // [Lcol/2 + 1][nkx] free-space kernel
  double2* tw = nullptr;     // exp(-2 pi i k / twLen)
  int twLen = 0;
  bool fp32 = false;         // CUP2D_PREC_FP32: float2 spectrum in spec, FP32 passes
  float2* tw32 = nullptr;    // tw rounded to FP32
  float* ghat32 = nullptr;   // ghat rounded to FP32
  int rb = 1, cb = 1;        // rows / columns per CTA
  int MX = 0, MY = 0;        // free space: the padded grid (powers of two >= 2Nx, 2Ny)
  // elements per thread of the forward and inverse row passes (FP64 free
  // space and periodic), and the times the autotuner measured (us; r2c with
  // 8 and 16, c2r with 8 and 16; zero when not tuned)
  int eR2C = 8, eC2R = 16;
  bool tuned = false;
  double tuneUs[4] = {0, 0, 0, 0};
};

namespace {

// The transforms are written once for a complex type C: double2 (the FP64
// solve) or float2 (the FP32 solve of CUP2D_PREC_FP32).
template <class C> struct CT;
template <> struct CT<double2> { using R = double; };
template <> struct CT<float2> { using R = float; };
template <class C> __device__ __forceinline__ C mk(typename CT<C>::R a, typename CT<C>::R b);
template <> __device__ __forceinline__ double2 mk<double2>(double a, double b) { return make_double2(a, b); }
template <> __device__ __forceinline__ float2 mk<float2>(float a, float b) { return make_float2(a, b); }
template <class C> __device__ __forceinline__ C cmul(C a, C b) {
  return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class C> __device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <class C> __device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <class C> __device__ __forceinline__ C conjg(C a) { return mk<C>(a.x, -a.y); }

__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }

// Per transform length L: padded stride SL of one sequence (one spare
// element per 16, plus 4 so that consecutive sequences start in different
// halves of the shared-memory banks), the staged quarter twiddle table
// (w^j, j < L/4), the sequences per CTA B and the threads per CTA NT
// (L/E per sequence: every thread owns E = 16 or 8 elements of a pass).
// ---- per-pass twiddle tables ---------------------------------------------
// The passes of fft_inplace<L, ..., E> (fft_passes): sub-transform sizes
// NS = 1, E, E^2, ... with radix E while NS E <= L, then one pass of radix
// L/NS.  The pass over sub-transforms of size NS scales input m of the
// butterfly with k = j mod NS by W^(m k), W = exp(-2 pi i/(R NS)).  For each
// pass with NS > 1 the tables hold W^(p k), k < NS, for the powers p = 1, 2,
// 4, 8 below R (one table of NS entries each): the butterflies of a warp
// read consecutive entries (no shared-memory bank conflicts, where indexing
// one table by m k made every lane of a warp hit the same banks), and the
// other powers are products of at most three table values.
constexpr int tw_npow(int R) { return R >= 16 ? 4 : (R >= 8 ? 3 : (R >= 4 ? 2 : (R >= 2 ? 1 : 0))); }
// offset of the tables of the pass over sub-transforms of size NS
template <int L, int E> constexpr int tw_off(int NS) {
  int off = 0, ns = 1;
  while (ns < L && ns < NS) {
    const int r = ns * E <= L ? E : L / ns;
    if (ns > 1) off += tw_npow(r) * ns;
    ns *= r;
  }
  return off;
}
template <int L, int E> constexpr int tw_size() { return tw_off<L, E>(L); }
// entries staged per CTA: enough for the element counts E = 8 and 16
template <int L> constexpr int tw_max() {
  const int a = tw_size<L, 8>(), b = tw_size<L, 16>();
  return a > b ? (a > 0 ? a : 1) : (b > 0 ? b : 1);
}

template <int L, int E = 16> struct Len {
  static constexpr int SL = L + L / 16 + 4;
  static constexpr int TW = tw_max<L>();
  static constexpr int B = 2048 / L < 1 ? 1 : (2048 / L > 8 ? 8 : 2048 / L);
  static constexpr int NT0 = B * L / E;
  static constexpr int NT = NT0 < 64 ? 64 : (NT0 > 512 ? 512 : NT0);
  static constexpr int REGS = E == 16 ? 128 : 64;   // register budget per thread
  static constexpr int MINB = 65536 / (NT * REGS) < 1 ? 1 : 65536 / (NT * REGS);
};
// elements per thread: the row passes have two instantiations each (8 and
// 16: a forward row of 4096 points runs faster with 16, shorter rows with
// 8, measured on B200), chosen per grid at set-up (table below, or timed
// by poisson_autotune); the column pass uses 16 (faster at every length
// measured)
constexpr int E_ROWS = 8;
constexpr int E_C2R = 16;
constexpr int E_COLS = 16;
// the same for the FP32 transforms (half the registers per value)
constexpr int E_ROWS32 = 8;
constexpr int E_C2R32 = 8;
constexpr int E_COLS32 = 16;

constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }

// Stages the per-pass tables of fft_inplace<L, ..., E> from the global
// table tw[j] = exp(-2 pi i j / twLen) (twLen a power of two, a multiple of
// 4 L): the tables of the pass over sub-transforms of size NS and of every
// later pass.  Entry t = p NS + k of a pass of radix R holds
// W^(k 2^p) = tw[(k 2^p) twLen / (R NS)]; the passes' sizes are
// compile-time powers of two, so every index is a shift.
template <int L, int E, int NS, class C>
__device__ __forceinline__ void load_twiddles_from(C* tws, const C* __restrict__ tw, int twShift) {
  if constexpr (NS < L) {
    constexpr int R = NS * E <= L ? E : L / NS;
    if constexpr (NS > 1) {
      constexpr int n = tw_npow(R) * NS, off = tw_off<L, E>(NS), sh = ilog2(R * NS);
      for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int p = t / NS, k = t - p * NS;
        tws[off + t] = tw[(size_t)(k << p) << (twShift - sh)];
      }
    }
    load_twiddles_from<L, E, NS * R>(tws, tw, twShift);
  }
}
template <int L, int E, class C>
__device__ __forceinline__ void load_twiddles(C* tws, const C* __restrict__ tw, int twLen) {
  load_twiddles_from<L, E, 1>(tws, tw, __ffs(twLen) - 1);
}

// Scales xb[m], 0 < m < R, of the butterfly k of the pass over
// sub-transforms of size NS by W^(m k) (conjugated for the inverse).
template <int L, int E, int R, int NS, bool INV, class C>
__device__ __forceinline__ void apply_twiddles(C* xb, const C* tws, int k) {
  const C* t = tws + tw_off<L, E>(NS) + k;
  auto ld = [&](int pi) { C w = t[pi * NS]; if (INV) w.y = -w.y; return w; };
  const C w1 = ld(0);
  xb[1] = cmul(xb[1], w1);
  if constexpr (R > 2) {
    const C w2 = ld(1), w3 = cmul(w1, w2);
    xb[2] = cmul(xb[2], w2);
    xb[3] = cmul(xb[3], w3);
    if constexpr (R > 4) {
      const C w4 = ld(2);
      xb[4] = cmul(xb[4], w4);
      xb[5] = cmul(xb[5], cmul(w1, w4));
      xb[6] = cmul(xb[6], cmul(w2, w4));
      xb[7] = cmul(xb[7], cmul(w3, w4));
      if constexpr (R > 8) {
        const C w8 = ld(3), w12 = cmul(w4, w8);
        xb[8] = cmul(xb[8], w8);
        xb[9] = cmul(xb[9], cmul(w1, w8));
        xb[10] = cmul(xb[10], cmul(w2, w8));
        xb[11] = cmul(xb[11], cmul(w3, w8));
        xb[12] = cmul(xb[12], w12);
        xb[13] = cmul(xb[13], cmul(w1, w12));
        xb[14] = cmul(xb[14], cmul(w2, w12));
        xb[15] = cmul(xb[15], cmul(w3, w12));
      }
    }
  }
}

// asynchronous global -> shared copies (sm_80+ cp.async), so that every
// load of a CTA's rows or columns is in flight at once
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n"
               :: "r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n"
               :: "r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n"
               :: "r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src) : "memory");
}
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" :: "n"(N) : "memory");
}

// ---- small DFTs in registers (forward exp(-2 pi i mq/R), inverse exp(+)) --
// multiply by -i (forward) or +i (inverse)
template <bool INV, class C> __device__ __forceinline__ C mul_mi(C a) {
  return INV ? mk<C>(-a.y, a.x) : mk<C>(a.y, -a.x);
}
template <bool INV, class C>
__device__ __forceinline__ void dft4(C& x0, C& x1, C& x2, C& x3) {
  const C t0 = cadd(x0, x2), t1 = csub(x0, x2), t2 = cadd(x1, x3), t3 = mul_mi<INV>(csub(x1, x3));
  x0 = cadd(t0, t2); x2 = csub(t0, t2);
  x1 = cadd(t1, t3); x3 = csub(t1, t3);
}
constexpr double C8 = 0.92387953251128675613;   // cos(pi/8)
constexpr double S8 = 0.38268343236508977173;   // sin(pi/8)
constexpr double R2 = 0.70710678118654752440;   // sqrt(2)/2
// W16^e for e in [0, 16): the first quadrant from (1, C8, R2, S8), the rest
// by exact quarter turns
template <bool INV, class C>
__device__ __forceinline__ C w16(int e) {
  using R = typename CT<C>::R;
  const int q = e >> 2, r = e & 3;
  const R cr = (R)(r == 0 ? 1.0 : (r == 1 ? C8 : (r == 2 ? R2 : S8)));
  const R sr = (R)(r == 0 ? 0.0 : (r == 1 ? S8 : (r == 2 ? R2 : C8)));
  C v = mk<C>(cr, -sr);
  for (int k = 0; k < q; k++) v = mk<C>(v.y, -v.x);
  if (INV) v.y = -v.y;
  return v;
}
// DFT of R values in x[0..R); the result for output q is in x[out_reg<R>(q)]
template <int R> __device__ __forceinline__ constexpr int out_reg(int q) {
  return R == 16 ? 4 * (q & 3) + (q >> 2) : q;
}
template <bool INV, class C> __device__ __forceinline__ void dft8(C* x) {
  // m = m1 + 2 m2: DFT4 over m2, twiddle W8^(m1 q2), DFT2 over m1
  dft4<INV>(x[0], x[2], x[4], x[6]);
  dft4<INV>(x[1], x[3], x[5], x[7]);
  C y[8];
#pragma unroll
  for (int q2 = 0; q2 < 4; q2++) {
    const C z0 = x[2 * q2], z1 = cmul(x[2 * q2 + 1], w16<INV, C>(2 * q2));
    y[q2] = cadd(z0, z1); y[q2 + 4] = csub(z0, z1);
  }
#pragma unroll
  for (int q = 0; q < 8; q++) x[q] = y[q];
}
template <bool INV, class C> __device__ __forceinline__ void dft16(C* x) {
  // m = m1 + 4 m2: DFT4 over m2 (result z[m1][q2] in x[m1 + 4 q2]),
  // twiddle W16^(m1 q2), DFT4 over m1 (output q2 + 4 q1 in x[4 q2 + q1])
#pragma unroll
  for (int m1 = 0; m1 < 4; m1++) dft4<INV>(x[m1], x[m1 + 4], x[m1 + 8], x[m1 + 12]);
#pragma unroll
  for (int m1 = 1; m1 < 4; m1++)
#pragma unroll
    for (int q2 = 1; q2 < 4; q2++) x[m1 + 4 * q2] = cmul(x[m1 + 4 * q2], w16<INV, C>(m1 * q2));
#pragma unroll
  for (int q2 = 0; q2 < 4; q2++) dft4<INV>(x[4 * q2], x[4 * q2 + 1], x[4 * q2 + 2], x[4 * q2 + 3]);
}
template <int R, bool INV, class C> __device__ __forceinline__ void dft(C* x) {
  if constexpr (R == 2) { const C t = x[0]; x[0] = cadd(t, x[1]); x[1] = csub(t, x[1]); }
  else if constexpr (R == 4) dft4<INV>(x[0], x[1], x[2], x[3]);
  else if constexpr (R == 8) dft8<INV>(x);
  else dft16<INV>(x);
}

// pad(j + u T + m Q) given pj = pad(j): a multiple C of 16 added to an index
// adds C + C/16 to its padded position, an immediate offset
template <int T, int Q>
__device__ __forceinline__ int pad_at(int pj, int j, int u, int m) {
  if constexpr (T % 16 == 0 && Q % 16 == 0) return pj + u * (T + T / 16) + m * (Q + Q / 16);
  else return pad(j + u * T + m * Q);
}
// pad(o + q NS) given po = pad(o), for an output o of a pass over sub-transforms
// of size NS: with NS = 1, o is a multiple of R (a divisor of 16) and q < R
// stays inside o's group of 16
template <int NS>
__device__ __forceinline__ int pad_out(int po, int o, int q) {
  if constexpr (NS % 16 == 0) return po + q * (NS + NS / 16);
  else if constexpr (NS == 1) return po + q;
  else return pad(o + q * NS);
}

// One in-place Stockham pass of radix R over sub-transforms of size NS on
// nseq sequences A + q*SL: butterfly j (k = j mod NS) reads x_m =
// a[j + m L/R], scales by w^(m k L/(R NS)), takes the DFT_R and writes
// output q at (j - k) R + k + q NS.  Thread t of a sequence owns the 16/R
// butterflies t + u L/16.  Loads go to registers before the barrier,
// stores after it, so one buffer suffices.
template <int L, int R, int NS, bool INV, bool HIN, bool HOUT, int E, class C>
__device__ __forceinline__ void fft_pass(C* A, int nseq, const C* tws)
{
  constexpr int SL = Len<L>::SL, T = L / E, NB = E / R, Q = L / R;
  // first pass of an input whose upper half is zero: inputs m >= R/2 sit at
  // indices >= L/2 (then NB == 1); last pass of which only the lower half of
  // the output is kept: outputs q >= R/2 land at indices >= L/2
  constexpr bool ZIN = HIN && NS == 1, HALFO = HOUT && NS * R == L;
  const int tid = threadIdx.x;
  const bool act = tid < nseq * T;
  const int sq = act ? tid / T : 0, j = tid - sq * T;
  C* a = A + sq * SL;
  C x[E];
  if (act) {
    const int pj = pad(j);
#pragma unroll
    for (int u = 0; u < NB; u++)
#pragma unroll
      for (int m = 0; m < R; m++)
        x[u * R + m] = (ZIN && m >= R / 2) ? mk<C>(0, 0)
                                           : a[pad_at<T, Q>(pj, j, u, m)];
  }
  __syncthreads();
  if (act) {
#pragma unroll
    for (int u = 0; u < NB; u++) {
      C* xb = x + u * R;
      const int jb = j + u * T, k = jb & (NS - 1);
      if (NS > 1 && k) apply_twiddles<L, E, R, NS, INV>(xb, tws, k);
      dft<R, INV>(xb);
      const int o = (jb - k) * R + k, po = pad(o);
#pragma unroll
      for (int q = 0; q < (HALFO ? R / 2 : R); q++) a[pad_out<NS>(po, o, q)] = xb[out_reg<R>(q)];
    }
  }
  __syncthreads();
}

template <int L, int NS, bool INV, bool HIN, bool HOUT, int E, class C>
__device__ __forceinline__ void fft_passes(C* A, int nseq, const C* tws) {
  if constexpr (NS * E <= L) {
    fft_pass<L, E, NS, INV, HIN, HOUT, E>(A, nseq, tws);
    fft_passes<L, NS * E, INV, HIN, HOUT, E>(A, nseq, tws);
  } else if constexpr (NS < L) {
    fft_pass<L, L / NS, NS, INV, HIN, HOUT, E>(A, nseq, tws);
  }
}

// In-place Stockham autosort FFT of nseq sequences of length L (A + q*SL,
// padded indexing; a power of two >= 16): radix-16 passes and one radix
// 2/4/8 pass for the remaining factor.  Forward exp(-2 pi i jk/L), inverse
// exp(+...), unnormalised.  Needs blockDim.x >= nseq * L/E.  HIN: the
// upper half of the input is zero and never read; HOUT: only the lower half
// of the output is written.
template <int L, bool INV, bool HIN = false, bool HOUT = false, int E = 16, class C>
__device__ void fft_inplace(C* A, int nseq, const C* tws)
{
  fft_passes<L, 1, INV, HIN, HOUT, E>(A, nseq, tws);
}

// sub-transform size NS of the last pass of fft_inplace<L, ..., E>
template <int L, int E> constexpr int last_ns() {
  int ns = 1;
  while (ns * E <= L) ns *= E;
  return ns == L ? ns / E : ns;
}
// the passes of fft_passes<L, NS, ...> whose sub-transform size is below NSEND
template <int L, int NS, int NSEND, bool INV, bool HIN, int E, class C>
__device__ __forceinline__ void fft_passes_below(C* A, int nseq, const C* tws) {
  if constexpr (NS < NSEND) {
    constexpr int R = NS * E <= L ? E : L / NS;
    fft_pass<L, R, NS, INV, HIN, false, E>(A, nseq, tws);
    fft_passes_below<L, NS * R, NSEND, INV, HIN, E>(A, nseq, tws);
  }
}

// Spectral convolution of nseq sequences in place: fft_inplace<L, false,
// HIN>, X[r] = mul(sequence, r, X[r]), fft_inplace<L, true, false, HOUT>.  The
// last forward pass, the multiplier and the first inverse pass run in
// registers: butterfly jb = j + u L/E of the last forward pass (radix R,
// NS = L/R, no stride: k = jb) produces X[jb + q NS] = X[j + (u + (E/R) q)
// L/E], which is input m = u + (E/R) q of thread j's radix-E first inverse
// butterfly (NS = 1).  With L <= E (one pass each way) the three steps run
// one after the other.
template <int L, bool HIN, bool HOUT, int E, class C, class Mul>
__device__ __forceinline__ void fft_convolve(C* A, int nseq, const C* tws, Mul mul)
{
  constexpr int SL = Len<L>::SL, T = L / E, NS = last_ns<L, E>(), R = L / NS, NB = E / R;
  if constexpr (L <= E) {
    fft_inplace<L, false, HIN, false, E>(A, nseq, tws);
    for (int idx = threadIdx.x; idx < nseq * L; idx += blockDim.x) {
      const int sq = idx / L, r = idx - sq * L;
      A[sq * SL + pad(r)] = mul(sq, r, A[sq * SL + pad(r)]);
    }
    __syncthreads();
    fft_inplace<L, true, false, HOUT, E>(A, nseq, tws);
    return;
  }
  fft_passes_below<L, 1, NS, false, HIN, E>(A, nseq, tws);
  const int tid = threadIdx.x;
  const bool act = tid < nseq * T;
  const int sq = act ? tid / T : 0, j = tid - sq * T;
  C* a = A + sq * SL;
  C x[E];
  if (act) {
    const int pj = pad(j);
#pragma unroll
    for (int u = 0; u < NB; u++)
#pragma unroll
      for (int m = 0; m < R; m++) x[u * R + m] = a[pad_at<T, NS>(pj, j, u, m)];
  }
  __syncthreads();
  if (act) {
    C y[E];
#pragma unroll
    for (int u = 0; u < NB; u++) {
      C* xb = x + u * R;
      const int jb = j + u * T;
      if (jb) apply_twiddles<L, E, R, NS, false>(xb, tws, jb);
      dft<R, false>(xb);
#pragma unroll
      for (int q = 0; q < R; q++) y[u + NB * q] = mul(sq, jb + q * NS, xb[out_reg<R>(q)]);
    }
    dft<E, true>(y);
#pragma unroll
    for (int q = 0; q < E; q++) a[pad_out<1>(pad(j * E), j * E, q)] = y[out_reg<E>(q)];
  }
  __syncthreads();
  fft_passes<L, E, true, false, HOUT, E>(A, nseq, tws);
}

// The first pass of a forward FFT (NS = 1, radix R) with its inputs read
// straight from global memory (ld(sequence, index)) into registers: the
// sequence is never staged in shared memory before the pass.  With ZIN the
// upper half of the input is zero and not read.  The outputs go to
// shared memory; the caller's barrier makes them visible.
template <int L, int R, bool ZIN, int E, class C, class Ld>
__device__ __forceinline__ void fft_first_pass_global(C* A, int nseq, Ld ld)
{
  constexpr int SL = Len<L>::SL, T = L / E, NB = E / R, Q = L / R;
  const int tid = threadIdx.x;
  if (tid >= nseq * T) return;
  const int sq = tid / T, j = tid - sq * T;
  C* a = A + sq * SL;
  C x[E];
#pragma unroll
  for (int u = 0; u < NB; u++)
#pragma unroll
    for (int m = 0; m < R; m++)
      x[u * R + m] = (ZIN && m >= R / 2) ? mk<C>(0, 0) : ld(sq, j + u * T + m * Q);
#pragma unroll
  for (int u = 0; u < NB; u++) {
    C* xb = x + u * R;
    dft<R, false>(xb);
    const int o = (j + u * T) * R, po = pad(o);
#pragma unroll
    for (int q = 0; q < R; q++) a[pad_out<1>(po, o, q)] = xb[out_reg<R>(q)];
  }
}

// The last pass of an inverse FFT (NS * R = L) with its outputs written
// straight to global memory (st(sequence, index, value)) from registers;
// with HOUT only the lower half of the output is formed.
template <int L, int R, int NS, bool HOUT, int E, class C, class St>
__device__ __forceinline__ void fft_last_pass_global(C* A, int nseq, const C* tws, St st)
{
  static_assert(NS * R == L, "the last pass");
  constexpr int SL = Len<L>::SL, T = L / E, NB = E / R, Q = L / R;
  const int tid = threadIdx.x;
  if (tid >= nseq * T) return;
  const int sq = tid / T, j = tid - sq * T;
  const C* a = A + sq * SL;
  C x[E];
  const int pj = pad(j);
#pragma unroll
  for (int u = 0; u < NB; u++)
#pragma unroll
    for (int m = 0; m < R; m++) x[u * R + m] = a[pad_at<T, Q>(pj, j, u, m)];
#pragma unroll
  for (int u = 0; u < NB; u++) {
    C* xb = x + u * R;
    const int jb = j + u * T, k = jb & (NS - 1);
    if (NS > 1 && k) apply_twiddles<L, E, R, NS, true>(xb, tws, k);
    dft<R, true>(xb);
    const int o = (jb - k) * R + k;
#pragma unroll
    for (int q = 0; q < (HOUT ? R / 2 : R); q++) st(sq, o + q * NS, xb[out_reg<R>(q)]);
  }
}

struct FadeArgs {
  int enabled;
  Scalars* sc;           // receives fadeCorr (from the first CTA)
  GridDesc g;
  double* writeback;     // rhs buffer receives the faded values (cub2rhs writes tmp)
  const double* partials;   // fade sums of the strip blocks, three each
  int nstrip;
  int bandX, bandY;         // cells of the fade band from each edge, (int)(fadeLen / h) + 2 (host-formed)
};

// fadeCorr for this CTA, formed by warp 0 (blockDim.x >= 32) into *s;
// visible to the CTA after its next barrier
__device__ __forceinline__ void fade_corr_cta(const FadeArgs& fa, double* s) {
  if (threadIdx.x < 32) {
    const double corr = fade_corr(fa.partials, fa.nstrip);
    if (threadIdx.x == 0) {
      *s = corr;
      if (blockIdx.x == 0) fa.sc->fadeCorr = corr;
    }
  }
}

// PoissonSolver::cub2rhs (PoissonSolver.cpp:101-125) for one cell
__device__ __forceinline__ double fade_cell(const GridDesc& g, int gx, int gy, double b, double corr) {
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
  return __dadd_rn(__dmul_rn(b, 1 - f2), fadeCorrection);   // never contracted into an FMA
}

// Real FFT of length 2L from the complex FFT Z of length L of its value
// pairs, even/odd split: X[k] = Fe[k] + W^k Fo[k], W = exp(-i pi / L),
// k in [0, L]; written to row row0 + r of out.  Thread t takes k = t + q NT
// of every row; its twiddles are read first, all in flight at once (read
// inside the loop, every iteration waited for its own).
template <int L, int ER, class C>
__device__ __forceinline__ void r2c_split(const C* A, int nb, int row0, C* __restrict__ out,
                                          int outStride, const C* __restrict__ tw, int twLen)
{
  using R = typename CT<C>::R;
  constexpr int SL = Len<L, ER>::SL, NT = Len<L, ER>::NT, KPT = (L + 1 + NT - 1) / NT;
  constexpr int KB = KPT < 8 ? KPT : 8;                 // twiddles in flight per batch
  const int twStep = twLen / (2 * L);
#pragma unroll
  for (int q0 = 0; q0 < KPT; q0 += KB) {
    C w[KB];
#pragma unroll
    for (int q = 0; q < KB; q++) {
      const int k = threadIdx.x + (q0 + q) * NT;
      w[q] = q0 + q < KPT && k <= L ? tw[k * twStep] : mk<C>(0, 0);
    }
#pragma unroll
    for (int q = 0; q < KB; q++) {
      const int k = threadIdx.x + (q0 + q) * NT;
      if (q0 + q >= KPT || k > L) break;                // k grows with q
      for (int r = 0; r < nb; r++) {
        const C Zk = A[r * SL + pad(k == L ? 0 : k)];
        const C Zc = conjg(A[r * SL + pad(k == 0 ? 0 : L - k)]);
        const C Fe = mk<C>(R(0.5) * (Zk.x + Zc.x), R(0.5) * (Zk.y + Zc.y));
        const C d = csub(Zk, Zc);
        const C Fo = mk<C>(R(0.5) * d.y, R(-0.5) * d.x);  // (Zk - Zc) / (2i)
        out[(size_t)(row0 + r) * outStride + k] = cadd(Fe, cmul(w[q], Fo));
      }
    }
  }
}

// inMode 0: rows of `in`; 1: the free-space Green's function on the MY x MX
// padded grid (FFTW_freespace.cpp:108-119) computed on the fly.  Each row of 2L
// reals is the complex sequence (x[2n], x[2n+1]) of length L.
template <int L, bool HIN, int ER>
__global__ void __launch_bounds__(Len<L, ER>::NT, Len<L, ER>::MINB)
k_rows_r2c(const double* in, int inStride, int nrows, int ncolsIn, int inMode,
           double2* __restrict__ out, int outStride,
           const double2* __restrict__ tw, int twLen, FadeArgs fa, double h, int MX, int MY)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_R2C);
  constexpr int SL = Len<L, ER>::SL, RB = Len<L, ER>::B, NT = Len<L, ER>::NT;
  extern __shared__ double2 sm[];
  double2* A = sm;
  double2* tws = sm + RB * SL;
  const int row0 = blockIdx.x * RB;
  const int nb = min(RB, nrows - row0);
  if (inMode == 0) {
    // the first pass reads the rows itself, fading the band cells as it
    // goes (cub2rhs, PoissonSolver.cpp:61-141) and writing them back
    __shared__ double sCorr0;
    if (fa.enabled) fade_corr_cta(fa, &sCorr0);
    load_twiddles<L, ER>(tws, tw, twLen);
    __syncthreads();
    const double corr = fa.enabled ? sCorr0 : 0.0;
    const int bandX = fa.enabled ? fa.bandX : 0;
    const int bandY = fa.enabled ? fa.bandY : 0;
    auto ld = [&](int r, int n) {
      const int row = row0 + r;
      const double* src = in + (size_t)row * inStride + 2 * n;
      double2 v = make_double2(0, 0);
      if (2 * n + 1 < ncolsIn) v = *reinterpret_cast<const double2*>(src);
      else if (2 * n < ncolsIn) v.x = src[0];
      if (fa.enabled && 2 * n + 1 < ncolsIn) {
        const bool rowBand = row < bandY || row >= fa.g.ny - bandY;
        if (rowBand || 2 * n < bandX || 2 * n + 1 >= fa.g.nx - bandX) {
          double* x = &v.x;
          for (int q = 0; q < 2; q++) {
            const int col = 2 * n + q;
            if (rowBand || col < bandX || col >= fa.g.nx - bandX) {
              x[q] = fade_cell(fa.g, col, row, x[q], corr);
              fa.writeback[(size_t)row * inStride + col] = x[q];
            }
          }
        }
      }
      return v;
    };
    fft_first_pass_global<L, ER, HIN, ER>(A, nb, ld);
    __syncthreads();
    fft_passes<L, ER, false, false, false, ER>(A, nb, tws);
    r2c_split<L, ER>(A, nb, row0, out, outStride, tw, twLen);
    return;
  }
  {
    // inMode 1: the Green's function, formed in place
    for (int idx = threadIdx.x; idx < RB * L; idx += NT) {
      const int r = idx / L, n = idx & (L - 1), row = row0 + r;
      if (r >= nb) continue;
      double x[2];
      for (int q = 0; q < 2; q++) {
        const int col = 2 * n + q;
        double val = 0;
        if (col < ncolsIn) {
          // wrapped offsets: index i stands for offset i below M/2 and for
          // i - M from M/2 on (offsets beyond N - 1 never reach the domain)
          const double fac = 1 / (2 * M_PI);
          if (row == 0 && col == 0) {
            val = fac / 2 * (2 * log(h / sqrt(M_PI)) - 1);
          } else {
            const double yi = row >= MY / 2 ? MY - row : row;
            const double xi = col >= MX / 2 ? MX - col : col;
            const double rr = sqrt(xi * xi + yi * yi);
            val = fac * log(h * rr);
          }
        }
        x[q] = val;
      }
      A[r * SL + pad(n)] = make_double2(x[0], x[1]);
    }
  }
  load_twiddles<L, ER>(tws, tw, twLen);
  __syncthreads();
  fft_inplace<L, false, HIN, false, ER>(A, nb, tws);
  r2c_split<L, ER>(A, nb, row0, out, outStride, tw, twLen);
}

// mode 0: forward, x G^ (real, symmetric in ky), inverse, keep nrowsOut rows
// mode 1: forward; write Re * norm for ky <= L/2 into ghat (kernel set-up)
// mode 2: forward, periodic multiplier -1/|k|^2 / (MX MY), inverse
// Rows r >= nrowsIn of the input are zero and never read.
template <int L, bool FS>
__global__ void __launch_bounds__(Len<L, E_COLS>::NT, Len<L, E_COLS>::MINB)
k_cols(double2* __restrict__ data, int stride, int ncols, int nrowsIn, int nrowsOut,
       const double* __restrict__ ghatIn, double* __restrict__ ghatOut, int mode,
       const double2* __restrict__ tw, int twLen, double norm, int MXp, int MYp)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_COLS);
  constexpr int SL = Len<L, E_COLS>::SL, CB = Len<L, E_COLS>::B, NT = Len<L, E_COLS>::NT, GR = L / 2 + 1;
  extern __shared__ double2 sm[];
  double2* A = sm;
  double2* tws = sm + CB * SL;
  double* Gs = reinterpret_cast<double*>(tws + Len<L>::TW);   // [GR][CB] kernel rows
  const int c0 = blockIdx.x * CB;
  const int nb = min(CB, ncols - c0);
  // consecutive threads take consecutive columns of one row
  for (int idx = threadIdx.x; idx < CB * nrowsIn; idx += NT) {
    const int r = idx / CB, j = idx & (CB - 1);
    if (j < nb) cp_async16(A + j * SL + pad(r), data + (size_t)r * stride + c0 + j);
  }
  cp_async_commit();
  if (mode == 0) {
    for (int idx = threadIdx.x; idx < CB * GR; idx += NT) {
      const int r = idx / CB, j = idx & (CB - 1);
      if (j < nb) cp_async8(Gs + r * CB + j, ghatIn + (size_t)r * stride + c0 + j);
    }
  }
  cp_async_commit();
  // rows beyond the input are zero; the free-space solve never reads its
  // upper half
  for (int idx = threadIdx.x; idx < CB * ((FS ? L / 2 : L) - nrowsIn); idx += NT) {
    const int r = nrowsIn + idx / CB, j = idx & (CB - 1);
    A[j * SL + pad(r)] = make_double2(0, 0);
  }
  load_twiddles<L, E_COLS>(tws, tw, twLen);
  if (mode == 1) {
    cp_async_wait<0>();
    __syncthreads();
    fft_inplace<L, false, FS, false, E_COLS>(A, nb, tws);
    for (int idx = threadIdx.x; idx < CB * nrowsOut; idx += NT) {
      const int r = idx / CB, j = idx & (CB - 1);
      if (j < nb) ghatOut[(size_t)r * stride + c0 + j] = A[j * SL + pad(r)].x * norm;
    }
    return;
  }
  cp_async_wait<0>();          // the columns and the kernel rows
  __syncthreads();
  if (mode == 0) {
    fft_convolve<L, FS, FS, E_COLS>(A, nb, tws, [&](int j, int r, double2 z) {
      const int ky = r <= L / 2 ? r : L - r;
      const double f = Gs[ky * CB + j];
      return make_double2(z.x * f, z.y * f);
    });
  } else {
    fft_convolve<L, FS, FS, E_COLS>(A, nb, tws, [&](int j, int r, double2 z) {
      // FFTW_periodic::_solve_spectral (FFTW_periodic.h:77-92)
      const int i = c0 + j;
      if (i == 0 && r == 0) return make_double2(0, 0);
      const int kx = i <= MXp / 2 ? i : MXp - i, ky = r <= MYp / 2 ? r : MYp - r;
      const double waveFactX = 2 * M_PI / MXp, waveFactY = 2 * M_PI / MYp;
      const double rkx = kx * waveFactX, rky = ky * waveFactY;
      const double f = -1 / (rkx * rkx + rky * rky) * norm;
      return make_double2(z.x * f, z.y * f);
    });
  }
  for (int idx = threadIdx.x; idx < CB * nrowsOut; idx += NT) {
    const int r = idx / CB, j = idx & (CB - 1);
    if (j < nb) data[(size_t)r * stride + c0 + j] = A[j * SL + pad(r)];
  }
}

// inverse real FFT of length 2L from X[0..L]; writes the first ncolsOut values
template <int L, bool HOUT, int EC>
__global__ void __launch_bounds__(Len<L, EC>::NT, Len<L, EC>::MINB)
k_rows_c2r(const double2* __restrict__ in, int inStride, int nrows, double* __restrict__ out,
           int outStride, int ncolsOut, const double2* __restrict__ tw, int twLen)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_C2R);
  constexpr int SL = Len<L, EC>::SL, RB = Len<L, EC>::B, NT = Len<L, EC>::NT, H = L / 2;
  extern __shared__ double2 sm[];
  double2* A = sm;
  double2* tws = sm + RB * SL;
  const int row0 = blockIdx.x * RB;
  const int nb = min(RB, nrows - row0);
  const int twStep = twLen / (2 * L);
  // X[0..L] of each row; X[L] lands in the spare slot pad(L) < SL
  for (int idx = threadIdx.x; idx < RB * (L + 1); idx += NT) {
    const int r = idx / (L + 1), k = idx - r * (L + 1);
    if (r < nb) cp_async16(A + r * SL + pad(k), in + (size_t)(row0 + r) * inStride + k);
  }
  cp_async_commit();
  load_twiddles<L, EC>(tws, tw, twLen);
  // the split's W^-k of the pairs (k, L - k) this thread forms, read while
  // the rows land
  constexpr int KPT = (H + NT - 1) / NT;
  double2 wk[KPT][2];
#pragma unroll
  for (int q = 0; q < KPT; q++) {
    const int k = threadIdx.x + q * NT;
    if (k < H) {
      wk[q][0] = conjg(tw[k * twStep]);
      wk[q][1] = conjg(tw[(k == 0 ? H : L - k) * twStep]);
    }
  }
  cp_async_wait<0>();
  __syncthreads();
  // z[k] = s + i t, s = X_k + conj(X_{L-k}), t = W^-k (X_k - conj(X_{L-k})):
  // thread (k, r), k < L/2, forms the pair k, L-k of every row in place;
  // k = 0 also L/2
#pragma unroll
  for (int q = 0; q < KPT; q++) {
    const int k = threadIdx.x + q * NT;
    if (k >= H) continue;
    const int kk[2] = {k, k == 0 ? H : L - k};
    for (int r = 0; r < nb; r++) {
      double2* a = A + r * SL;
      double2 Xa = a[pad(k)], Xb = a[pad(k == 0 ? L : L - k)];
      if (k == 0) { Xa.y = 0; Xb.y = 0; }         // c2r ignores Im X[0], Im X[L]
      double2 res[2];
#pragma unroll
      for (int e = 0; e < 2; e++) {
        double2 Xk, XL;
        if (e == 0) { Xk = Xa; XL = Xb; }
        else if (k == 0) { Xk = a[pad(H)]; XL = Xk; }
        else { Xk = Xb; XL = Xa; }
        const double2 Xc = conjg(XL);
        const double2 sv = cadd(Xk, Xc), d = csub(Xk, Xc);
        const double2 t = cmul(wk[q][e], d);
        res[e] = make_double2(sv.x - t.y, sv.y + t.x);
      }
      a[pad(kk[0])] = res[0];
      a[pad(kk[1])] = res[1];
    }
  }
  __syncthreads();
  // the inverse FFT; its last pass writes the value pairs of the row
  constexpr int NSL = last_ns<L, EC>();
  fft_passes_below<L, 1, NSL, true, false, EC>(A, nb, tws);
  fft_last_pass_global<L, L / NSL, NSL, HOUT, EC>(A, nb, tws, [&](int r, int n, double2 v) {
    double* o = out + (size_t)(row0 + r) * outStride;
    if (2 * n + 1 < ncolsOut) *reinterpret_cast<double2*>(o + 2 * n) = v;
    else if (2 * n < ncolsOut) o[2 * n] = v.x;
  });
}

// ---- FP32 transforms (CUP2D_PREC_FP32) ------------------------------------
// The free-space and periodic solves with float2 spectra and FP32 passes:
// the same kernels' structure, the fade and its write-back in FP64 (so the
// RHS written back is the one of the FP64 path), rows converted to FP32 as
// they enter shared memory, the pressure written back in FP64.
template <int L, bool HIN>
__global__ void __launch_bounds__(Len<L, E_ROWS32>::NT, Len<L, E_ROWS32>::MINB)
k_rows_r2c32(const double* __restrict__ in, int inStride, int nrows, int ncolsIn,
             float2* __restrict__ out, int outStride, const float2* __restrict__ tw, int twLen, FadeArgs fa)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_R2C);
  constexpr int SL = Len<L, E_ROWS32>::SL, RB = Len<L, E_ROWS32>::B, NT = Len<L, E_ROWS32>::NT;
  constexpr int PER = (RB * L + NT - 1) / NT;          // value pairs per thread
  extern __shared__ float2 sm32[];
  float2* A = sm32;
  float2* tws = sm32 + RB * SL;
  const int row0 = blockIdx.x * RB;
  const int nb = min(RB, nrows - row0);
  double2 v[PER];                                      // this thread's pairs, all loads in flight
#pragma unroll
  for (int u = 0; u < PER; u++) {
    const int idx = threadIdx.x + u * NT;
    const int r = idx / L, n = idx & (L - 1), row = row0 + r;
    v[u] = make_double2(0, 0);
    if (idx < RB * L && r < nb) {
      if (2 * n + 1 < ncolsIn) v[u] = *reinterpret_cast<const double2*>(in + (size_t)row * inStride + 2 * n);
      else if (2 * n < ncolsIn) v[u].x = in[(size_t)row * inStride + 2 * n];
    }
  }
  __shared__ double sCorr;
  if (fa.enabled) fade_corr_cta(fa, &sCorr);
  load_twiddles<L, E_ROWS32>(tws, tw, twLen);
  __syncthreads();
  const double corr = fa.enabled ? sCorr : 0.0;
  const int bandX = fa.enabled ? fa.bandX : 0;
  const int bandY = fa.enabled ? fa.bandY : 0;
#pragma unroll
  for (int u = 0; u < PER; u++) {
    const int idx = threadIdx.x + u * NT;
    const int r = idx / L, n = idx & (L - 1), row = row0 + r;
    if (idx >= RB * L || r >= nb) continue;
    if (HIN && n >= L / 2) continue;                   // the zero upper half is never read
    if (fa.enabled && 2 * n + 1 < ncolsIn) {
      // fade band as in k_rows_r2c (cub2rhs, PoissonSolver.cpp:61-141)
      const bool rowBand = row < bandY || row >= fa.g.ny - bandY;
      double* x = &v[u].x;
      for (int q = 0; q < 2; q++) {
        const int col = 2 * n + q;
        if (rowBand || col < bandX || col >= fa.g.nx - bandX) {
          x[q] = fade_cell(fa.g, col, row, x[q], corr);
          fa.writeback[(size_t)row * inStride + col] = x[q];
        }
      }
    }
    A[r * SL + pad(n)] = make_float2((float)v[u].x, (float)v[u].y);
  }
  __syncthreads();
  fft_inplace<L, false, HIN, false, E_ROWS32>(A, nb, tws);
  r2c_split<L, E_ROWS32>(A, nb, row0, out, outStride, tw, twLen);
}

// mode 0: forward, x G^, inverse, keep nrowsOut rows; mode 2: the periodic
// multiplier -1/|k|^2 / (MX MY) (formed in FP64, applied in FP32)
template <int L, bool FS>
__global__ void __launch_bounds__(Len<L, E_COLS32>::NT, Len<L, E_COLS32>::MINB)
k_cols32(float2* __restrict__ data, int stride, int ncols, int nrowsIn, int nrowsOut,
         const float* __restrict__ ghat, int mode, const float2* __restrict__ tw, int twLen,
         double norm, int MXp, int MYp)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_COLS);
  constexpr int SL = Len<L, E_COLS32>::SL, CB = Len<L, E_COLS32>::B, NT = Len<L, E_COLS32>::NT, GR = L / 2 + 1;
  extern __shared__ float2 sm32[];
  float2* A = sm32;
  float2* tws = sm32 + CB * SL;
  float* Gs = reinterpret_cast<float*>(tws + Len<L>::TW);   // [GR][CB] kernel rows
  const int c0 = blockIdx.x * CB;
  const int nb = min(CB, ncols - c0);
  for (int idx = threadIdx.x; idx < CB * nrowsIn; idx += NT) {
    const int r = idx / CB, j = idx & (CB - 1);
    if (j < nb) cp_async8(A + j * SL + pad(r), data + (size_t)r * stride + c0 + j);
  }
  if (mode == 0)
    for (int idx = threadIdx.x; idx < CB * GR; idx += NT) {
      const int r = idx / CB, j = idx & (CB - 1);
      if (j < nb) cp_async4(Gs + r * CB + j, ghat + (size_t)r * stride + c0 + j);
    }
  cp_async_commit();
  // rows beyond the input are zero; the free-space solve never reads its
  // upper half
  for (int idx = threadIdx.x; idx < CB * ((FS ? L / 2 : L) - nrowsIn); idx += NT) {
    const int r = nrowsIn + idx / CB, j = idx & (CB - 1);
    A[j * SL + pad(r)] = make_float2(0, 0);
  }
  load_twiddles<L, E_COLS32>(tws, tw, twLen);
  cp_async_wait<0>();
  __syncthreads();
  if (mode == 0) {
    fft_convolve<L, FS, FS, E_COLS32>(A, nb, tws, [&](int j, int r, float2 z) {
      const int ky = r <= L / 2 ? r : L - r;
      const float f = Gs[ky * CB + j];
      return make_float2(z.x * f, z.y * f);
    });
  } else {
    fft_convolve<L, FS, FS, E_COLS32>(A, nb, tws, [&](int j, int r, float2 z) {
      // FFTW_periodic::_solve_spectral (FFTW_periodic.h:77-92)
      const int i = c0 + j;
      if (i == 0 && r == 0) return make_float2(0, 0);
      const int kx = i <= MXp / 2 ? i : MXp - i, ky = r <= MYp / 2 ? r : MYp - r;
      const double waveFactX = 2 * M_PI / MXp, waveFactY = 2 * M_PI / MYp;
      const double rkx = kx * waveFactX, rky = ky * waveFactY;
      const float f = (float)(-1 / (rkx * rkx + rky * rky) * norm);
      return make_float2(z.x * f, z.y * f);
    });
  }
  for (int idx = threadIdx.x; idx < CB * nrowsOut; idx += NT) {
    const int r = idx / CB, j = idx & (CB - 1);
    if (j < nb) data[(size_t)r * stride + c0 + j] = A[j * SL + pad(r)];
  }
}

// inverse real FFT of length 2L from X[0..L] (float2); writes the first
// ncolsOut values in FP64
template <int L, bool HOUT>
__global__ void __launch_bounds__(Len<L, E_C2R32>::NT, Len<L, E_C2R32>::MINB)
k_rows_c2r32(const float2* __restrict__ in, int inStride, int nrows, double* __restrict__ out, int outStride,
             int ncolsOut, const float2* __restrict__ tw, int twLen)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_C2R);
  constexpr int SL = Len<L, E_C2R32>::SL, RB = Len<L, E_C2R32>::B, NT = Len<L, E_C2R32>::NT, H = L / 2;
  extern __shared__ float2 sm32[];
  float2* A = sm32;
  float2* tws = sm32 + RB * SL;
  const int row0 = blockIdx.x * RB;
  const int nb = min(RB, nrows - row0);
  const int twStep = twLen / (2 * L);
  for (int idx = threadIdx.x; idx < RB * (L + 1); idx += NT) {
    const int r = idx / (L + 1), k = idx - r * (L + 1);
    if (r < nb) cp_async8(A + r * SL + pad(k), in + (size_t)(row0 + r) * inStride + k);
  }
  cp_async_commit();
  load_twiddles<L, E_C2R32>(tws, tw, twLen);
  // the split's W^-k of the pairs (k, L - k) this thread forms, read while
  // the rows land (as in k_rows_c2r)
  constexpr int KPT = (H + NT - 1) / NT;
  float2 wk[KPT][2];
#pragma unroll
  for (int q = 0; q < KPT; q++) {
    const int k = threadIdx.x + q * NT;
    if (k < H) {
      wk[q][0] = conjg(tw[k * twStep]);
      wk[q][1] = conjg(tw[(k == 0 ? H : L - k) * twStep]);
    }
  }
  cp_async_wait<0>();
  __syncthreads();
#pragma unroll
  for (int q = 0; q < KPT; q++) {
    const int k = threadIdx.x + q * NT;
    if (k >= H) continue;
    const int kk[2] = {k, k == 0 ? H : L - k};
    for (int r = 0; r < nb; r++) {
      float2* a = A + r * SL;
      float2 Xa = a[pad(k)], Xb = a[pad(k == 0 ? L : L - k)];
      if (k == 0) { Xa.y = 0; Xb.y = 0; }
      float2 res[2];
#pragma unroll
      for (int e = 0; e < 2; e++) {
        float2 Xk, XL;
        if (e == 0) { Xk = Xa; XL = Xb; }
        else if (k == 0) { Xk = a[pad(H)]; XL = Xk; }
        else { Xk = Xb; XL = Xa; }
        const float2 Xc = conjg(XL);
        const float2 sv = cadd(Xk, Xc), d = csub(Xk, Xc);
        const float2 t = cmul(wk[q][e], d);
        res[e] = make_float2(sv.x - t.y, sv.y + t.x);
      }
      a[pad(kk[0])] = res[0];
      a[pad(kk[1])] = res[1];
    }
  }
  __syncthreads();
  fft_inplace<L, true, false, HOUT, E_C2R32>(A, nb, tws);
  const int half = (ncolsOut + 1) / 2;
  for (int idx = threadIdx.x; idx < nb * half; idx += NT) {
    const int r = idx / half, n = idx - r * half;
    const float2 v = A[r * SL + pad(n)];
    double* o = out + (size_t)(row0 + r) * outStride;
    if (2 * n + 1 < ncolsOut) *reinterpret_cast<double2*>(o + 2 * n) = make_double2(v.x, v.y);
    else o[2 * n] = v.x;
  }
}

// ---- cosine-transform solver (FFTW_dirichlet.h:30-130) --------------------
// DCT-II (FFTW REDFT10, Y_k = 2 sum x_j cos(pi (j+1/2) k / n)) is the real
// FFT of the even extension y = [x, reversed x] of length 2n:
// Y_k = exp(-i pi k / 2n) FFT_2n(y)_k.  DCT-III (REDFT01,
// x'_m = Y_0 + 2 sum_{k>=1} Y_k cos(pi k (m+1/2) / n)) is the inverse real FFT
// of length 2n of Z_k = exp(+i pi k / 2n) Y_k (Z_n = 0), first n outputs.

// rows: fade on load, DCT-II along x into D (real, Ny x Nx); L = Nx
template <int L>
__global__ void __launch_bounds__(Len<L>::NT, Len<L>::MINB)
k_dct_rows_fwd(const double* in, int Nx, int nrows, double* __restrict__ D, int rb,
               const double2* __restrict__ tw, int twLen, FadeArgs fa)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_DCT_FWD);
  constexpr int SL = Len<L>::SL;
  extern __shared__ double2 sm[];
  double2* A = sm;
  double2* tws = sm + rb * SL;
  double* Bx = reinterpret_cast<double*>(tws + Len<L>::TW);     // staged real row values
  __shared__ double sCorr;
  if (fa.enabled) fade_corr_cta(fa, &sCorr);
  load_twiddles<L, 16>(tws, tw, twLen);
  const int row0 = blockIdx.x * rb;
  const int nb = min(rb, nrows - row0);
  __syncthreads();
  const double corr = fa.enabled ? sCorr : 0.0;
  const int bandX = fa.enabled ? fa.bandX : 0;
  const int bandY = fa.enabled ? fa.bandY : 0;
  // faded row values, then the even extension y[j] = x[j] (j < n), x[2n-1-j]
  for (int idx = threadIdx.x; idx < nb * L; idx += blockDim.x) {
    const int r = idx / L, col = idx - r * L, row = row0 + r;
    double v = in[(size_t)row * Nx + col];
    if (fa.enabled && (row < bandY || row >= fa.g.ny - bandY || col < bandX || col >= fa.g.nx - bandX)) {
      v = fade_cell(fa.g, col, row, v, corr);
      fa.writeback[(size_t)row * Nx + col] = v;
    }
    Bx[r * L + col] = v;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < nb * L; idx += blockDim.x) {
    const int r = idx / L, n = idx - r * L;
    const int j0 = 2 * n, j1 = 2 * n + 1;
    const double y0 = Bx[r * L + (j0 < L ? j0 : 2 * L - 1 - j0)];
    const double y1 = Bx[r * L + (j1 < L ? j1 : 2 * L - 1 - j1)];
    A[r * SL + pad(n)] = make_double2(y0, y1);
  }
  __syncthreads();
  fft_inplace<L, false>(A, nb, tws);
  double2* Z = A;
  const int st2 = twLen / (2 * L), st4 = twLen / (4 * L);
  // four iterations' global loads in flight before the first store
#pragma unroll 4
  for (int idx = threadIdx.x; idx < nb * L; idx += blockDim.x) {
    const int r = idx / L, k = idx - r * L;
    const double2 Zk = Z[r * SL + pad(k)];
    const double2 Zc = conjg(Z[r * SL + pad(k == 0 ? 0 : L - k)]);
    const double2 Fe = make_double2(0.5 * (Zk.x + Zc.x), 0.5 * (Zk.y + Zc.y));
    const double2 d = csub(Zk, Zc);
    const double2 Fo = make_double2(0.5 * d.y, -0.5 * d.x);
    const double2 X = cadd(Fe, cmul(tw[k * st2], Fo));          // FFT_2n(y)_k
    const double2 Y = cmul(tw[k * st4], X);                     // exp(-i pi k/2n) X_k
    D[(size_t)(row0 + r) * Nx + k] = Y.x;
  }
}

// columns, two per complex FFT of length L = 2 Ny: DCT-II along y, the
// multiplier of FFTW_dirichlet::_solve (FFTW_dirichlet.h:49-61), DCT-III.
template <int L>
__global__ void __launch_bounds__(Len<L>::NT, Len<L>::MINB)
k_dct_cols(double* D, int Nx, int Ny, int cb, const float* __restrict__ cosX, const float* __restrict__ cosY,
           double tol, const double2* __restrict__ tw, int twLen)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_DCT_COLS);
  constexpr int SL = Len<L>::SL;
  extern __shared__ double2 sm[];
  double2* A = sm;
  double2* tws = sm + cb * SL;
  load_twiddles<L, 16>(tws, tw, twLen);
  const int n = Ny;                                   // L = 2n
  const int c0 = blockIdx.x * cb * 2;                 // first column of this CTA
  const int np = min(cb, (Nx - c0) / 2);              // column pairs
  for (int idx = threadIdx.x; idx < np * L; idx += blockDim.x) {
    const int j = idx / np, q = idx - j * np;         // j: extended row index
    const int row = j < n ? j : 2 * n - 1 - j;
    const double2 ab = *reinterpret_cast<const double2*>(D + (size_t)row * Nx + c0 + 2 * q);
    A[q * SL + pad(j)] = ab;                          // a + i b
  }
  __syncthreads();
  fft_inplace<L, false>(A, np, tws);
  double2* Z = A;
  // each thread reads the pair (k, L-k) before writing the same pair, and
  // slot n is read by none, so the inverse input overwrites Z in place
  double2* W = Z;
  const int st4 = twLen / (2 * L);                    // exp(-i pi k/2n) = tw[k twLen/(4n)]
  const double MX = Nx, MY = Ny;
  const double waveFactX = M_PI / MX, waveFactY = M_PI / MY;
  const double norm_factor = 0.25 / (MX * MY);
  // separate the two real columns, DCT-II values, multiplier, then the
  // Hermitian spectra of both DCT-III inputs packed as Za + i Zb
#pragma unroll 4
  for (int idx = threadIdx.x; idx < np * n; idx += blockDim.x) {
    const int q = idx / n, k = idx - q * n;
    const double2 Zk = Z[q * SL + pad(k)];
    const double2 Zc = conjg(Z[q * SL + pad(k == 0 ? 0 : L - k)]);
    const double2 Ak = make_double2(0.5 * (Zk.x + Zc.x), 0.5 * (Zk.y + Zc.y));     // FFT of a
    const double2 dd = csub(Zk, Zc);
    const double2 Bk = make_double2(0.5 * dd.y, -0.5 * dd.x);                      // FFT of b
    const double2 w = tw[k * st4];
    double ya = cmul(w, Ak).x, yb = cmul(w, Bk).x;                                 // DCT-II
    for (int e = 0; e < 2; e++) {
      const int i = c0 + 2 * q + e, jj = k;
      const double rkx = (i + 0.5) * waveFactX, rky = (jj + 0.5) * waveFactY;
      const float denomF = 1 - cosX[i] / 2 - cosY[jj] / 2;                         // float, as written
      const double denomFD = denomF;
      const double denomSP = rkx * rkx + rky * rky;
      double& y = e == 0 ? ya : yb;
      y *= -norm_factor / ((1 - tol) * denomFD + tol * denomSP);
      if (i == 0 && jj == 0) y = 0;                                                // in_out[0] = 0
    }
    // Z_k = exp(+i pi k/2n) Y_k for both columns, packed
    const double2 wc = conjg(w);
    const double2 za = make_double2(wc.x * ya, wc.y * ya), zb = make_double2(wc.x * yb, wc.y * yb);
    W[q * SL + pad(k)] = make_double2(za.x - zb.y, za.y + zb.x);                     // za + i zb
    if (k > 0) {   // k' = 2n - k: conj(za) + i conj(zb)
      W[q * SL + pad(L - k)] = make_double2(za.x + zb.y, -za.y + zb.x);
    }
  }
  for (int q = threadIdx.x; q < np; q += blockDim.x) W[q * SL + pad(n)] = make_double2(0, 0);
  __syncthreads();
  fft_inplace<L, true, false, true>(W, np, tws);          // outputs m < n = L/2
  double2* Y = W;
#pragma unroll 4
  for (int idx = threadIdx.x; idx < np * n; idx += blockDim.x) {
    const int m = idx / np, q = idx - m * np;
    *reinterpret_cast<double2*>(D + (size_t)m * Nx + c0 + 2 * q) = Y[q * SL + pad(m)];
  }
}

// rows: DCT-III along x from D into p; L = Nx
template <int L>
__global__ void __launch_bounds__(Len<L>::NT, Len<L>::MINB)
k_dct_rows_inv(const double* __restrict__ D, int Nx, int nrows, double* __restrict__ out, int rb,
               const double2* __restrict__ tw, int twLen)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_DCT_INV);
  constexpr int SL = Len<L>::SL;
  extern __shared__ double2 sm[];
  double2* A = sm;
  double2* tws = sm + rb * SL;
  load_twiddles<L, 16>(tws, tw, twLen);
  const int row0 = blockIdx.x * rb;
  const int nb = min(rb, nrows - row0);
  const int st2 = twLen / (2 * L), st4 = twLen / (4 * L);
  // four iterations' global loads in flight before the first store
#pragma unroll 4
  for (int idx = threadIdx.x; idx < nb * L; idx += blockDim.x) {
    const int r = idx / L, k = idx - r * L;
    const double* Yr = D + (size_t)(row0 + r) * Nx;
    // X_k = exp(i pi k/2n) Y_k, X_n = 0; then the c2r combination of k_rows_c2r
    const double2 wk = conjg(tw[k * st4]);
    double2 Xk = make_double2(wk.x * Yr[k], wk.y * Yr[k]);
    double2 XL = make_double2(0, 0);
    if (k > 0) { const double2 wl = conjg(tw[(L - k) * st4]); XL = make_double2(wl.x * Yr[L - k], wl.y * Yr[L - k]); }
    if (k == 0) { Xk.y = 0; XL.y = 0; }
    const double2 Xc = conjg(XL);
    const double2 s = cadd(Xk, Xc), d = csub(Xk, Xc);
    const double2 t = cmul(conjg(tw[k * st2]), d);
    A[r * SL + pad(k)] = make_double2(s.x - t.y, s.y + t.x);
  }
  __syncthreads();
  fft_inplace<L, true, false, true>(A, nb, tws);          // outputs m < L/2
  double2* z = A;
  for (int idx = threadIdx.x; idx < nb * (L / 2); idx += blockDim.x) {
    const int r = idx / (L / 2), m = idx - r * (L / 2);
    *reinterpret_cast<double2*>(out + (size_t)(row0 + r) * Nx + 2 * m) = z[r * SL + pad(m)];
  }
}

inline bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

bool g_smemOk = true;
void set_smem(const void* f) { if (allow_max_dynamic_smem(f) != cudaSuccess) g_smemOk = false; }

// B padded sequences, the staged twiddles, and extraReals doubles
template <int L> inline size_t smem_for(size_t extraReals = 0) {
  return sizeof(double2) * ((size_t)Len<L>::B * Len<L>::SL + Len<L>::TW) + sizeof(double) * extraReals;
}

template <int L> inline size_t smem_for32(size_t extraReals = 0) {
  return sizeof(float2) * ((size_t)Len<L>::B * Len<L>::SL + Len<L>::TW) + sizeof(float) * extraReals;
}

#define CUP2D_FFT_LENGTHS(X) X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048) X(4096)

void set_all_smem() {
#define X(L) set_smem((const void*)k_rows_r2c<L, false, 8>); set_smem((const void*)k_rows_r2c<L, true, 8>); \
             set_smem((const void*)k_rows_r2c<L, false, 16>); set_smem((const void*)k_rows_r2c<L, true, 16>); \
             set_smem((const void*)k_rows_c2r<L, false, 8>); set_smem((const void*)k_rows_c2r<L, true, 8>); \
             set_smem((const void*)k_rows_c2r<L, false, 16>); set_smem((const void*)k_rows_c2r<L, true, 16>); \
             set_smem((const void*)k_cols<L, false>); set_smem((const void*)k_cols<L, true>); \
             set_smem((const void*)k_dct_rows_fwd<L>); \
             set_smem((const void*)k_dct_cols<L>); set_smem((const void*)k_dct_rows_inv<L>); \
             set_smem((const void*)k_rows_r2c32<L, false>); set_smem((const void*)k_rows_r2c32<L, true>); \
             set_smem((const void*)k_rows_c2r32<L, false>); set_smem((const void*)k_rows_c2r32<L, true>); \
             set_smem((const void*)k_cols32<L, false>); set_smem((const void*)k_cols32<L, true>);
  CUP2D_FFT_LENGTHS(X)
#undef X
}

template <int LL, int ER>
void rows_r2c_e(cudaStream_t st, const double* in, int inStride, int nrows, int ncolsIn, int inMode,
                double2* out, int outStride, const double2* tw, int twLen, FadeArgs fa, double h, int MX, int MY,
                bool halfIn) {
  const int grid = (nrows + Len<LL>::B - 1) / Len<LL>::B;
  if (halfIn) launch_k(k_rows_r2c<LL, true, ER>, grid, Len<LL, ER>::NT, smem_for<LL>(), st,
                       in, inStride, nrows, ncolsIn, inMode, out, outStride, tw, twLen, fa, h, MX, MY);
  else launch_k(k_rows_r2c<LL, false, ER>, grid, Len<LL, ER>::NT, smem_for<LL>(), st,
                in, inStride, nrows, ncolsIn, inMode, out, outStride, tw, twLen, fa, h, MX, MY);
}

// e: elements per thread (8 or 16)
bool rows_r2c(int L, cudaStream_t st, const double* in, int inStride, int nrows, int ncolsIn, int inMode,
              double2* out, int outStride, const double2* tw, int twLen, FadeArgs fa, double h, int MX, int MY,
              bool halfIn, int e) {
  switch (L) {
#define X(LL) case LL: \
    if (e == 16) rows_r2c_e<LL, 16>(st, in, inStride, nrows, ncolsIn, inMode, out, outStride, tw, twLen, fa, h, \
                                    MX, MY, halfIn); \
    else rows_r2c_e<LL, 8>(st, in, inStride, nrows, ncolsIn, inMode, out, outStride, tw, twLen, fa, h, MX, MY, \
                           halfIn); \
    return true;
    CUP2D_FFT_LENGTHS(X)
#undef X
  }
  return false;
}

bool cols(int L, cudaStream_t st, double2* data, int stride, int ncols, int nrowsIn, int nrowsOut,
          double* ghat, int mode, const double2* tw, int twLen, double norm, int MXp, int MYp) {
  switch (L) {
#define X(LL) case LL: \
    if (mode == 0) launch_k(k_cols<LL, true>, (ncols + Len<LL>::B - 1) / Len<LL>::B, Len<LL, E_COLS>::NT, \
        smem_for<LL>((size_t)(LL / 2 + 1) * Len<LL>::B), st, data, stride, ncols, nrowsIn, \
        nrowsOut, ghat, ghat, mode, tw, twLen, norm, MXp, MYp); \
    else launch_k(k_cols<LL, false>, (ncols + Len<LL>::B - 1) / Len<LL>::B, Len<LL, E_COLS>::NT, \
        smem_for<LL>((size_t)(LL / 2 + 1) * Len<LL>::B), st, data, stride, ncols, nrowsIn, \
        nrowsOut, ghat, ghat, mode, tw, twLen, norm, MXp, MYp); \
    return true;
    CUP2D_FFT_LENGTHS(X)
#undef X
  }
  return false;
}

template <int LL, int EC>
void rows_c2r_e(cudaStream_t st, const double2* in, int inStride, int nrows, double* out, int outStride,
                int ncolsOut, const double2* tw, int twLen, bool halfOut) {
  const int grid = (nrows + Len<LL>::B - 1) / Len<LL>::B;
  if (halfOut) launch_k(k_rows_c2r<LL, true, EC>, grid, Len<LL, EC>::NT, smem_for<LL>(), st,
                        in, inStride, nrows, out, outStride, ncolsOut, tw, twLen);
  else launch_k(k_rows_c2r<LL, false, EC>, grid, Len<LL, EC>::NT, smem_for<LL>(), st,
                in, inStride, nrows, out, outStride, ncolsOut, tw, twLen);
}

// e: elements per thread (8 or 16)
bool rows_c2r(int L, cudaStream_t st, const double2* in, int inStride, int nrows, double* out, int outStride,
              int ncolsOut, const double2* tw, int twLen, bool halfOut, int e) {
  switch (L) {
#define X(LL) case LL: \
    if (e == 8) rows_c2r_e<LL, 8>(st, in, inStride, nrows, out, outStride, ncolsOut, tw, twLen, halfOut); \
    else rows_c2r_e<LL, 16>(st, in, inStride, nrows, out, outStride, ncolsOut, tw, twLen, halfOut); \
    return true;
    CUP2D_FFT_LENGTHS(X)
#undef X
  }
  return false;
}

bool rows_r2c32(int L, cudaStream_t st, const double* in, int inStride, int nrows, int ncolsIn,
                float2* out, int outStride, const float2* tw, int twLen, FadeArgs fa, bool halfIn) {
  switch (L) {
#define X(LL) case LL: \
    if (halfIn) launch_k(k_rows_r2c32<LL, true>, (nrows + Len<LL>::B - 1) / Len<LL>::B, Len<LL, E_ROWS32>::NT, \
        smem_for32<LL>(), st, in, inStride, nrows, ncolsIn, out, outStride, tw, twLen, fa); \
    else launch_k(k_rows_r2c32<LL, false>, (nrows + Len<LL>::B - 1) / Len<LL>::B, Len<LL, E_ROWS32>::NT, \
        smem_for32<LL>(), st, in, inStride, nrows, ncolsIn, out, outStride, tw, twLen, fa); \
    return true;
    CUP2D_FFT_LENGTHS(X)
#undef X
  }
  return false;
}

bool cols32(int L, cudaStream_t st, float2* data, int stride, int ncols, int nrowsIn, int nrowsOut,
            const float* ghat, int mode, const float2* tw, int twLen, double norm, int MXp, int MYp) {
  switch (L) {
#define X(LL) case LL: \
    if (mode == 0) launch_k(k_cols32<LL, true>, (ncols + Len<LL>::B - 1) / Len<LL>::B, Len<LL, E_COLS32>::NT, \
        smem_for32<LL>((size_t)(LL / 2 + 1) * Len<LL>::B), st, data, stride, ncols, nrowsIn, nrowsOut, \
        ghat, mode, tw, twLen, norm, MXp, MYp); \
    else launch_k(k_cols32<LL, false>, (ncols + Len<LL>::B - 1) / Len<LL>::B, Len<LL, E_COLS32>::NT, \
        smem_for32<LL>((size_t)(LL / 2 + 1) * Len<LL>::B), st, data, stride, ncols, nrowsIn, nrowsOut, \
        ghat, mode, tw, twLen, norm, MXp, MYp); \
    return true;
    CUP2D_FFT_LENGTHS(X)
#undef X
  }
  return false;
}

bool rows_c2r32(int L, cudaStream_t st, const float2* in, int inStride, int nrows, double* out, int outStride,
                int ncolsOut, const float2* tw, int twLen, bool halfOut) {
  switch (L) {
#define X(LL) case LL: \
    if (halfOut) launch_k(k_rows_c2r32<LL, true>, (nrows + Len<LL>::B - 1) / Len<LL>::B, Len<LL, E_C2R32>::NT, \
        smem_for32<LL>(), st, in, inStride, nrows, out, outStride, ncolsOut, tw, twLen); \
    else launch_k(k_rows_c2r32<LL, false>, (nrows + Len<LL>::B - 1) / Len<LL>::B, Len<LL, E_C2R32>::NT, \
        smem_for32<LL>(), st, in, inStride, nrows, out, outStride, ncolsOut, tw, twLen); \
    return true;
    CUP2D_FFT_LENGTHS(X)
#undef X
  }
  return false;
}

bool dct_rows_fwd(int L, cudaStream_t st, const double* in, int Nx, int nrows, double* D,
                  const double2* tw, int twLen, FadeArgs fa) {
  switch (L) {
#define X(LL) case LL: launch_k(k_dct_rows_fwd<LL>, (nrows + Len<LL>::B - 1) / Len<LL>::B, Len<LL>::NT, \
                  smem_for<LL>((size_t)Len<LL>::B * LL), st, in, Nx, nrows, D, Len<LL>::B, tw, twLen, fa); return true;
    CUP2D_FFT_LENGTHS(X)
#undef X
  }
  return false;
}

bool dct_cols(int L, cudaStream_t st, double* D, int Nx, int Ny, const float* cx, const float* cy, double tol,
              const double2* tw, int twLen) {
  const int pairs = Nx / 2;
  switch (L) {
#define X(LL) case LL: launch_k(k_dct_cols<LL>, (pairs + Len<LL>::B - 1) / Len<LL>::B, Len<LL>::NT, smem_for<LL>(), st,  \
                  D, Nx, Ny, Len<LL>::B, cx, cy, tol, tw, twLen); return true;
    CUP2D_FFT_LENGTHS(X)
#undef X
  }
  return false;
}

bool dct_rows_inv(int L, cudaStream_t st, const double* D, int Nx, int nrows, double* out,
                  const double2* tw, int twLen) {
  switch (L) {
#define X(LL) case LL: launch_k(k_dct_rows_inv<LL>, (nrows + Len<LL>::B - 1) / Len<LL>::B, Len<LL>::NT, smem_for<LL>(), st,  \
                  D, Nx, nrows, out, Len<LL>::B, tw, twLen); return true;
    CUP2D_FFT_LENGTHS(X)
#undef X
  }
  return false;
}

} // namespace

namespace {
inline int pow2_at_least(int n) { int p = 1; while (p < n) p <<= 1; return p; }
}

// The transforms are radix-16 Stockham FFTs of power-of-two lengths 16 ..
// 4096 held in shared memory.  Free space pads to powers of two, so any
// grid with Nx <= 4096 and Ny <= 2048 works; the periodic and cosine
// solvers transform the grid's own lengths, which must be powers of two.
bool poisson_size_ok(int type, int nx, int ny) {
  if (type == CUP2D_POISSON_FREESPACE) {
    const int lrow = pow2_at_least(2 * nx) / 2, lcol = pow2_at_least(2 * ny);
    return lrow >= 16 && lcol >= 16 && lrow <= 4096 && lcol <= 4096;
  }
  if (!is_pow2(nx) || !is_pow2(ny)) return false;
  const int lrow = type == CUP2D_POISSON_PERIODIC ? nx / 2 : nx;
  const int lcol = type == CUP2D_POISSON_PERIODIC ? ny : 2 * ny;
  return lrow >= 16 && lcol >= 16 && lrow <= 4096 && lcol <= 4096;
}

const char* poisson_size_limits(int type) {
  if (type == CUP2D_POISSON_FREESPACE)
    return "grid beyond the free-space solver's transforms: Nx = 32 bpdx <= 4096 and Ny = 32 bpdy <= 2048";
  if (type == CUP2D_POISSON_PERIODIC)
    return "grid beyond the periodic solver's transforms: Nx and Ny powers of two, Nx <= 8192, Ny <= 4096";
  return "grid beyond the cosine solver's transforms: Nx and Ny powers of two, Nx <= 4096, Ny <= 2048";
}

Poisson* poisson_create(Ctx& c) {
  Poisson* P = new Poisson();
  P->type = c.cfg.poisson;
  const int Nx = c.g.nx, Ny = c.g.ny;
  if (P->type == CUP2D_POISSON_FREESPACE) {
    // the padded grid: any size >= 2N - 1 gives the same linear convolution
    // on the domain (FFTW_freespace.cpp pads to 2N - 1); powers of two >= 2N
    // keep every transform a radix-16 Stockham FFT in shared memory
    P->MX = 2 * Nx; P->MY = 2 * Ny;
    while (!is_pow2(P->MX)) P->MX++;
    while (!is_pow2(P->MY)) P->MY++;
    P->Lrow = P->MX / 2;   // real length MX
    P->Lcol = P->MY;
  } else if (P->type == CUP2D_POISSON_PERIODIC) {
    P->Lrow = Nx / 2;      // real length Nx
    P->Lcol = Ny;
  } else {
    P->Lrow = Nx;          // DCT of length Nx via a real FFT of length 2Nx
    P->Lcol = 2 * Ny;      // DCT of length Ny via a complex FFT of length 2Ny
  }
  // the built-in choice, measured on B200 (forward rows of 4096 points: 115
  // us with 16 elements per thread against 127 with 8; 1024 points: 17 us
  // with 8 against 21; the inverse pass: 16 at both)
  P->eR2C = P->Lrow >= 4096 ? 16 : 8;
  P->eC2R = 16;
  if (!is_pow2(P->Lrow) || !is_pow2(P->Lcol) || P->Lrow < 16 || P->Lcol < 16 ||
      P->Lrow > 4096 || P->Lcol > 4096) { delete P; return nullptr; }   // shared-memory limit
  P->nkx = P->Lrow + 1;
  P->twLen = 4 * (P->Lrow > P->Lcol ? P->Lrow : P->Lcol);
  std::vector<double2> tw(P->twLen);
  for (int k = 0; k < P->twLen; k++) {
    const long double a = -2.0L * 3.14159265358979323846264338327950288L * k / P->twLen;
    tw[k] = make_double2((double)cosl(a), (double)sinl(a));
  }
  if (cudaMalloc(&P->tw, sizeof(double2) * P->twLen) != cudaSuccess) { delete P; return nullptr; }
  h2d_sync(P->tw, tw.data(), sizeof(double2) * P->twLen, c.stream);
  const size_t specRows = (size_t)P->Lcol;
  if (cudaMalloc(&P->spec, sizeof(double2) * specRows * P->nkx) != cudaSuccess) { poisson_destroy(P); return nullptr; }
  set_all_smem();
  if (!g_smemOk) { poisson_destroy(P); return nullptr; }
  if (P->type == CUP2D_POISSON_COSINE) {
    // FFTW_dirichlet constructor (FFTW_dirichlet.h:74-76): cosines stored as float
    std::vector<float> cx(Nx), cy(Ny);
    for (int j = 0; j < Ny; j++) cy[j] = (float)std::cos(M_PI / Ny * 2.0 * j);
    for (int i = 0; i < Nx; i++) cx[i] = (float)std::cos(M_PI / Nx * 2.0 * i);
    if (cudaMalloc(&P->cosX, sizeof(float) * Nx) != cudaSuccess ||
        cudaMalloc(&P->cosY, sizeof(float) * Ny) != cudaSuccess) { poisson_destroy(P); return nullptr; }
    h2d_sync(P->cosX, cx.data(), sizeof(float) * Nx, c.stream);
    h2d_sync(P->cosY, cy.data(), sizeof(float) * Ny, c.stream);
  }
  if (P->type == CUP2D_POISSON_FREESPACE) {
    // G^ = Re FFT[G] / (MX MY) on the MY x MX padded grid, kept for ky <= MY/2
    if (cudaMalloc(&P->ghat, sizeof(double) * (P->Lcol / 2 + 1) * P->nkx) != cudaSuccess) { poisson_destroy(P); return nullptr; }
    FadeArgs fa{}; fa.enabled = 0;
    // (always with 8 elements per thread: G^ does not depend on the tuning)
    rows_r2c(P->Lrow, c.stream, nullptr, 0, P->MY, P->MX, 1, P->spec, P->nkx, P->tw, P->twLen, fa, c.g.h,
             P->MX, P->MY, false, 8);
    CUP2D_LAUNCHED(c);
    const double norm = 1.0 / ((double)P->MX * (double)P->MY);
    cols(P->Lcol, c.stream, P->spec, P->nkx, P->nkx, P->MY, P->Lcol / 2 + 1, P->ghat, 1, P->tw, P->twLen, norm, 0, 0);
    CUP2D_LAUNCHED(c);
  }
  if (c.cfg.precision == CUP2D_PREC_FP32) {
    // the FP32 solve: twiddles and G^ formed in FP64 as above, then rounded
    P->fp32 = true;
    std::vector<float2> tw32(P->twLen);
    for (int k = 0; k < P->twLen; k++) tw32[k] = make_float2((float)tw[k].x, (float)tw[k].y);
    if (cudaMalloc(&P->tw32, sizeof(float2) * P->twLen) != cudaSuccess) { poisson_destroy(P); return nullptr; }
    h2d_sync(P->tw32, tw32.data(), sizeof(float2) * P->twLen, c.stream);
    if (P->type == CUP2D_POISSON_FREESPACE) {
      const size_t ng = (size_t)(P->Lcol / 2 + 1) * P->nkx;
      std::vector<double> g64(ng);
      std::vector<float> g32(ng);
      if (cudaStreamSynchronize(c.stream) != cudaSuccess ||
          cudaMemcpy(g64.data(), P->ghat, sizeof(double) * ng, cudaMemcpyDeviceToHost) != cudaSuccess ||
          cudaMalloc(&P->ghat32, sizeof(float) * ng) != cudaSuccess) { poisson_destroy(P); return nullptr; }
      for (size_t i = 0; i < ng; i++) g32[i] = (float)g64[i];
      h2d_sync(P->ghat32, g32.data(), sizeof(float) * ng, c.stream);
    }
  }
  return P;
}

void poisson_destroy(Poisson* P) {
  if (!P) return;
  cudaFree(P->spec); cudaFree(P->ghat); cudaFree(P->tw); cudaFree(P->cosX); cudaFree(P->cosY);
  cudaFree(P->tw32); cudaFree(P->ghat32);
  delete P;
}

// PoissonSolver::solve: cub2rhs (the fade; every CTA of the first row pass
// forms fadeCorr from the strip blocks' sums that the RHS kernels left), the
// transform passes, sol2cub (the inverse row pass writes pres directly).
void poisson_rows_fwd(Ctx& c) {
  Poisson* P = c.poisson;
  const int Nx = c.g.nx, Ny = c.g.ny;
  FadeArgs fa{c.solveNoFade ? 0 : 1, c.dsc, c.g, c.rhs, fade_partials(c), c.nfade,
              (int)(c.g.fadeLenX / c.g.h) + 2, (int)(c.g.fadeLenY / c.g.h) + 2};
  if (P->type == CUP2D_POISSON_COSINE) {
    dct_rows_fwd(P->Lrow, c.stream, c.rhs, Nx, Ny, reinterpret_cast<double*>(P->spec), P->tw, P->twLen, fa);
    CUP2D_LAUNCHED(c);
    return;
  }
  // free space: the row's zero padding is the upper half of the length-Lrow sequence
  if (P->fp32)
    rows_r2c32(P->Lrow, c.stream, c.rhs, Nx, Ny, Nx, reinterpret_cast<float2*>(P->spec), P->nkx, P->tw32,
               P->twLen, fa, P->type == CUP2D_POISSON_FREESPACE);
  else
    rows_r2c(P->Lrow, c.stream, c.rhs, Nx, Ny, Nx, 0, P->spec, P->nkx, P->tw, P->twLen, fa, c.g.h, P->MX, P->MY,
             P->type == CUP2D_POISSON_FREESPACE, P->eR2C);
  CUP2D_LAUNCHED(c);
}

void poisson_cols(Ctx& c) {
  Poisson* P = c.poisson;
  const int Nx = c.g.nx, Ny = c.g.ny;
  if (P->type == CUP2D_POISSON_COSINE) {
    dct_cols(P->Lcol, c.stream, reinterpret_cast<double*>(P->spec), Nx, Ny, P->cosX, P->cosY, P->tol, P->tw, P->twLen);
  } else if (P->type == CUP2D_POISSON_FREESPACE) {
    if (P->fp32)
      cols32(P->Lcol, c.stream, reinterpret_cast<float2*>(P->spec), P->nkx, P->nkx, Ny, Ny, P->ghat32, 0,
             P->tw32, P->twLen, 0.0, 0, 0);
    else
      cols(P->Lcol, c.stream, P->spec, P->nkx, P->nkx, Ny, Ny, P->ghat, 0, P->tw, P->twLen, 0.0, 0, 0);
  } else {
    const double norm = 1.0 / ((double)Nx * (double)Ny);
    if (P->fp32)
      cols32(P->Lcol, c.stream, reinterpret_cast<float2*>(P->spec), P->nkx, P->nkx, Ny, Ny, nullptr, 2,
             P->tw32, P->twLen, norm, Nx, Ny);
    else
      cols(P->Lcol, c.stream, P->spec, P->nkx, P->nkx, Ny, Ny, nullptr, 2, P->tw, P->twLen, norm, Nx, Ny);
  }
  CUP2D_LAUNCHED(c);
}

void poisson_rows_inv(Ctx& c) {
  Poisson* P = c.poisson;
  const int Nx = c.g.nx, Ny = c.g.ny;
  if (P->type == CUP2D_POISSON_COSINE) {
    dct_rows_inv(P->Lrow, c.stream, reinterpret_cast<const double*>(P->spec), Nx, Ny, c.pres, P->tw, P->twLen);
    CUP2D_LAUNCHED(c);
    return;
  }
  if (P->fp32)
    rows_c2r32(P->Lrow, c.stream, reinterpret_cast<const float2*>(P->spec), P->nkx, Ny, c.pres, Nx, Nx,
               P->tw32, P->twLen, P->type == CUP2D_POISSON_FREESPACE);
  else
    rows_c2r(P->Lrow, c.stream, P->spec, P->nkx, Ny, c.pres, Nx, Nx, P->tw, P->twLen,
             P->type == CUP2D_POISSON_FREESPACE, P->eC2R);        // free space keeps the first half
  CUP2D_LAUNCHED(c);
}

namespace {
// choices already made in this process, per transform set-up: every context
// of a grid takes the same variants (so their results agree bitwise)
using TuneKey = std::tuple<int, int, int, int, int>;   // solver, Lrow, Lcol, Nx, Ny
std::mutex g_tuneMu;
std::map<TuneKey, std::array<int, 2>> g_tuned;

// median device time (us) of 5 launches after one warm-up, CUDA events on st
template <class F> double median_us(cudaStream_t st, F launch) {
  cudaEvent_t a, b;
  if (cudaEventCreate(&a) != cudaSuccess) return -1;
  if (cudaEventCreate(&b) != cudaSuccess) { cudaEventDestroy(a); return -1; }
  launch();
  std::array<float, 5> t{};
  for (float& x : t) {
    cudaEventRecord(a, st);
    launch();
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&x, a, b);
  }
  cudaEventDestroy(a); cudaEventDestroy(b);
  std::sort(t.begin(), t.end());
  return 1e3 * t[2];
}
} // namespace

// The project autotuner: for the FP64 free-space and periodic solves, times
// the forward and the inverse row pass with 8 and with 16 elements per
// thread on this grid (the context's own RHS and pressure buffers, fade
// off: run at set-up, before the fields hold state) and keeps the faster of
// each.  A grid tuned before in this process reuses that choice.
cudaError_t poisson_autotune(Ctx& c) {
  Poisson* P = c.poisson;
  if (P->type == CUP2D_POISSON_COSINE || P->fp32) return cudaSuccess;
  const TuneKey key{P->type, P->Lrow, P->Lcol, c.g.nx, c.g.ny};
  std::lock_guard<std::mutex> lock(g_tuneMu);
  auto it = g_tuned.find(key);
  if (it != g_tuned.end()) {
    P->eR2C = it->second[0]; P->eC2R = it->second[1];
    P->tuned = true;
    return cudaSuccess;
  }
  const int Nx = c.g.nx, Ny = c.g.ny;
  const bool fs = P->type == CUP2D_POISSON_FREESPACE;
  FadeArgs fa{}; fa.enabled = 0;
  for (int q = 0; q < 2; q++) {
    const int e = q ? 16 : 8;
    P->tuneUs[q] = median_us(c.stream, [&] {
      rows_r2c(P->Lrow, c.stream, c.rhs, Nx, Ny, Nx, 0, P->spec, P->nkx, P->tw, P->twLen, fa, c.g.h, P->MX,
               P->MY, fs, e);
    });
    P->tuneUs[2 + q] = median_us(c.stream, [&] {
      rows_c2r(P->Lrow, c.stream, P->spec, P->nkx, Ny, c.pres, Nx, Nx, P->tw, P->twLen, fs, e);
    });
  }
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  for (double t : P->tuneUs) if (!(t > 0)) return cudaErrorUnknown;
  P->eR2C = P->tuneUs[1] < P->tuneUs[0] ? 16 : 8;
  P->eC2R = P->tuneUs[3] < P->tuneUs[2] ? 16 : 8;
  P->tuned = true;
  g_tuned[key] = {P->eR2C, P->eC2R};
  return cudaSuccess;
}

void poisson_tuning(const Ctx& c, cup2d_tuning* out) {
  const Poisson* P = c.poisson;
  out->fft_rows_fwd_e = P->eR2C;
  out->fft_rows_inv_e = P->eC2R;
  out->tuned = P->tuned ? 1 : 0;
  for (int q = 0; q < 4; q++) out->us[q] = P->tuneUs[q];
}

void poisson_solve(Ctx& c) {
  poisson_rows_fwd(c);
  poisson_cols(c);
  poisson_rows_inv(c);
}

} // namespace cup2d

#ifdef CUP2D_TRACE
namespace cup2d { void trace_bind_poisson(unsigned long long* p) { trace_bind_this_unit(p); } }
#endif
