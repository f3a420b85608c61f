// Internal device-side data model of the B200 pipeline.
//
// Layout (all in HBM, one context = one grid):
//  - dense fields are row-major planes of Ny x Nx values (x fastest), one
//    plane per component (SoA): u, v, chi, pres, rhs (the reference's "tmp"
//    during PressureSingle), sdf (the reference's "tmp" during
//    PutObjectsOnGrid).  Nx = 32*bpdx is a multiple of 32, so every row is a
//    whole number of 256-byte (fp64) segments and every 32x32 reference block
//    is the tile at (32*bx, 32*by).
//  - obstacle data is sparse: per shape, a list of touched 32x32 tiles (the
//    reference's obstacleBlocks[blockID] != nullptr, Shape.h:20) with a dense
//    32x32 payload per tile (ObstacleBlock.h:25-31): chi, dist, udef and the
//    surface delta/normal of putChiOnGrid.
//  - scalars (time, dt, u_inf, ...) and rigid-body state live in device
//    memory so a whole timestep needs no host round trip.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "../../include/cup2d.h"

namespace cup2d {

constexpr int BS = 32;            // _BS_ of the reference (Definitions.h:30-32)
constexpr int BS2 = BS * BS;
constexpr double EPSd = 2.220446049250313e-16;   // std::numeric_limits<double>::epsilon()
constexpr int MAX_SHAPES = 8;
constexpr int NFORCE = 17;        // additive sums of ObstacleBlock.h:33-36

// Device status flags (bit set = raised); cup2d_sync reports the first.
enum : int { ST_NAN = 1, ST_DOMAIN = 2, ST_CAPACITY = 4, ST_TIMEOUT = 8 };

struct GridDesc {
  int nx, ny, bpdx, bpdy, nblocks;
  double h, extent;
  double ext[2];                  // SimulationData::extents (SimulationData.cpp:34-35)
  double nu, CFL, dlm;
  double fadeLenX, fadeLenY;
  int implicitPenal;              // cup2d_config.implicit_penalization
};

// PressureIterator_unif's state between steps (PressureIterator_unif.h:15-16)
// and of its last call: the relative momentum change of the last iteration,
// the adaptive target, the previous iteration count, the last count.
struct IterState {
  double relDF, target;
  int oldNsteps, last;
  double relDP;                   // PressureVarRho_approx: relative pressure change
};

// Per-step scalars (SimulationData.h:45-49 plus values passed between kernels).
struct Scalars {
  double time, dt, uinfx, uinfy, lambda;
  double maxU;
  double outflowCorr;             // advDiff.cpp:105
  double fadeCorr;                // PoissonSolver.cpp:86
  int step;
  int status;
  double rampCFL[100];            // Simulation.cpp:266-267, host-evaluated
  // calcMaxTimestep of the next step, formed at the end of a graph step from
  // the maxima the pressure correction and the force pass leave behind;
  // dtNextValid is cleared by every host-side change of the state
  double dtNext, maxUNext;
  int dtNextValid;
  // the next step's findMaxU maximum over the final velocity of a graph
  // step, accumulated by exact atomic max; reset at the start of the step
  double maxNext;
  // set by the midline launched at the start of a graph step: 1 if it could
  // run (the step's dt was carried), else the launch after the step's dt does
  int midlineEarly;
  IterState it;                   // iterated penalization (-iterativePenalization)
  // advDiff's coefficients of the step (afac, dfac, the W, S, E, N inflow
  // fades) and the RHS factor h/(2 dt), formed once by the outflow-flux
  // kernel that precedes every advDiff update
  double advCoef[6], facDiv;
};

struct ShapeCfg {
  int kind;
  double rhoS;
  int bFixedx, bFixedy, bForcedx, bForcedy, bBlockang;
  double forcedu, forcedv, forcedomega, timeForced;
  double origC[2], origAng;
  double radius, tAccel;                          // Disk
  double length, Tperiod, phaseShift, ampFac;     // Fish
  double curvScale[6];                            // StefanFish: scales of its curvature control values
  double envFourier[8];                           // envelope swimmer: its amplitude's Fourier coefficients
  int capacity;                                   // obstacle tile slots
  int nm;                                         // fish midline points
  int pid, pidpos;                                // StefanFish -pid / -pidpos (StefanFish.cpp:209-211)
};

// Fish frame bookkeeping (Fish.h:21-23).
struct FishState {
  double area_internal, J_internal;
  double CoM_internal[2], vCoM_internal[2];
  double theta_internal, angvel_internal, angvel_internal_prev;
  double cosTh, sinTh;            // cos/sin(theta_internal), set where theta_internal moves
  int midBuf;                     // midline buffer of the last placement
};

// CurvatureFish's actuation state (StefanFish.cpp:20-51, 85-131): the RL
// bending wave of ParameterSchedulerLearnWave<7> (node values and the time
// of the last turn, FishUtilities.h:317-385; t0 = -1 before any), the tail
// period with its phase bookkeeping, the PID curvature terms and the last
// actions (for StefanFish::state).
struct FishCtl {
  double bend[7], bendT0;
  double periodPIDval, periodPIDdif, time0, timeshift;
  double pidFac, pidDif;
  double lastTact, lastCurv, oldrCurv;
  // the PID controllers' exponential averages and memory (StefanFish.cpp:24-41)
  double avgDeltaY, avgDangle, avgAngVel, lastTime, lastAvel;
  int TperiodPID;
};

struct DevShape {
  cup2d_shape_state s;
  ShapeCfg cfg;
  FishState f;
  FishCtl ctl;
  int ntiles;                     // obstacle tiles this step
  int ntilesPrev;
  double rhoTile;                 // ObstacleBlock::rho: rhoS (disk), 1 (fish)
  double rhsCorr;                 // PressureSingle.cpp:183-186 corr of this shape
  double bbox[2][2];              // disk bounding box (ShapeLibrary.h:40-43)
  double cosO, sinO;              // cos/sin(orientation), set where the orientation moves
  int nseg;                       // fish AreaSegments this step
  // rigid part of udef removed by Shape::removeMoments (Shape.cpp:197-204):
  // consumers read udef - (Iu - Ia p_y, Iv + Ia p_x), the same expression
  double Iu, Iv, Ia;
};

// One fish AreaSegment (FishLibrary.h:149-168) in the computational frame.
struct Segment {
  int first, second;              // s_range
  double w[2], c[2];
  double normalI[2], normalJ[2];
  double boxLab[2][2], boxObj[2][2];
};

// Pointers to one shape's obstacle tiles (passed by value to kernels).
struct ObstTiles {
  int* tiles;                     // [capacity] block index of each slot
  int* slot;                      // [nblocks] slot of each block or -1
  double* chi;                    // [capacity][32][32]
  double* dist;
  double* udx;
  double* udy;
  double* sD;                     // surface delta D (0: not a surface point)
  double* sdx;                    // dchidx = -D * gradUX (ObstacleBlock.h:98)
  double* sdy;
  int capacity;
};

// One fish midline (the arrays of FishLibrary.h:49-60); the two step
// buffers also keep the skin of FishData::computeSurface
// (FishLibrary.cpp:178-194) in the midline's own frame: upper / lower x, y.
struct FishMidline {
  double *rX, *rY, *vX, *vY, *norX, *norY, *vNorX, *vNorY;
  double *uX, *uY, *lX, *lY;
};

// Per-fish device arrays.  The midline depends only on time, so the one for
// step n+1 is computed while step n runs: mid[] is double-buffered by step
// parity and holds the midline in the CoM frame with its integrals
// (integ[p*8 + ..]: area, CoM_internal[2], vCoM_internal[2], J_internal,
// angvel_internal, time); frame holds it rotated by theta_internal, which is
// what PutFishOnBlocks reads.
// PutFishOnBlocks' interior points: those of midline index ss are numbered
// off[ss] .. off[ss+1) for width offsets iw = -Nw+1 .. Nw-1 (Nw =
// floor(width/h), time-independent), ipIdx[] = (ss, iw) of each; the raster
// forms the points themselves from the frame midline.
struct FishArrays {
  double *rS, *width, *p1f;
  double* w3;                             // pow(width, 3), time-independent
  FishMidline mid[2];
  double* integ;
  FishMidline frame;
  Segment* seg;                           // [nseg]
  double* pool;                           // single allocation behind all arrays
  int* nw;                                // [nm] floor(width / h)
  int* off;                               // [nm + 1] interior point offsets
  int2* ipIdx;                            // [nint] (ss, iw) of each interior point
  int nm, nseg, nint;
};

// ---- optional in-graph timeline ------------------------------------------
// Built with -DCUP2D_TRACE, thread 0 of every CTA of every kernel records
// the %globaltimer at entry (atomicMin into slot 2*id) and at exit
// (atomicMax into slot 2*id+1), so one step's overlapped schedule can be
// read back.  Without the define the scope compiles to nothing.
enum TraceId : int {
  TR_MAXU, TR_SETDT, TR_ENDSTEP, TR_ADVDIFF, TR_RHSDIV, TR_PCORR, TR_FADE,
  TR_OBJBEGIN, TR_DISK_PLACE, TR_RASTER_DISK, TR_CHI, TR_MOMENTS,
  TR_UDEF, TR_RHSOBST, TR_RHSCORR, TR_MOMENTA, TR_COLLIDE, TR_PENALIZE, TR_FORCES,
  TR_MIDLINE, TR_FRAME, TR_RASTER, TR_R2C, TR_COLS, TR_C2R, TR_DCT_FWD, TR_DCT_COLS,
  TR_DCT_INV, TR_SELECT, TR_MAXNEXT, TR_N
};
// per-work-item phase stamps of the trace build: slot 2*TR_N + 8*item + phase
constexpr int TRACE_ITEMS = 4096;
#ifdef CUP2D_TRACE
static __device__ unsigned long long* g_trace = nullptr;   // one copy per translation unit
__device__ __forceinline__ unsigned long long global_timer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
struct TraceScope {
  int id;
  __device__ explicit TraceScope(int i) : id(i) {
    if (g_trace && threadIdx.x + threadIdx.y + threadIdx.z == 0) atomicMin(&g_trace[2 * id], global_timer());
  }
  __device__ ~TraceScope() {
    if (g_trace && threadIdx.x + threadIdx.y + threadIdx.z == 0) atomicMax(&g_trace[2 * id + 1], global_timer());
  }
};
#define CUP2D_TRACE_CAT2(a, b) a##b
#define CUP2D_TRACE_CAT(a, b) CUP2D_TRACE_CAT2(a, b)
#define CUP2D_TRACE_SCOPE(id) TraceScope CUP2D_TRACE_CAT(cup2d_trace_scope_, __LINE__)(id)
__device__ __forceinline__ unsigned long long global_timer_after(double dep) {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t) : "d"(dep));
  return t;
}
// the stamp is taken once dep has been computed
#define CUP2D_TRACE_MARK_AFTER(item, phase, dep) \
  do { if (g_trace && threadIdx.x + threadIdx.y + threadIdx.z == 0 && (item) < TRACE_ITEMS) \
         g_trace[2 * TR_N + 8 * (item) + (phase)] = global_timer_after(dep); } while (0)
#define CUP2D_TRACE_MARK(item, phase) \
  do { if (g_trace && threadIdx.x + threadIdx.y + threadIdx.z == 0 && (item) < TRACE_ITEMS) \
         g_trace[2 * TR_N + 8 * (item) + (phase)] = global_timer(); } while (0)
static inline void trace_bind_this_unit(unsigned long long* p) { cudaMemcpyToSymbol(g_trace, &p, sizeof(p)); }
#else
#define CUP2D_TRACE_SCOPE(id) ((void)0)
#define CUP2D_TRACE_MARK(item, phase) ((void)0)
#define CUP2D_TRACE_MARK_AFTER(item, phase, dep) ((void)0)
#endif

// Raise a kernel's dynamic shared-memory limit to what the device allows
// beside the kernel's static shared memory (opt-in maximum minus static).
// Done once per kernel with the device's maximum, so a context with a small
// grid never lowers the limit under a larger one.
inline cudaError_t allow_max_dynamic_smem(const void* f) {
  int dev = 0, maxOptin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&maxOptin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes a{};
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, f);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, maxOptin - (int)a.sharedSizeBytes);
  return e;
}

// ---- programmatic dependent launch ---------------------------------------
// Every pipeline kernel is launched with programmatic stream serialization
// (launch_k): the next kernel of the stream is launched as the CTAs of the
// previous one exit (the implicit trigger), without waiting for the grid's
// completion to be signalled.  Each kernel first waits for its predecessor's
// completion and memory, so completion stays transitive along the stream.
__device__ __forceinline__ void pdl_begin() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}
// Lets the next kernel of the stream launch now (its CTAs then run up to
// their pdl_begin, which still waits for this whole grid and its writes).
__device__ __forceinline__ void pdl_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ---- small device helpers ------------------------------------------------

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ int lin_tid() {
  return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
}
__device__ __forceinline__ int lin_nthreads() { return blockDim.x * blockDim.y * blockDim.z; }

// Warp reduce-scatter of KP (a power of two <= 32) values per lane: at each
// xor step (offsets 16, 8, .., 1) a lane keeps half of its list and adds
// its partner's copy of that half, so value k ends up, fully summed, in
// lanes k*32/KP .. k*32/KP + 32/KP - 1.  Every value is summed over the same
// xor pairing tree as a per-value butterfly: the totals are bitwise those
// of warp_sum, with KP - 1 + 5 - log2(KP) shuffles instead of 5 per value.
template <int KP>
__device__ __forceinline__ double warp_reduce_scatter(double (&x)[KP], int lane) {
  int m = KP;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    if (m > 1) {
      const int half = m >> 1;
      const bool upper = (lane & o) != 0;
#pragma unroll
      for (int i = 0; i < KP / 2; i++) {
        if (i < half) {
          const double lo = x[i], hi = x[i + half];
          const double recv = __shfl_xor_sync(0xffffffffu, upper ? lo : hi, o);
          x[i] = (upper ? hi : lo) + recv;
        }
      }
      m = half;
    } else {
      x[0] += __shfl_xor_sync(0xffffffffu, x[0], o);
    }
  }
  return x[0];
}

template <int K> struct Pow2Up { static constexpr int v = K <= 1 ? 1 : K <= 2 ? 2 : K <= 4 ? 4 : K <= 8 ? 8 : K <= 16 ? 16 : 32; };

// Block-wide sum of K (<= 32) values per thread; result valid in linear
// thread 0.  smem must hold 32*K doubles.  Fixed reduction order
// (deterministic): the xor tree within each warp, then the xor tree over
// the warps' partial sums.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* smem) {
  constexpr int KP = Pow2Up<K>::v, STRIDE = 32 / KP;
  const int t = lin_tid(), lane = t & 31, wid = t >> 5;
  const int nw = (lin_nthreads() + 31) >> 5;
  double x[KP];
#pragma unroll
  for (int k = 0; k < KP; k++) x[k] = k < K ? v[k] : 0.0;
  const double r = warp_reduce_scatter<KP>(x, lane);
  __syncthreads();
  if (lane % STRIDE == 0 && lane / STRIDE < K) smem[wid * K + lane / STRIDE] = r;
  __syncthreads();
  if (wid == 0) {
    double y[KP];
#pragma unroll
    for (int k = 0; k < KP; k++) y[k] = (k < K && lane < nw) ? smem[lane * K + k] : 0.0;
    const double r2 = warp_reduce_scatter<KP>(y, lane);
    __syncwarp();
    if (lane % STRIDE == 0 && lane / STRIDE < K) smem[lane / STRIDE] = r2;
    __syncwarp();
    if (lane == 0)
#pragma unroll
      for (int k = 0; k < K; k++) v[k] = smem[k];
  }
  __syncthreads();
}

// One warp's fixed-order sum of K values over n rows (value k of row i at
// p[stride i + k], read through L2): lane l adds rows l, l + 32, ..., then
// the xor reduce-scatter of block_sum; every lane returns all K totals.  For
// the last-CTA finishes, whose rows (tiles) number tens: a CTA-wide
// block_sum would only add barriers.  All 32 lanes of the warp call it.
template <int K>
__device__ __forceinline__ void warp_sum_rows(const double* p, int n, int stride, double (&out)[K]) {
  constexpr int KP = Pow2Up<K>::v, STRIDE = 32 / KP;
  const int lane = lin_tid() & 31;
  double x[KP];
#pragma unroll
  for (int k = 0; k < KP; k++) x[k] = 0.0;
  for (int i = lane; i < n; i += 32)
#pragma unroll
    for (int k = 0; k < K; k++) x[k] += __ldcg(&p[(size_t)stride * i + k]);
  const double r = warp_reduce_scatter<KP>(x, lane);
#pragma unroll
  for (int k = 0; k < K; k++) out[k] = __shfl_sync(0xffffffffu, r, k * STRIDE);
}

__device__ __forceinline__ double block_max(double v, double* smem) {
  const int t = lin_tid(), lane = t & 31, wid = t >> 5;
  const int nw = (lin_nthreads() + 31) >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) smem[wid] = v;
  __syncthreads();
  if (wid == 0) v = warp_max(lane < nw ? smem[lane] : 0.0);
  __syncthreads();
  return v;
}

// "last block done" ticket: returns true in every thread of the CTA that
// finished last.  The counter is re-armed by that CTA (its next user is a
// later kernel).  The CTA barrier orders every thread's earlier writes
// before thread 0's ticket, an acquire-release atomic at gpu scope: its
// release covers the whole CTA's writes (cumulativity), and in the last CTA
// its acquire covers everybody else's before the closing barrier.
__device__ __forceinline__ bool last_block_done(unsigned* counter, unsigned nblocks) {
  __shared__ bool amLast;
  __syncthreads();
  if (lin_tid() == 0) {
    unsigned t;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(t) : "l"(counter) : "memory");
    amLast = (t == nblocks - 1);
    if (amLast) *counter = 0;
  }
  __syncthreads();
  return amLast;
}

// atomic max on doubles through the ordered-integer mapping of IEEE-754
// Max of non-negative doubles (speeds: +0 and up, +inf, never NaN): their
// bit patterns order as the values do, so one native 64-bit unsigned atomic
// max (no compare-and-swap retries) suffices where many CTAs finishing at
// once contend on one address.
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double val) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(__double_as_longlong(val)));
}
__device__ __forceinline__ void atomic_max_double(double* addr, double val) {
  unsigned long long* a = reinterpret_cast<unsigned long long*>(addr);
  unsigned long long old = *a, assumed;
  do {
    assumed = old;
    if (__longlong_as_double(assumed) >= val) return;
    old = atomicCAS(a, assumed, __double_as_longlong(val));
  } while (old != assumed);
}

// Per-tile udef after Shape::removeMoments (Shape.cpp:197-204), evaluated
// where it is read: udef - (I.u - I.a p1), udef - (I.v + I.a p0), p = x - CoM.
__device__ __forceinline__ void udef_at(const ObstTiles& t, size_t o, const DevShape& S,
                                        double p0, double p1, double& u0, double& u1) {
  u0 = t.udx[o] - (S.Iu - S.Ia * p1);
  u1 = t.udy[o] - (S.Iv + S.Ia * p0);
}

// Cell-centre position of cell (ix,iy) of block (bx,by); the same expression
// as the oracle's BlockInfo::pos (origin + h*(i + 1/2), origin = 32*b*h).
__host__ __device__ __forceinline__ double cell_x(const GridDesc& g, int bx, int ix) {
  return (double)(bx * BS) * g.h + g.h * (ix + 0.5);
}
__host__ __device__ __forceinline__ double cell_y(const GridDesc& g, int by, int iy) {
  return (double)(by * BS) * g.h + g.h * (iy + 0.5);
}
__device__ __forceinline__ double gx_pos(const GridDesc& g, int gx) {
  return cell_x(g, gx >> 5, gx & 31);
}
__device__ __forceinline__ double gy_pos(const GridDesc& g, int gy) {
  return cell_y(g, gy >> 5, gy & 31);
}

// ---- fade sums of PoissonSolver::solve (PoissonSolver.cpp:61-100) ----------
// The strip blocks (those that reach the boundary fade strip, the test of
// PoissonSolver.cpp:71-79) each own three sums of the faded RHS (sumRHS,
// sumPOS, sumNEG), kept at rank slot (block order among strip blocks).
// Both producers of a block's sums (the RHS divergence, and the RHS
// correction of an obstacle tile in the strip) use one order: 32 x 8
// threads, thread (tx, ty) adds rows ty + 8r, r = 0..3, then block_sum<3>
// over the CTA (further warps adding zeros), so the sums are the same
// whichever kernel wrote them last.
// A kernel's last word to mapped host memory: everything it wrote before
// becomes visible to the host first (system-scope fence), then the host's
// spin word takes seqVal.
__device__ __forceinline__ void signal_host(unsigned long long* seqOut, unsigned long long seqVal) {
  if (!seqOut) return;
  __threadfence_system();
  *reinterpret_cast<volatile unsigned long long*>(seqOut) = seqVal;
}

__device__ __forceinline__ bool fade_touch(const GridDesc& g, int bx, int by) {
  const double minx = cell_x(g, bx, 0), maxx = cell_x(g, bx, BS - 1);
  const double miny = cell_y(g, by, 0), maxy = cell_y(g, by, BS - 1);
  return g.fadeLenX >= minx || g.fadeLenX >= g.ext[0] - maxx ||
         g.fadeLenY >= miny || g.fadeLenY >= g.ext[1] - maxy;
}
// adds cell (ix, iy) of block (bx, by), of RHS b, to s (PoissonSolver.cpp:86-95)
__device__ __forceinline__ void fade_accumulate(const GridDesc& g, int bx, int by, int ix, int iy,
                                                double b, double (&s)[3]) {
  const double fadeLenX = g.fadeLenX, invFadeX = 1 / fmax(fadeLenX, EPSd);
  const double fadeLenY = g.fadeLenY, invFadeY = 1 / fmax(fadeLenY, EPSd);
  const double px = cell_x(g, bx, ix), py = cell_y(g, by, iy);
  const double yt = invFadeY * fmax(0.0, fadeLenY - g.ext[1] + py);
  const double yb = invFadeY * fmax(0.0, fadeLenY - py);
  const double xt = invFadeX * fmax(0.0, fadeLenX - g.ext[0] + px);
  const double xb = invFadeX * fmax(0.0, fadeLenX - px);
  const double fadeArg = fmin(fmax(fmax(yt, yb), fmax(xt, xb)), 1.0);
  const double fadedRHS = b * (fadeArg * fadeArg);
  if (fadedRHS < 0) s[2] -= fadedRHS;
  if (fadedRHS > 0) s[1] += fadedRHS;
  s[0] += fadedRHS;
}
// fadeCorr (PoissonSolver.cpp:80-86) from the sums of the n strip blocks,
// formed by one warp (all 32 lanes call it) in an order that depends on n
// alone: lane l adds slots l, l + 32, ... (loads issued four at a time),
// then an xor butterfly, which leaves the same sums in every lane.  Every
// CTA that needs the value forms it itself and all get the same bits.
__device__ __forceinline__ double fade_corr(const double* partials, int n) {
  const int lane = threadIdx.x & 31;
  double t[3] = {0, 0, 0};
  for (int i0 = 0; i0 < n; i0 += 128) {
    double v[4][3];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int i = i0 + lane + 32 * u;
#pragma unroll
      for (int k = 0; k < 3; k++) v[u][k] = i < n ? __ldcg(&partials[3 * i + k]) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int k = 0; k < 3; k++) t[k] += v[u][k];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int k = 0; k < 3; k++) t[k] += __shfl_xor_sync(0xffffffffu, t[k], o);
  const double sumNEG = fmax(t[2], EPSd), sumPOS = fmax(t[1], EPSd);
  return t[0] > 0 ? t[0] / sumPOS : t[0] / sumNEG;
}

} // namespace cup2d
