// Dense grid kernels of the timestep: findMaxU + dt, advDiff, the outflow
// correction, the pressure RHS divergence, the fade reductions of cub2rhs,
// the pressure correction, IC and ApplyObjVel.
//
// Every kernel maps one CTA to one 32x32 reference block (blockDim 32x8,
// 4 rows per thread): a warp reads one 256-byte fp64 row segment, the
// 5-point halo comes from L1/L2 (neighbour rows are read by the CTA itself,
// neighbour columns by the adjacent CTA), so DRAM sees each plane once.
// Arithmetic is written in the reference's operation order and the library
// is compiled without FMA contraction, so a stage fed the same inputs as the
// reference reproduces it bit for bit (reductions excepted: their order
// differs).
#include <cmath>
#include "context.hpp"
#include "step_begin.cuh"

namespace cup2d {

namespace {

__global__ void __launch_bounds__(512)
k_max_u_dt(GridDesc g, Scalars* sc, const DevShape* sh, int nsh,
           const double* __restrict__ u, const double* __restrict__ v,
           double* partials, unsigned* counter)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_MAXU);
  __shared__ double red[64];
  max_u_dt_cta(g, sc, sh, nsh, u, v, partials, counter, red);
}

__global__ void k_set_dt(Scalars* sc, double dt) { pdl_begin(); CUP2D_TRACE_SCOPE(TR_SETDT); sc->dt = dt; }

__global__ void k_end_step(Scalars* sc) { pdl_begin(); CUP2D_TRACE_SCOPE(TR_ENDSTEP);
  sc->time += sc->dt;
  sc->step += 1;
}

// End of a graph step: t += dt, step += 1, then the next step's
// calcMaxTimestep from the maximum k_max_next formed on the final velocity
// (max is exact in any order: dtNext equals what k_max_u_dt would form).
__global__ void k_end_step_dt(GridDesc g, Scalars* sc, const DevShape* sh, int nsh)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_ENDSTEP);
  const double m = sc->maxNext;
  sc->time += sc->dt;
  sc->step += 1;
  sc->dtNext = dt_from_max_u(g, sc, sh, nsh, m);
  sc->maxUNext = m;
  sc->dtNextValid = 1;
}

// advDiff.cpp:14-87.  Ghosts: neighbour cells, or at the domain edge the
// zero-gradient copy scaled by the inflow fade of advDiff.cpp:50-55,68-71.
__global__ void __launch_bounds__(256, 4)
k_advdiff(GridDesc g, const Scalars* sc,
          const double* __restrict__ u, const double* __restrict__ v,
          double* __restrict__ un, double* __restrict__ vn,
          double* partials, unsigned* counter, Scalars* scw)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_ADVDIFF);
  __shared__ double red[32];
  const double dt = sc->dt, h = g.h;
  const double UINF0 = sc->uinfx, UINF1 = sc->uinfy;
  // the step's coefficients dfac = (nu/h)(dt/h), afac = -0.5 dt/h and the
  // inflow fades 1 - r^2/100 of r = max/min(U, 0)/max(|U|): seven quotients
  // (eleven divisions), each evaluated by its own lane of the warp (lane =
  // threadIdx.x) and shared by shuffles, the same operations as evaluating
  // all of them in every thread
  double qa = 1.0, qb = 1.0;
  {
    const double norUinf = fmax(fmax(fabs(UINF0), fabs(UINF1)), EPSd);
    switch (threadIdx.x) {
      case 0: qa = -0.5 * dt; qb = h; break;
      case 1: qa = g.nu; qb = h; break;
      case 2: qa = dt; qb = h; break;
      case 3: qa = fmax(UINF0, 0.0); qb = norUinf; break;     // W
      case 4: qa = fmax(UINF1, 0.0); qb = norUinf; break;     // S
      case 5: qa = fmin(UINF0, 0.0); qb = norUinf; break;     // E
      case 6: qa = fmin(UINF1, 0.0); qb = norUinf; break;     // N
      default: break;
    }
  }
  const double q = qa / qb, fq = 1 - q * q / 100;
  const double afac = __shfl_sync(0xffffffffu, q, 0);
  const double dfac = __shfl_sync(0xffffffffu, q, 1) * __shfl_sync(0xffffffffu, q, 2);
  const double fadeW = __shfl_sync(0xffffffffu, fq, 3), fadeS = __shfl_sync(0xffffffffu, fq, 4);
  const double fadeE = __shfl_sync(0xffffffffu, fq, 5), fadeN = __shfl_sync(0xffffffffu, fq, 6);
  const int nx = g.nx, ny = g.ny;
  const int gx = blockIdx.x * BS + threadIdx.x;
  double IF = 0;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int gy = blockIdx.y * BS + threadIdx.y + 8 * r;
    const size_t c = (size_t)gy * nx + gx;
    const double ucc = u[c], vcc = v[c];
    double ulx, vlx, upx, vpx, uly, vly, upy, vpy;
    if (gx > 0) { ulx = u[c - 1]; vlx = v[c - 1]; } else { ulx = ucc * fadeW; vlx = vcc * fadeW; }
    if (gx < nx - 1) { upx = u[c + 1]; vpx = v[c + 1]; } else { upx = ucc * fadeE; vpx = vcc * fadeE; }
    if (gy > 0) { uly = u[c - nx]; vly = v[c - nx]; } else { uly = ucc * fadeS; vly = vcc * fadeS; }
    if (gy < ny - 1) { upy = u[c + nx]; vpy = v[c + nx]; } else { upy = ucc * fadeN; vpy = vcc * fadeN; }
    const double dUadv = (ucc + UINF0) * (upx - ulx) + (vcc + UINF1) * (upy - uly);
    const double dUdif = upx + upy + ulx + uly - 4 * ucc;
    const double dVadv = (ucc + UINF0) * (vpx - vlx) + (vcc + UINF1) * (vpy - vly);
    const double dVdif = vpx + vpy + vlx + vly - 4 * vcc;
    const double unew = ucc + (afac * dUadv + dfac * dUdif);
    const double vnew = vcc + (afac * dVadv + dfac * dVdif);
    un[c] = unew; vn[c] = vnew;
    // advDiff.cpp:93-102: net outflow through the domain boundary
    if (gx == 0) IF -= unew;
    if (gx == nx - 1) IF += unew;
    if (gy == 0) IF -= vnew;
    if (gy == ny - 1) IF += vnew;
  }
  const bool edgeBlock = blockIdx.x == 0 || blockIdx.y == 0 ||
                         blockIdx.x == gridDim.x - 1 || blockIdx.y == gridDim.y - 1;
  const unsigned nb = gridDim.x * gridDim.y, bid = blockIdx.x + gridDim.x * blockIdx.y;
  if (edgeBlock) {
    double s[1] = {IF};
    block_sum<1>(s, red);
    if (threadIdx.x == 0 && threadIdx.y == 0) partials[bid] = s[0];
  } else if (threadIdx.x == 0 && threadIdx.y == 0) {
    partials[bid] = 0.0;
  }
  if (!last_block_done(counter, nb)) return;
  const int tid = threadIdx.x + 32 * threadIdx.y;
  double s[1] = {0.0};
  for (unsigned i = tid; i < nb; i += 256) s[0] += __ldcg(&partials[i]);
  block_sum<1>(s, red);
  __shared__ double corrS;
  if (tid == 0) {  // advDiff.cpp:105
    corrS = s[0] / (2 * (BS * g.bpdy - 0) + 2 * (BS * g.bpdx - 0));
    scw->outflowCorr = corrS;
  }
  __syncthreads();
  // advDiff.cpp:107-115, applied by this last CTA once every new value exists.
  // Item k < ny is row k (u at its west and east cells), item ny + i column
  // i (v at its south and north cells); a thread loads the pairs of UB
  // items before it stores any, so their L2 round trips overlap.
  const double corr = corrS;
  constexpr int UB = 4;
  const int nitems = ny + nx;
  for (int k0 = tid; k0 < nitems; k0 += 256 * UB) {
    double lo[UB], hi[UB];
    size_t alo[UB], ahi[UB];
    bool isU[UB];
#pragma unroll
    for (int u = 0; u < UB; u++) {
      const int k = k0 + 256 * u;
      isU[u] = k < ny;
      alo[u] = isU[u] ? (size_t)k * nx : (size_t)(k - ny);
      ahi[u] = isU[u] ? (size_t)k * nx + nx - 1 : (size_t)(ny - 1) * nx + (k - ny);
      if (k < nitems) {
        const double* f = isU[u] ? un : vn;
        lo[u] = __ldcg(&f[alo[u]]);
        hi[u] = __ldcg(&f[ahi[u]]);
      }
    }
#pragma unroll
    for (int u = 0; u < UB; u++)
      if (k0 + 256 * u < nitems) {
        double* f = isU[u] ? un : vn;
        f[alo[u]] = lo[u] + corr;
        f[ahi[u]] = hi[u] - corr;
      }
  }
}

// PressureSingle.cpp:112-128: tmp = (h / 2dt) * div_2h(u); zero-gradient ghosts
__global__ void __launch_bounds__(256)
k_rhs_div(GridDesc g, const Scalars* sc, const double* __restrict__ u,
          const double* __restrict__ v, double* __restrict__ rhs,
          const int* __restrict__ fadeSlot, double* __restrict__ fadePartials)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_RHSDIV);
  const double h = g.h, facDiv = 0.5 * h / sc->dt;
  const int nx = g.nx, ny = g.ny;
  const int bx = blockIdx.x, by = blockIdx.y;
  const int gx = bx * BS + threadIdx.x;
  const bool touch = fade_touch(g, bx, by);
  double s[3] = {0, 0, 0};
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int iy = threadIdx.y + 8 * r, gy = by * BS + iy;
    const size_t c = (size_t)gy * nx + gx;
    const double uW = u[gx > 0 ? c - 1 : c], uE = u[gx < nx - 1 ? c + 1 : c];
    const double vS = v[gy > 0 ? c - nx : c], vN = v[gy < ny - 1 ? c + nx : c];
    const double divVx = uE - uW, divVy = vN - vS;
    const double b = facDiv * (divVx + divVy);
    rhs[c] = b;
    if (touch) fade_accumulate(g, bx, by, threadIdx.x, iy, b, s);
  }
  // a strip block's fade sums of the RHS as it leaves the divergence; the
  // obstacle terms rewrite those of their own tiles
  if (touch) {
    __shared__ double red[96];
    block_sum<3>(s, red);
    if (lin_tid() == 0) {
      const int q = fadeSlot[bx + g.bpdx * by];
      for (int k = 0; k < 3; k++) fadePartials[3 * q + k] = s[k];
    }
  }
}

// fadeSlot[b] = rank of block b among the strip blocks (block order), or -1;
// fadeSlot[nblocks] = their number.  Once per grid, one thread.
__global__ void k_fade_slots(GridDesc g, int* fadeSlot)
{
  int n = 0;
  for (int b = 0; b < g.nblocks; b++) fadeSlot[b] = fade_touch(g, b % g.bpdx, b / g.bpdx) ? n++ : -1;
  fadeSlot[g.nblocks] = n;
}

// PressureSingle.cpp:216-241: V += -(dt/2h) grad_2h P; zero-gradient P ghosts.
// Reads the velocity written by advDiff (ui, vi) and writes the current one.
__global__ void __launch_bounds__(256)
k_pcorr(GridDesc g, const Scalars* sc, const double* __restrict__ p,
        const double* __restrict__ ui, const double* __restrict__ vi,
        double* __restrict__ uo, double* __restrict__ vo)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_PCORR);
  const double pFac = -0.5 * sc->dt / g.h;
  const int nx = g.nx, ny = g.ny;
  const int gx = blockIdx.x * BS + threadIdx.x;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int gy = blockIdx.y * BS + threadIdx.y + 8 * r;
    const size_t c = (size_t)gy * nx + gx;
    const double pW = p[gx > 0 ? c - 1 : c], pE = p[gx < nx - 1 ? c + 1 : c];
    const double pS = p[gy > 0 ? c - nx : c], pN = p[gy < ny - 1 ? c + nx : c];
    uo[c] = ui[c] + pFac * (pE - pW);
    vo[c] = vi[c] + pFac * (pN - pS);
  }
}

// The next step's findMaxU (Helpers.cpp:136-176) on the step's final
// velocity, beside the force pass (which only reads it).  Per-CTA maxima
// meet in sc->maxNext by exact atomic max.
__global__ void __launch_bounds__(256)
k_max_next(GridDesc g, Scalars* sc, const double* __restrict__ u, const double* __restrict__ v)
{
  pdl_begin();
  CUP2D_TRACE_SCOPE(TR_MAXNEXT);
  __shared__ double red[32];
  const double UINF = sc->uinfx, VINF = sc->uinfy;
  double m = 0.0;
  int bad = 0;
  const size_t n2 = (size_t)g.nx * g.ny / 2;
  const double2* u2 = reinterpret_cast<const double2*>(u);
  const double2* v2 = reinterpret_cast<const double2*>(v);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n2; i += (size_t)gridDim.x * blockDim.x) {
    const double2 a = u2[i], b = v2[i];
    m = fmax(m, cell_speed(a.x, b.x, UINF, VINF));
    m = fmax(m, cell_speed(a.y, b.y, UINF, VINF));
    bad |= !isfinite(a.x) || !isfinite(b.x) || !isfinite(a.y) || !isfinite(b.y);
  }
  m = block_max(m, red);
  const int anyBad = __syncthreads_or(bad);
  if (lin_tid() == 0) {
    atomic_max_double(&sc->maxNext, m);
    if (anyBad) atomicOr(&sc->status, ST_NAN);
  }
}

__global__ void k_ic(size_t n, double* u, double* v, double* chi, double* pres,
                     double* rhs, double* sdf, double* udx, double* udy)
{
  pdl_begin();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    u[i] = 0; v[i] = 0; chi[i] = 0; pres[i] = 0; rhs[i] = 0;
    sdf[i] = -1; udx[i] = 0; udy[i] = 0;
  }
}

// Helpers.cpp:290-307: u <- u (1 - chi) + udef chi
__global__ void k_apply_obj_vel(size_t n, double* u, double* v, const double* chi,
                                const double* udx, const double* udy)
{
  pdl_begin();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double X = chi[i];
    u[i] = u[i] * (1 - X) + udx[i] * X;
    v[i] = v[i] * (1 - X) + udy[i] * X;
  }
}

inline int reduce_grid(const Ctx& c) {
  int n = (int)((c.ncells() + 255) / 256);
  return n < 148 * 8 ? n : 148 * 8;
}
inline int max_grid(const Ctx& c) {
  int n = (int)((c.ncells() / 2 + 511) / 512);
  return n < 148 * 2 ? n : 148 * 2;
}

} // namespace

void launch_max_u_dt(Ctx& c) {
  const int nb = max_grid(c);
  launch_k(k_max_u_dt, nb, 512, 0, c.stream, c.g, c.dsc, c.dshapes, c.nshapes, c.u(), c.v(),
                                        c.partials, c.counters + CNT_MAXU);
  CUP2D_LAUNCHED(c);
}

void launch_set_dt(Ctx& c, double dt) {
  launch_k(k_set_dt, 1, 1, 0, c.stream, c.dsc, dt);
  CUP2D_LAUNCHED(c);
}

void launch_end_step(Ctx& c) {
  launch_k(k_end_step, 1, 1, 0, c.stream, c.dsc);
  CUP2D_LAUNCHED(c);
}

void launch_max_next(Ctx& c) {
  launch_k(k_max_next, max_grid(c), 256, 0, c.stream, c.g, c.dsc, c.u(), c.v());
  CUP2D_LAUNCHED(c);
}

void launch_end_step_dt(Ctx& c) {
  launch_k(k_end_step_dt, 1, 1, 0, c.stream, c.g, c.dsc, c.dshapes, c.nshapes);
  CUP2D_LAUNCHED(c);
}

void launch_advdiff(Ctx& c) {
  dim3 grid(c.g.bpdx, c.g.bpdy), block(32, 8);
  launch_k(k_advdiff, grid, block, 0, c.stream, c.g, c.dsc, c.u(), c.v(), c.uo(), c.vo(),
                                          c.partials, c.counters + CNT_ADV, c.dsc);
  CUP2D_LAUNCHED(c);
  c.cur = 1 - c.cur;   // advDiff.cpp:81-87: the new field becomes the velocity
}

// timing helpers: return the velocity to the buffer it came from (no launch)
void launch_advdiff_undo(Ctx& c) { c.cur = 1 - c.cur; }
void launch_pcorr_undo(Ctx& c) { c.cur = 1 - c.cur; }

void launch_outflow(Ctx& c) {
  // applied by the last CTA of k_advdiff (advDiff.cpp:89-116)
  (void)c;
}

void launch_rhs_div(Ctx& c) {
  dim3 grid(c.g.bpdx, c.g.bpdy), block(32, 8);
  launch_k(k_rhs_div, grid, block, 0, c.stream, c.g, c.dsc, c.u(), c.v(), c.rhs, (const int*)c.fadeSlot,
           fade_partials(c));
  CUP2D_LAUNCHED(c);
}

int build_fade_slots(Ctx& c) {
  k_fade_slots<<<1, 1, 0, c.stream>>>(c.g, c.fadeSlot);
  int n = -1;
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(&n, c.fadeSlot + c.g.nblocks, sizeof(int), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
      cudaStreamSynchronize(c.stream) != cudaSuccess) return -1;
  return n;
}

void launch_pcorr(Ctx& c) {
  dim3 grid(c.g.bpdx, c.g.bpdy), block(32, 8);
  launch_k(k_pcorr, grid, block, 0, c.stream, c.g, c.dsc, c.pres, c.u(), c.v(), c.uo(), c.vo());
  CUP2D_LAUNCHED(c);
  c.cur = 1 - c.cur;
}

void launch_ic(Ctx& c) {
  launch_k(k_ic, reduce_grid(c), 256, 0, c.stream, c.ncells(), c.u(), c.v(), c.chi, c.pres, c.rhs,
                                              c.sdf, c.udefx, c.udefy);
  CUP2D_LAUNCHED(c);
}

void launch_apply_obj_vel(Ctx& c) {
  launch_k(k_apply_obj_vel, reduce_grid(c), 256, 0, c.stream, c.ncells(), c.u(), c.v(), c.chi,
                                                         c.udefx, c.udefy);
  CUP2D_LAUNCHED(c);
}

} // namespace cup2d

#ifdef CUP2D_TRACE
namespace cup2d { void trace_bind_fluid(unsigned long long* p) { trace_bind_this_unit(p); } }
#endif
