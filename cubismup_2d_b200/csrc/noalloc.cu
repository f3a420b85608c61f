// cup2d_adv_diff_noalloc: the advDiff operator on caller-owned device
// buffers, for callers that cannot allocate device memory.
//
// The regular entry points allocate their reduction scratch once per
// context with cudaMalloc.  Some hosts cannot do that: applications that
// hand all of the GPU's memory to their own pool or caching allocator (a raw
// cudaMalloc then fails, or carves memory the pool believes it owns), and
// latency-critical loops that must not call cudaMalloc/cudaFree because those
// calls synchronise the device and take far longer than the stencil itself.
// This entry point therefore keeps its scratch -- the per-CTA partial sums of
// the boundary outflow and the "last CTA" ticket -- in one fixed
// file-scope device array that is part of the loaded library.
//
// Contract
//  - scratch: g_advdiff_scratch below, CUP2D_NOALLOC_MAX_BLOCKS partial sums
//    (one per 32x32 block) plus a few slots, about 128 KB; every GPU that
//    loads the library holds it until the process exits;
//  - grids with more than CUP2D_NOALLOC_MAX_BLOCKS blocks are rejected with
//    CUP2D_ETOOLARGE before anything is launched;
//  - the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it; make the
//    first call on each device before any stream capture begins;
//  - all calls share the one array and it keeps the last call's contents:
//    each call clears the ticket counter on its stream first, and calls whose
//    executions overlap on the GPU (other streams, other host threads) race
//    on the array and give wrong results;
//  - no cudaMalloc, cudaFree or allocating library routine is called.
#include <mutex>
#include "internal.cuh"

namespace cup2d {
namespace {

constexpr int kMaxDevices = 64;
constexpr int kScratchHead = 32;   // [0] ticket counter, [1] outflow correction

static __device__ __align__(256) double g_advdiff_scratch[kScratchHead + CUP2D_NOALLOC_MAX_BLOCKS];

std::mutex g_mutex;
double* g_scratch_ptr[kMaxDevices] = {nullptr};

struct Args {
  int nx, ny, bpdx, bpdy;
  double h, nu, dt, uinfx, uinfy;
};

// advDiff.cpp:14-87 (explicit Euler, central advection, 5-point diffusion,
// inflow-fade ghosts) with the boundary outflow sum of advDiff.cpp:93-102.
__global__ void __launch_bounds__(256)
k_advdiff_noalloc(Args a, const double* __restrict__ u, const double* __restrict__ v,
                  double* __restrict__ un, double* __restrict__ vn, double* scratch)
{
  __shared__ double red[32];
  const double dt = a.dt, h = a.h;
  const double UINF0 = a.uinfx, UINF1 = a.uinfy;
  const double dfac = (a.nu / h) * (dt / h), afac = -0.5 * dt / h;
  const double norUinf = fmax(fmax(fabs(UINF0), fabs(UINF1)), EPSd);
  const double rW = fmax(UINF0, 0.0) / norUinf, rS = fmax(UINF1, 0.0) / norUinf;
  const double rE = fmin(UINF0, 0.0) / norUinf, rN = fmin(UINF1, 0.0) / norUinf;
  const double fadeW = 1 - rW * rW / 100, fadeS = 1 - rS * rS / 100;
  const double fadeE = 1 - rE * rE / 100, fadeN = 1 - rN * rN / 100;
  const int nx = a.nx, ny = a.ny;
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
    if (gx == 0) IF -= unew;
    if (gx == nx - 1) IF += unew;
    if (gy == 0) IF -= vnew;
    if (gy == ny - 1) IF += vnew;
  }
  const unsigned nb = gridDim.x * gridDim.y, bid = blockIdx.x + gridDim.x * blockIdx.y;
  double* partials = scratch + kScratchHead;
  double s[1] = {IF};
  block_sum<1>(s, red);
  if (lin_tid() == 0) partials[bid] = s[0];
  if (!last_block_done(reinterpret_cast<unsigned*>(scratch), nb)) return;
  const int tid = lin_tid();
  double t[1] = {0.0};
  for (unsigned i = tid; i < nb; i += 256) t[0] += __ldcg(&partials[i]);
  block_sum<1>(t, red);
  if (tid == 0) scratch[1] = t[0] / (2 * (BS * a.bpdy - 0) + 2 * (BS * a.bpdx - 0));   // advDiff.cpp:105
}

// advDiff.cpp:107-115: subtract the mean outflow on the boundary cells
__global__ void k_outflow_noalloc(Args a, double* __restrict__ u, double* __restrict__ v,
                                  const double* scratch)
{
  const double corr = scratch[1];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = a.nx, ny = a.ny;
  if (i < ny) {
    u[(size_t)i * nx] += corr;
    u[(size_t)i * nx + nx - 1] -= corr;
  }
  if (i < nx) {
    v[i] += corr;
    v[(size_t)(ny - 1) * nx + i] -= corr;
  }
}

// Device address of the scratch array on the current device, looked up once.
int scratch_address(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return CUP2D_ECUDA;
  if (dev < 0 || dev >= kMaxDevices) return CUP2D_EINVAL;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_ptr[dev]) {
    double* p = nullptr;
    if (cudaGetSymbolAddress((void**)&p, g_advdiff_scratch) != cudaSuccess || !p) return CUP2D_ECUDA;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return CUP2D_OK;
}

} // namespace
} // namespace cup2d

extern "C" int cup2d_adv_diff_noalloc(const double* u, const double* v, double* u_out, double* v_out,
                                      int bpdx, int bpdy, double h, double nu, double dt,
                                      double uinfx, double uinfy, void* stream)
{
  using namespace cup2d;
  if (!u || !v || !u_out || !v_out || bpdx <= 0 || bpdy <= 0 || !(h > 0) || !(dt >= 0))
    return CUP2D_EINVAL;
  if ((long long)bpdx * bpdy > CUP2D_NOALLOC_MAX_BLOCKS) return CUP2D_ETOOLARGE;
  if (u_out == u || v_out == v || u_out == v || v_out == u) return CUP2D_EINVAL;
  double* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc != CUP2D_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(scratch, 0, sizeof(double), s) != cudaSuccess) return CUP2D_ECUDA;  // ticket = 0
  Args a{BS * bpdx, BS * bpdy, bpdx, bpdy, h, nu, dt, uinfx, uinfy};
  k_advdiff_noalloc<<<dim3(bpdx, bpdy), dim3(32, 8), 0, s>>>(a, u, v, u_out, v_out, scratch);
  const int n = a.nx > a.ny ? a.nx : a.ny;
  k_outflow_noalloc<<<(n + 255) / 256, 256, 0, s>>>(a, u_out, v_out, scratch);
  return cudaGetLastError() == cudaSuccess ? CUP2D_OK : CUP2D_ECUDA;
}
