// The C ABI (include/cup2d.h): context lifetime, shapes, the pipeline stages
// in Simulation::advance order, CUDA-graph replay of whole steps, and state
// exchange.  No entry point aborts: failures come back as status codes.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>
#include "context.hpp"
#include "fish.cuh"

using namespace cup2d;

namespace {

#define CK(call)                                                                \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      ctx->c.err = std::string(#call) + ": " + cudaGetErrorString(e_);          \
      return CUP2D_ECUDA;                                                       \
    }                                                                           \
  } while (0)

int fail(cup2d_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->c.err = msg;
  return code;
}

int check_launch(cup2d_ctx* ctx) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ctx, CUP2D_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return CUP2D_OK;
}

template <typename T>
int dalloc(cup2d_ctx* ctx, T** p, size_t n) {
  if (cudaMalloc((void**)p, sizeof(T) * (n ? n : 1)) != cudaSuccess)
    return fail(ctx, CUP2D_ENOMEM, "cudaMalloc failed");
  return CUP2D_OK;
}

// Natural cubic spline, IF2D_Interpolation1D::naturalCubicSpline
// (FishUtilities.h:85-130): second derivatives by the tridiagonal sweep,
// then bisection and the cubic in the bracketing interval.
void natural_spline(const double* x, const double* y, int n, const double* xx, double* yy, int nn) {
  std::vector<double> y2(n), u(n > 1 ? n - 1 : 1);
  y2[0] = 0; u[0] = 0;
  for (int i = 1; i < n - 1; i++) {
    const double sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
    const double p = sig * y2[i - 1] + 2;
    y2[i] = (sig - 1) / p;
    u[i] = (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
    u[i] = (6 * u[i] / (x[i + 1] - x[i - 1]) - sig * u[i - 1]) / p;
  }
  const double qn = 0, un = 0;
  y2[n - 1] = (un - qn * u[n - 2]) / (qn * y2[n - 2] + 1);
  for (int k = n - 2; k > 0; k--) y2[k] = y2[k] * y2[k + 1] + u[k];
  for (int j = 0; j < nn; j++) {
    unsigned klo = 0, khi = n - 1, k = 0;
    while (khi - klo > 1) {
      k = (khi + klo) >> 1;
      if (x[k] > (xx[j] + 0)) khi = k; else klo = k;
    }
    const double h = x[khi] - x[klo];
    const double a = (x[khi] - (xx[j] + 0)) / h;
    const double b = ((xx[j] + 0) - x[klo]) / h;
    yy[j] = a * y[klo] + b * y[khi] + ((a * a * a - a) * y2[klo] + (b * b * b - b) * y2[khi]) * (h * h) / 6;
  }
}

// The curvature amplitude along the body, sampled at rS: StefanFish's
// control values (StefanFish.cpp:187-193), each times its scale, splined
// onto rS; the envelope swimmer's carangiform envelope (cup2d.h) times the
// Fourier series f_0 + sum_{k=1..7} (f_k - 1) cos(k pi s / L) of its
// coefficients (1 as built: the envelope itself).
std::vector<double> curvature_profile(const ShapeCfg& f, const std::vector<double>& rS) {
  const int Nm = (int)rS.size();
  const double L = f.length;
  const double pts[6] = {0, .15 * L, .4 * L, .65 * L, .9 * L, L};
  const double base[6] = {0.82014 / L, 1.46515 / L, 2.57136 / L, 3.75425 / L, 5.09147 / L, 5.70449 / L};
  std::vector<double> p1f(Nm);
  if (f.kind == CUP2D_SHAPE_ENVELOPEFISH) {
    for (int i = 0; i < Nm; i++) {
      double m = f.envFourier[0];
      for (int k = 1; k < 8; k++) {
        if (f.envFourier[k] == 1) continue;
        m += (f.envFourier[k] - 1) * std::cos(k * M_PI * rS[i] / L);
      }
      p1f[i] = 0.82 * (rS[i] / L + 0.0025) / 1.0025 / L * m;
    }
  } else {
    double vals[6];
    for (int j = 0; j < 6; j++) vals[j] = base[j] * f.curvScale[j];
    natural_spline(pts, vals, 6, rS.data(), p1f.data(), Nm);
  }
  return p1f;
}

// FishData arclength grid (FishLibrary.cpp:14-38, FishLibrary.h:62-74) and
// the width profile of CurvatureFish/AmplitudeFish (StefanFish.cpp:175-182).
bool fish_grid(double L, double h, std::vector<double>& rS, std::vector<double>& width) {
  const double fracRefined = 0.1, fracMid = 1 - 2 * fracRefined;
  const double dSmid_tgt = h / std::sqrt(2);
  const double dSrefine_tgt = 0.125 * h;
  const int Nmid = (int)std::ceil(L * fracMid / dSmid_tgt / 8) * 8;
  const double dSmid = L * fracMid / Nmid;
  const int Nend = (int)std::ceil(fracRefined * L * 2 / (dSmid + dSrefine_tgt) / 4) * 4;
  const double dSref = fracRefined * L * 2 / Nend - dSmid;
  const int Nm = Nmid + 2 * Nend + 1;
  if (!(dSref > 0)) return false;       // FishLibrary.cpp:21 assert(dSref > 0)
  rS.assign(Nm, 0.0);
  int k = 0;
  for (int i = 0; i < Nend; ++i, k++) rS[k + 1] = rS[k] + dSref + (dSmid - dSref) * i / ((double)Nend - 1.);
  for (int i = 0; i < Nmid; ++i, k++) rS[k + 1] = rS[k] + dSmid;
  for (int i = 0; i < Nend; ++i, k++)
    rS[k + 1] = rS[k] + dSref + (dSmid - dSref) * (Nend - i - 1) / ((double)Nend - 1.);
  rS[k] = std::min(rS[k], L);
  width.assign(Nm, 0.0);
  for (int i = 0; i < Nm; i++) {
    const double s = rS[i];
    const double sb = .04 * L, st = .95 * L, wt = .01 * L, wh = .04 * L;
    double w;
    if (s < 0 or s > L) w = 0;
    else w = (s < sb ? std::sqrt(2 * wh * s - s * s) : (s < st ? wh - (wh - wt) * ((s - sb) / (st - sb)) : (wt * (L - s) / (L - st))));
    width[i] = w;
  }
  return true;
}

int upload_shapes(cup2d_ctx* ctx) {
  Ctx& c = ctx->c;
  if (c.nshapes == 0) return CUP2D_OK;
  CK(cudaMemcpyAsync(c.dshapes, c.hshapes.data(), sizeof(DevShape) * c.nshapes, cudaMemcpyHostToDevice, c.stream));
  return CUP2D_OK;
}

int upload_scalars_reset(cup2d_ctx* ctx) {
  Ctx& c = ctx->c;
  Scalars s{};
  s.time = 0; s.dt = 0; s.uinfx = 0; s.uinfy = 0; s.lambda = c.cfg.lambda;
  s.step = 0; s.status = 0;
  s.it.relDF = 0; s.it.target = 1e-4; s.it.oldNsteps = 10000; s.it.last = 0;   // PressureIterator_unif.h:15-16
  for (int i = 0; i < 100; i++) {        // Simulation.cpp:266-267, evaluated with the host libm
    const double x = (i + 1.0) / 100;
    s.rampCFL[i] = std::exp(std::log(1e-3) * (1 - x) + std::log(c.cfg.CFL) * x);
  }
  CK(cudaMemcpyAsync(c.dsc, &s, sizeof(Scalars), cudaMemcpyHostToDevice, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  return CUP2D_OK;
}

void invalidate_graph(Ctx& c) {
  if (c.graph) { cudaGraphExecDestroy(c.graph); c.graph = nullptr; }
  c.graphGen++;                             // ensembles holding this context re-capture
}

// one pass of Simulation::simulate's loop body (Simulation.cpp:245-251)
// Routes the launches of one scope to another stream (graph branch).
struct StreamScope {
  Ctx& c; cudaStream_t saved;
  StreamScope(Ctx& cc, cudaStream_t s) : c(cc), saved(cc.stream) { c.stream = s; }
  ~StreamScope() { c.stream = saved; }
};

// PressureSingle.cpp:216-241 and 362-372: the pressure correction and the
// momentum integrals run side by side (the integrals evaluate the corrected
// velocity of their own cells), then collisions and penalization.  The
// integrals, the longer of the two, stay on the main stream.
void launch_pressure_tail(Ctx& c, bool maxNext) {
  const double* ui = c.u();
  const double* vi = c.v();
  if (c.nshapes == 0) {
    launch_pcorr(c, maxNext);                // with the next step's findMaxU
    return;
  }
  cudaEventRecord(c.evPres, c.stream);
  cudaStreamWaitEvent(c.side2, c.evPres, 0);
  {
    StreamScope scope(c, c.side2);
    launch_pcorr(c, maxNext);                // flips the current velocity buffer
  }
  cudaEventRecord(c.evMom, c.side2);
  launch_momenta(c, ui, vi);
  cudaStreamWaitEvent(c.stream, c.evMom, 0);
  launch_collide_penalize(c);
}

// One pass of Simulation::simulate's loop body (Simulation.cpp:245-251) as a
// graph with three branches:
//   main : dt + reset of last step's tiles + body motion -> fish frames and
//          tile search, rasters, Towers chi with the moments -> [join side2] -> RHS
//          obstacle terms, Poisson -> momentum integrals [beside the
//          pressure correction on side2] -> collisions, penalization, forces
//          -> [join side, side2] -> t += dt and the next step's dt
//   side : the fish midlines of the next step (they depend on time only):
//          from the graph's start when the step's dt was carried, else
//          once step_begin has set it
//   side2: once the tiles are placed, advDiff's outflow flux, then advDiff
//          with the RHS divergence in place (advDiff reads no obstacle data);
//          later the pressure correction (with the next step's findMaxU
//          over the blocks without obstacle tiles; the tiles' part follows
//          the penalization on main)
void enqueue_step(Ctx& c) {
  struct GraphStepFlag { Ctx& c; explicit GraphStepFlag(Ctx& cc) : c(cc) { c.graphStep = true; }
                         ~GraphStepFlag() { c.graphStep = false; } } flag(c);
  bool anyFish = false, anyAhead = false;
  for (int k = 0; k < c.nshapes; k++) {
    anyFish |= c.hshapes[k].cfg.kind != CUP2D_SHAPE_DISK;
    anyAhead |= midline_ahead(c, k);
  }
  if (anyAhead) {
    // the next step's midlines depend on time only: with a carried dt they
    // start with the graph, beside the step's own start
    cudaEventRecord(c.evStart, c.stream);
    cudaStreamWaitEvent(c.side, c.evStart, 0);
    for (int k = 0; k < c.nshapes; k++)
      if (midline_ahead(c, k)) launch_fish_midline(c, k, c.side, 2);
  }
  launch_step_begin(c);                     // dt, last step's tiles reset, body motion
  cudaEventRecord(c.evFork, c.stream);
  if (anyAhead) {
    // otherwise once the step has its dt
    cudaStreamWaitEvent(c.side, c.evFork, 0);
    for (int k = 0; k < c.nshapes; k++)
      if (midline_ahead(c, k)) launch_fish_midline(c, k, c.side, 3);
    cudaEventRecord(c.evJoin, c.side);
  }
  // a swimmer under PID control forms its midline within the step, after
  // the controller has run (StefanFish::create)
  for (int k = 0; k < c.nshapes; k++)
    if (midline_in_step(c, k)) launch_fish_midline(c, k, c.stream, 0);
  // the obstacle chain, the step's critical path, stays on the main stream
  // (programmatic launches chain only within a stream)
  // advDiff and the RHS divergence beside the obstacle chain: with a fish,
  // once the tiles are placed -- the fish frame is a single-CTA latency chain
  // that any kernel beside it slows (measured: even the 12-CTA outflow flux),
  // while the rasters after it leave most SMs free; with disks only, from
  // the step's start (advDiff reads no obstacle data)
  c.recordPlaced = anyFish;
  if (!c.recordPlaced) cudaEventRecord(c.evPlaced, c.stream);
  launch_objects_rest(c);
  c.recordPlaced = false;
  cudaStreamWaitEvent(c.side2, c.evPlaced, 0);
  {
    StreamScope scope(c, c.side2);
    launch_outflow_flux(c);
    launch_advdiff_rhs_div(c);              // the update with the flux's correction, then the RHS
  }
  cudaEventRecord(c.evObjDone, c.side2);
  cudaStreamWaitEvent(c.stream, c.evObjDone, 0);
  launch_rhs_obstacles(c);
  poisson_solve(c);
  launch_pressure_tail(c, true);
  launch_forces(c, c.forcesOut, true);
  if (anyAhead) cudaStreamWaitEvent(c.stream, c.evJoin, 0);
  launch_end_step_dt(c);                    // t += dt, and the next step's dt
}

// PressureIterator_unif::operator() (PressureIterator_unif.cpp:214-270): the
// velocity after advDiff kept as TMPV, then per iteration the fluid velocity
// UF = TMPV - (dt/2h) grad P (P of the previous iteration, or step), the
// bodies' momenta on UF and their velocities, the penalization of the
// velocity towards the bodies' with its relative momentum change, the RHS
// div V - chi div UDEF and a Poisson solve; converged (the change below the
// adaptive target, or more than 100 iterations, or more than twice the
// previous call's count), V -= (dt/2h) grad P.  The target then adapts to
// the count as in the reference.  The change is read back each iteration.
int pressure_iterative(cup2d_ctx* ctx) {
  Ctx& c = ctx->c;
  const size_t nb = sizeof(double) * c.ncells();
  CK(cudaMemcpyAsync(c.itmp[0], c.u(), nb, cudaMemcpyDeviceToDevice, c.stream));
  CK(cudaMemcpyAsync(c.itmp[1], c.v(), nb, cudaMemcpyDeviceToDevice, c.stream));
  CK(cudaMemcpyAsync(&c.pin->it, &c.dsc->it, sizeof(IterState), cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  IterState st = c.pin->it;
  int iter = 0;
  double relDF = 1e3;
  for (iter = 0; iter < 1000; iter++) {
    launch_pcorr_from(c, c.itmp[0], c.itmp[1], c.ifluid[0], c.ifluid[1]);
    launch_momenta_iter(c, c.itmp[0], c.itmp[1]);    // UF's values, formed in place
    launch_penalize_iter(c, c.itmp[0], c.itmp[1], c.ifluid[0], c.ifluid[1]);
    launch_rhs_iter(c);
    poisson_solve(c);
    CK(cudaMemcpyAsync(&c.pin->it.relDF, &c.dsc->it.relDF, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    if (int rc = check_launch(ctx)) return rc;
    relDF = c.pin->it.relDF;
    if (relDF < st.target || iter > 100 || iter > 2 * st.oldNsteps) {
      launch_pcorr(c);                          // finalizePressure
      break;
    }
  }
  st.oldNsteps = iter + 1;
  if (st.oldNsteps > 30) st.target = std::max(relDF, st.target);
  if (st.oldNsteps > 10) st.target *= 1.01;
  if (st.oldNsteps <= 2) st.target *= 0.99;
  st.target = std::min(1e-3, std::max(1e-5, st.target));
  st.relDF = relDF;
  st.last = iter + 1;
  launch_set_iter_state(c, st);
  return check_launch(ctx);
}

// PressureVarRho_approx::operator() (PressureIterator_approx.cpp:378-468):
// pressureCorrectionInit (vFluid from the last pressure, the velocity part
// of the RHS, F = 0, uDef cleared), then per iteration the bodies' momenta
// on vFluid and their velocities, the penalization force F with its
// relative change relDF, the RHS, a Poisson solve into tmp (the RHS
// buffer, as solve(tmp, tmp)), the pressure correction of vFluid with the
// relative pressure change relDP; converged (max(relDF, relDP) below the
// adaptive target, or more than 100 iterations, or more than twice the
// previous call's count), finalizePressure updates the velocity; each
// iteration ends with pres = tmp (the two buffers trade places; the next
// RHS overwrites tmp), and the call with tmp = pres, as the reference leaves
// them.  The target adapts as in the reference.
}  // namespace
cudaError_t fill_udef_grid(Ctx& c);
namespace {
int pressure_varrho(cup2d_ctx* ctx) {
  Ctx& c = ctx->c;
  const size_t nb = sizeof(double) * c.ncells();
  CK(cudaMemcpyAsync(&c.pin->it, &c.dsc->it, sizeof(IterState), cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  IterState st = c.pin->it;
  if (c.udefStale) CK(fill_udef_grid(c));
  launch_vr_init(c);
  CK(cudaMemsetAsync(c.udefx, 0, nb, c.stream));
  CK(cudaMemsetAsync(c.udefy, 0, nb, c.stream));
  int iter = 0;
  double relDF = 1e3, relDP = 1e3;
  for (iter = 0; iter < 1000; iter++) {
    launch_momenta_varrho(c, c.ifluid[0], c.ifluid[1]);
    launch_vr_penalize(c);
    launch_vr_rhs(c);
    double* const P = c.pres;
    c.pres = c.rhs;                               // solve(tmp, tmp)
    poisson_solve(c);
    c.pres = P;
    launch_vr_pcorr(c, false);
    CK(cudaMemcpyAsync(&c.pin->it, &c.dsc->it, sizeof(IterState), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    if (int rc = check_launch(ctx)) return rc;
    relDF = c.pin->it.relDF;
    relDP = c.pin->it.relDP;
    const bool converged = std::max(relDF, relDP) < st.target || iter > 2 * st.oldNsteps || iter > 100;
    if (converged) launch_vr_pcorr(c, true);     // finalizePressure
    std::swap(c.pres, c.rhs);                     // pres = tmp
    if (converged) break;
  }
  CK(cudaMemcpyAsync(c.rhs, c.pres, nb, cudaMemcpyDeviceToDevice, c.stream));
  st.oldNsteps = iter + 1;
  if (st.oldNsteps > 30) st.target = std::max({relDF, relDP, st.target});
  if (st.oldNsteps > 10) st.target *= 1.01;
  if (st.oldNsteps <= 2) st.target *= 0.99;
  st.target = std::min(1e-3, std::max(1e-5, st.target));
  st.relDF = relDF;
  st.relDP = relDP;
  st.last = iter + 1;
  launch_set_iter_state(c, st);
  c.udefStale = false;                          // cleared by pressureCorrectionInit
  return check_launch(ctx);
}

} // namespace

// The graph step's calcMaxTimestep reuses the maximum formed at the end of
// the previous graph step only while nothing else has touched the state.
cudaError_t invalidate_dt_next(Ctx& c) {
  if (!c.dtValidMaybe) return cudaSuccess;
  c.dtValidMaybe = c.dtCarried = false;
  return cudaMemsetAsync(&c.dsc->dtNextValid, 0, sizeof(int), c.stream);
}

// An ABI call outside the operator sequence: the in-place RHS and the
// placement mark no longer describe the state the next stage sees.
void forget_chain(Ctx& c) { c.rhsFresh = false; c.placedPending = false; c.maxNextState = 0; }

// PutObjectsOnGrid.cpp:195 and 149-184: uDef cleared, then every shape's
// deformation velocity added where its chi is the grid's, from the tiles of
// the last placement (their udef is final once removeMoments has run).
cudaError_t fill_udef_grid(Ctx& c) {
  cudaError_t e = cudaMemsetAsync(c.udefx, 0, sizeof(double) * c.ncells(), c.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c.udefy, 0, sizeof(double) * c.ncells(), c.stream);
  if (e != cudaSuccess) return e;
  launch_obj_vel_on_grid(c);
  c.udefStale = false;
  return cudaGetLastError();
}

bool same_bits(double a, double b) { return std::memcmp(&a, &b, sizeof(double)) == 0; }

extern "C" {

int cup2d_config_default(cup2d_config* cfg) {
  if (!cfg) return CUP2D_EINVAL;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->bpdx = 0; cfg->bpdy = 0;
  cfg->extent = 1;
  cfg->CFL = 0.1;
  cfg->lambda = 1e3 / cfg->CFL;
  cfg->dlm = 0;
  cfg->nu = 1e-2;
  cfg->fadeLen = 0.01;
  cfg->nsteps = 0; cfg->tend = 0;
  cfg->poisson = CUP2D_POISSON_COSINE;   // -poissonType "" selects FFTW_dirichlet
  cfg->precision = CUP2D_PREC_FP64;
  cfg->device = 0;
  cfg->gravity[0] = 0; cfg->gravity[1] = -9.8;      // SimulationData.h:57
  return CUP2D_OK;
}

namespace {
thread_local std::string g_createErr;   // why this thread's last cup2d_create failed
int create_fail(int code, const std::string& msg) { g_createErr = msg; return code; }
}

const char* cup2d_last_error(const cup2d_ctx* ctx) {
  return ctx ? ctx->c.err.c_str() : g_createErr.c_str();
}

int cup2d_create(const cup2d_config* cfg, cup2d_ctx** out) {
  if (!cfg || !out) return create_fail(CUP2D_EINVAL, "null argument");
  *out = nullptr;
  g_createErr.clear();
  if (cfg->bpdx <= 0 || cfg->bpdy <= 0) return create_fail(CUP2D_EINVAL, "bpdx and bpdy must be positive");
  // CUP2D_PREC_FP32: the free-space and periodic Poisson transforms in FP32
  // (fields, stencils, obstacle sums and forces stay FP64); the cosine solver
  // has FP64 transforms only
  if (cfg->precision != CUP2D_PREC_FP64 && cfg->precision != CUP2D_PREC_FP32)
    return create_fail(CUP2D_ENOTSUP, "unknown precision");
  if (cfg->precision == CUP2D_PREC_FP32 && cfg->poisson == CUP2D_POISSON_COSINE)
    return create_fail(CUP2D_ENOTSUP, "the cosine solver has FP64 transforms only");
  if (!poisson_size_ok(cfg->poisson, 32 * cfg->bpdx, 32 * cfg->bpdy))
    return create_fail(CUP2D_ENOTSUP, poisson_size_limits(cfg->poisson));
  cup2d_ctx* ctx = new (std::nothrow) cup2d_ctx();
  if (!ctx) return CUP2D_ENOMEM;
  Ctx& c = ctx->c;
  c.cfg = *cfg;
  c.device = cfg->device;
  if (cudaSetDevice(c.device) != cudaSuccess) { delete ctx; return CUP2D_ECUDA; }
  cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, c.device);
  if (c.sms <= 0) c.sms = 1;
  // the main stream carries the step's critical path (the obstacle chain):
  // its CTAs go first when side-branch kernels compete for the SMs (graph
  // kernel nodes keep the stream priority)
  int prLeast = 0, prGreatest = 0;
  cudaDeviceGetStreamPriorityRange(&prLeast, &prGreatest);
  if (cudaStreamCreateWithPriority(&c.stream, cudaStreamNonBlocking, prGreatest) != cudaSuccess) {
    delete ctx; return CUP2D_ECUDA;
  }
  GridDesc& g = c.g;
  g.bpdx = cfg->bpdx; g.bpdy = cfg->bpdy;
  g.nx = BS * g.bpdx; g.ny = BS * g.bpdy; g.nblocks = g.bpdx * g.bpdy;
  g.extent = cfg->extent;
  g.h = cfg->extent / std::max(g.bpdx * BS, g.bpdy * BS);     // Cubism Grid spacing
  g.ext[0] = g.bpdx * g.h * BS;                                // SimulationData.cpp:34-35
  g.ext[1] = g.bpdy * g.h * BS;
  g.nu = cfg->nu; g.CFL = cfg->CFL; g.dlm = cfg->dlm;
  g.fadeLenX = cfg->fadeLen * cfg->extent;                     // Simulation.cpp:97-98
  g.fadeLenY = cfg->fadeLen * cfg->extent;
  g.implicitPenal = cfg->implicit_penalization ? 1 : 0;
  const size_t n = c.ncells();
  int rc = CUP2D_OK;
  for (int b = 0; b < 2 && !rc; b++)
    for (int d = 0; d < 2 && !rc; d++) rc = dalloc(ctx, &c.vel[b][d], n);
  if (!rc) rc = dalloc(ctx, &c.chi, n);
  if (!rc) rc = dalloc(ctx, &c.pres, n);
  if (!rc) rc = dalloc(ctx, &c.rhs, n);
  if (!rc) rc = dalloc(ctx, &c.sdf, n);
  if (!rc) rc = dalloc(ctx, &c.udefx, n);
  if (!rc) rc = dalloc(ctx, &c.udefy, n);
  for (int d = 0; d < 2 && !rc && cfg->iterative; d++) {
    rc = dalloc(ctx, &c.itmp[d], n);
    if (!rc) rc = dalloc(ctx, &c.ifluid[d], n);
  }
  for (int b = 0; b < 2 && !rc; b++)
    for (int d = 0; d < 2 && !rc; d++)
      if (make_tmap_f64(&c.tmVel[b][d], c.vel[b][d], g.nx, g.ny, ADV_HT, ADV_HT) != cudaSuccess)
        rc = fail(ctx, CUP2D_ECUDA, "TMA tensor maps of the velocity planes could not be made");
  c.advTx = 2u * ADV_HT * ADV_HT * sizeof(double);
  if (const char* inj = std::getenv("CUP2D_FAULT_TMA_WAIT"))      // fault injection (cup2d.h)
    if (std::atoi(inj) != 0) c.advTx += 16;
  if (!rc) rc = dalloc(ctx, &c.dsc, 1);
  if (!rc) rc = dalloc(ctx, &c.dshapes, MAX_SHAPES);
  if (!rc) rc = dalloc(ctx, &c.counters, Ctx::NCOUNTERS);
  if (!rc && (cudaStreamCreateWithFlags(&c.side, cudaStreamNonBlocking) != cudaSuccess ||
              cudaStreamCreateWithFlags(&c.side2, cudaStreamNonBlocking) != cudaSuccess ||
              cudaEventCreateWithFlags(&c.evFork, cudaEventDisableTiming) != cudaSuccess ||
              cudaEventCreateWithFlags(&c.evStart, cudaEventDisableTiming) != cudaSuccess ||
              cudaEventCreateWithFlags(&c.evSideMid, cudaEventDisableTiming) != cudaSuccess ||
              cudaEventCreateWithFlags(&c.evDtNext, cudaEventDisableTiming) != cudaSuccess ||
              cudaEventCreateWithFlags(&c.evShapes, cudaEventDisableTiming) != cudaSuccess ||
              cudaMallocHost(&c.pin, sizeof(Ctx::HostPin)) != cudaSuccess ||
              cudaHostAlloc(&c.map, sizeof(Ctx::HostMapped), cudaHostAllocMapped) != cudaSuccess ||
              cudaHostGetDevicePointer(&c.mapDev, c.map, 0) != cudaSuccess ||
              cudaEventCreateWithFlags(&c.evForces, cudaEventDisableTiming) != cudaSuccess ||
              cudaEventCreateWithFlags(&c.evJoin, cudaEventDisableTiming) != cudaSuccess ||
              cudaEventCreateWithFlags(&c.evObj, cudaEventDisableTiming) != cudaSuccess ||
              cudaEventCreateWithFlags(&c.evObjDone, cudaEventDisableTiming) != cudaSuccess ||
              cudaEventCreateWithFlags(&c.evPres, cudaEventDisableTiming) != cudaSuccess ||
              cudaEventCreateWithFlags(&c.evMom, cudaEventDisableTiming) != cudaSuccess ||
              cudaEventCreateWithFlags(&c.evPlaced, cudaEventDisableTiming) != cudaSuccess))
    rc = fail(ctx, CUP2D_ECUDA, "stream/event creation failed");
  if (!rc && fish_setup_kernels() != cudaSuccess)
    rc = fail(ctx, CUP2D_ECUDA, "shared-memory limits of the fish kernels could not be set");
  if (rc) { cup2d_destroy(ctx); return rc; }
  std::memset(c.map, 0, sizeof(Ctx::HostMapped));     // the signal words start below every launch's value
  if (cudaMemsetAsync(c.counters, 0, sizeof(unsigned) * Ctx::NCOUNTERS, c.stream) != cudaSuccess ||
      cudaStreamSynchronize(c.stream) != cudaSuccess) { cup2d_destroy(ctx); return CUP2D_ECUDA; }
  c.poisson = poisson_create(c);
  if (!c.poisson) { cup2d_destroy(ctx); return create_fail(CUP2D_ENOMEM, "Poisson solver set-up failed"); }
  if (cfg->autotune && poisson_autotune(c) != cudaSuccess) {
    cup2d_destroy(ctx); return create_fail(CUP2D_ECUDA, "transform autotuning failed");
  }
  if (cudaStreamSynchronize(c.stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    cup2d_destroy(ctx); return CUP2D_ECUDA;
  }
  *out = ctx;
  return CUP2D_OK;
}

int cup2d_destroy(cup2d_ctx* ctx) {
  if (!ctx) return CUP2D_OK;
  Ctx& c = ctx->c;
  for (cup2d_ctx* sh : c.gaitShadows) cup2d_destroy(sh);
  c.gaitShadows.clear();
  if (c.stream) cudaStreamSynchronize(c.stream);
  invalidate_graph(c);
  for (int b = 0; b < 2; b++) for (int d = 0; d < 2; d++) cudaFree(c.vel[b][d]);
  cudaFree(c.chi); cudaFree(c.pres); cudaFree(c.rhs); cudaFree(c.sdf);
  cudaFree(c.udefx); cudaFree(c.udefy); cudaFree(c.dsc); cudaFree(c.dshapes);
  for (int d = 0; d < 2; d++) { cudaFree(c.itmp[d]); cudaFree(c.ifluid[d]); }
  cudaFree(c.invRho); cudaFree(c.prhs);
  cudaFree(c.counters); cudaFree(c.partials); cudaFree(c.fadeSlot);
  if (c.flushBuf) cudaFree(c.flushBuf);
  if (c.hashAcc) cudaFree(c.hashAcc);
  if (c.side) cudaStreamDestroy(c.side);
  if (c.side2) cudaStreamDestroy(c.side2);
  if (c.evObj) cudaEventDestroy(c.evObj);
  if (c.evObjDone) cudaEventDestroy(c.evObjDone);
  if (c.evFork) cudaEventDestroy(c.evFork);
  if (c.evStart) cudaEventDestroy(c.evStart);
  if (c.evSideMid) cudaEventDestroy(c.evSideMid);
  if (c.evDtNext) cudaEventDestroy(c.evDtNext);
  if (c.evShapes) cudaEventDestroy(c.evShapes);
  if (c.pin) cudaFreeHost(c.pin);
  if (c.map) cudaFreeHost(c.map);
  if (c.evForces) cudaEventDestroy(c.evForces);
  if (c.evJoin) cudaEventDestroy(c.evJoin);
  if (c.evPres) cudaEventDestroy(c.evPres);
  if (c.evMom) cudaEventDestroy(c.evMom);
  if (c.evPlaced) cudaEventDestroy(c.evPlaced);
  for (auto& t : c.tiles) {
    cudaFree(t.tiles); cudaFree(t.slot); cudaFree(t.chi); cudaFree(t.dist); cudaFree(t.udx);
    cudaFree(t.udy); cudaFree(t.sD); cudaFree(t.sdx); cudaFree(t.sdy);
  }
  for (auto& f : c.fish) {
    cudaFree(f.pool); cudaFree(f.seg); cudaFree(f.nw); cudaFree(f.off);
    cudaFree(f.ipIdx);
  }
  poisson_destroy(c.poisson);
  if (c.stream) cudaStreamDestroy(c.stream);
  delete ctx;
  return CUP2D_OK;
}

int cup2d_shape_params_default(cup2d_shape_params* p) {
  if (!p) return CUP2D_EINVAL;
  std::memset(p, 0, sizeof(*p));
  p->xpos = -1; p->ypos = -1;     // -1: centre of the domain (Simulation.cpp:132-135)
  p->angle = 0; p->rhoS = 1;
  p->bFixed = 0; p->bFixedx = -1; p->bFixedy = -1;
  p->bForced = 0; p->bForcedx = -1; p->bForcedy = -1; p->bBlockAng = -1;
  p->xvel = 0; p->yvel = 0; p->angvel = 0;
  p->timeForced = DBL_MAX;
  p->radius = 0.1; p->tAccel = -1;
  p->L = 0.1; p->T = 1; p->phi = 0; p->amplitudeFactor = 1;
  return CUP2D_OK;
}

int cup2d_add_shape(cup2d_ctx* ctx, int kind, const cup2d_shape_params* p, int* id) {
  if (!ctx || !p) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  if (c.initialised) return fail(ctx, CUP2D_ESTATE, "shapes must be added before cup2d_init");
  if (c.nshapes >= MAX_SHAPES) return fail(ctx, CUP2D_EINVAL, "too many shapes");
  if (kind != CUP2D_SHAPE_DISK && kind != CUP2D_SHAPE_STEFANFISH && kind != CUP2D_SHAPE_CARLINGFISH &&
      kind != CUP2D_SHAPE_ENVELOPEFISH)
    return fail(ctx, CUP2D_ENOTSUP, "unknown shape kind");
  // Shape::bVariableDensity (Shape.cpp:21-23) selects the variable-density
  // pipeline (Simulation.cpp:185-204): advDiffGrav + PressureVarRho_approx
  // with -iterativePenalization, else PressureVarRho_proper (HYPRE)
  if (std::fabs(p->rhoS - 1.0) > DBL_EPSILON && !c.cfg.iterative)
    return fail(ctx, CUP2D_ENOTSUP, "rhoS != 1 without -iterativePenalization selects PressureVarRho_proper, "
                                    "a HYPRE solver (Simulation.cpp:194-199): set iterative");
  if (!(p->rhoS > 0)) return fail(ctx, CUP2D_EINVAL, "rhoS must be positive");
  DevShape S{};
  ShapeCfg& f = S.cfg;
  f.kind = kind;
  f.rhoS = p->rhoS;
  const int bFixed = p->bFixed != 0, bForced = p->bForced != 0;
  f.bFixedx = p->bFixedx < 0 ? bFixed : p->bFixedx != 0;      // Shape.cpp:335-341
  f.bFixedy = p->bFixedy < 0 ? bFixed : p->bFixedy != 0;
  f.bForcedx = p->bForcedx < 0 ? bForced : p->bForcedx != 0;
  f.bForcedy = p->bForcedy < 0 ? bForced : p->bForcedy != 0;
  f.bBlockang = p->bBlockAng < 0 ? (f.bForcedx || f.bForcedy) : p->bBlockAng != 0;
  f.forcedu = -p->xvel; f.forcedv = -p->yvel; f.forcedomega = -p->angvel;
  f.timeForced = p->timeForced;
  f.origC[0] = p->xpos < 0 ? .5 * c.g.ext[0] : p->xpos;
  f.origC[1] = p->ypos < 0 ? .5 * c.g.ext[1] : p->ypos;
  f.origAng = p->angle * M_PI / 180;
  f.radius = p->radius; f.tAccel = p->tAccel;
  f.length = p->L; f.Tperiod = p->T; f.phaseShift = p->phi; f.ampFac = p->amplitudeFactor;
  for (double& x : f.curvScale) x = 1;
  for (double& x : f.envFourier) x = 1;
  const bool curvatureFish = kind == CUP2D_SHAPE_STEFANFISH || kind == CUP2D_SHAPE_ENVELOPEFISH;
  f.pid = curvatureFish && p->pid != 0;             // other shapes ignore -pid (StefanFish.cpp:209-211)
  f.pidpos = curvatureFish && p->pidpos != 0;
  const double h = c.g.h;
  double span;
  if (kind == CUP2D_SHAPE_DISK) span = 2 * (f.radius + 2 * h);
  else span = 2 * (1.2 * f.length + 8 * h);
  int nb1 = (int)std::ceil(span / (BS * h)) + 2;
  int cap = nb1 * nb1;
  if (cap > c.g.nblocks) cap = c.g.nblocks;
  // fault injection on the host: a smaller tile capacity makes a body
  // overflow it, which the tile search reports as CUP2D_ECAPACITY
  if (const char* inj = std::getenv("CUP2D_FAULT_TILE_CAPACITY")) {
    const int v = std::atoi(inj);
    if (v > 0 && v < cap) cap = v;
  }
  f.capacity = cap;
  S.rhoTile = kind == CUP2D_SHAPE_DISK ? f.rhoS : 1.0;
  ObstTiles t{};
  t.capacity = cap;
  int rc = dalloc(ctx, &t.tiles, cap);
  if (!rc) rc = dalloc(ctx, &t.slot, c.g.nblocks);
  double** arrs[] = {&t.chi, &t.dist, &t.udx, &t.udy, &t.sD, &t.sdx, &t.sdy};
  for (auto a : arrs) if (!rc) rc = dalloc(ctx, a, (size_t)cap * BS2);
  if (rc) return rc;
  CK(cudaMemsetAsync(t.slot, 0xff, sizeof(int) * c.g.nblocks, c.stream));
  FishArrays F{};
  if (kind != CUP2D_SHAPE_DISK) {
    std::vector<double> rS, width;
    if (!fish_grid(f.length, h, rS, width))
      return fail(ctx, CUP2D_EINVAL, "fish midline spacing degenerate at this resolution (dSref <= 0, FishLibrary.cpp:21)");
    const int Nm = (int)rS.size();
    f.nm = Nm;
    F.nm = Nm; F.nseg = (Nm - 1) / 8;
    if (!fish_fits_on_chip(Nm, F.nseg, c.device))
      return fail(ctx, CUP2D_ENOTSUP, "fish midline too fine: its kernels' staged arrays exceed shared memory");
    // 3 static arrays + 3 midlines of 8 arrays + 16 integrals, one allocation
    if (!rc) rc = dalloc(ctx, &F.pool, fish_pool_len(Nm));
    if (!rc) rc = dalloc(ctx, &F.seg, F.nseg);
    if (rc) return rc;
    {
      double* q = F.pool;
      F.rS = q; q += Nm; F.width = q; q += Nm; F.p1f = q; q += Nm; F.w3 = q; q += Nm;
      FishMidline* mids[3] = {&F.mid[0], &F.mid[1], &F.frame};
      for (FishMidline* m : mids) {
        double** a[8] = {&m->rX, &m->rY, &m->vX, &m->vY, &m->norX, &m->norY, &m->vNorX, &m->vNorY};
        for (auto x : a) { *x = q; q += Nm; }
      }
      F.integ = q; q += 16;
      for (int b = 0; b < 2; b++) {
        FishMidline* m = &F.mid[b];
        double** a[4] = {&m->uX, &m->uY, &m->lX, &m->lY};
        for (auto x : a) { *x = q; q += Nm; }
      }
      F.frame.uX = F.frame.uY = F.frame.lX = F.frame.lY = nullptr;
    }
    // no midline formed yet: integrals (with their time) NaN (all-ones bytes)
    CK(cudaMemsetAsync(F.integ, 0xff, sizeof(double) * 16, c.stream));
    // interior-point layout of PutFishOnBlocks::constructInternl
    // (FishLibrary.cpp:594-596): Nw = floor(width/h) points each side
    std::vector<int> nw(Nm), off(Nm + 1, 0);
    for (int i = 0; i < Nm; i++) {
      nw[i] = (int)std::floor(width[i] / h);
      off[i + 1] = off[i] + (nw[i] > 0 ? 2 * nw[i] - 1 : 0);
    }
    F.nint = off[Nm];
    if (!rc) rc = dalloc(ctx, &F.nw, Nm);
    if (!rc) rc = dalloc(ctx, &F.off, Nm + 1);
    if (!rc) rc = dalloc(ctx, &F.ipIdx, (size_t)F.nint);
    if (rc) return rc;
    std::vector<int2> ipIdx(F.nint);
    for (int i = 0; i < Nm; i++)
      for (int j = 0; j < (nw[i] > 0 ? 2 * nw[i] - 1 : 0); j++) ipIdx[off[i] + j] = make_int2(i, -nw[i] + 1 + j);
    CK(h2d_sync(F.ipIdx, ipIdx.data(), sizeof(int2) * F.nint, c.stream));
    CK(h2d_sync(F.nw, nw.data(), sizeof(int) * Nm, c.stream));
    CK(h2d_sync(F.off, off.data(), sizeof(int) * (Nm + 1), c.stream));
    const std::vector<double> p1f = curvature_profile(f, rS);
    CK(h2d_sync(F.rS, rS.data(), sizeof(double) * Nm, c.stream));
    CK(h2d_sync(F.width, width.data(), sizeof(double) * Nm, c.stream));
    CK(h2d_sync(F.p1f, p1f.data(), sizeof(double) * Nm, c.stream));
    CK(fish_width_cubes(F, c.stream));
    CK(cudaStreamSynchronize(c.stream));
  }
  c.hshapes.push_back(S);
  c.shapeParams.push_back(*p);
  c.shapeKinds.push_back(kind);
  c.tiles.push_back(t);
  c.fish.push_back(F);
  if (id) *id = c.nshapes;
  c.nshapes++;
  if (cap > c.maxCapacity) c.maxCapacity = cap;
  return CUP2D_OK;
}

int cup2d_init(cup2d_ctx* ctx) {
  if (!ctx) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  if (c.nshapes == 0) return fail(ctx, CUP2D_EINVAL, "no shapes (Simulation.cpp:167-169)");
  invalidate_graph(c);
  // reduction scratch: dense region + per-shape tile regions
  cudaFree(c.partials);
  c.npartials = (size_t)3 * c.g.nblocks + 4096 + (size_t)MAX_SHAPES * c.maxCapacity * 24;
  int rc = dalloc(ctx, &c.partials, c.npartials);
  if (rc) return rc;
  cudaFree(c.fadeSlot);
  c.fadeSlot = nullptr;
  if ((rc = dalloc(ctx, &c.fadeSlot, (size_t)c.g.nblocks + 1))) return rc;
  if ((c.nfade = build_fade_slots(c)) < 0) return fail(ctx, CUP2D_ECUDA, "fade strip table");
  // SimulationData::checkVariableDensity and minRho (SimulationData.cpp:116-130)
  c.varRho = false;
  c.rho0 = 1;
  for (int k = 0; k < c.nshapes; k++) {
    const double r = c.hshapes[k].cfg.rhoS;
    c.varRho |= std::fabs(r - 1.0) > DBL_EPSILON;
    c.rho0 = std::min(c.rho0, r);
  }
  if (c.varRho && !c.invRho) {
    if ((rc = dalloc(ctx, &c.invRho, c.ncells()))) return rc;
    if ((rc = dalloc(ctx, &c.prhs, c.ncells()))) return rc;
  }
  c.cur = 0;
  // Simulation::reset (Simulation.cpp:232-241): resetAll, IC, objects at t=0, ApplyObjVel
  if ((rc = upload_scalars_reset(ctx))) return rc;
  c.dtValidMaybe = c.dtCarried = false;
  c.shapesAtEvent = c.shapesMapped = false;
  c.stateSeq++;
  forget_chain(c);
  for (int k = 0; k < c.nshapes; k++) {
    DevShape& S = c.hshapes[k];
    const ShapeCfg& f = S.cfg;
    std::memset(&S.s, 0, sizeof(S.s));
    std::memset(&S.f, 0, sizeof(S.f));
    std::memset(&S.ctl, 0, sizeof(S.ctl));        // CurvatureFish::resetAll (StefanFish.cpp:64-83)
    S.ctl.bendT0 = -1;                            // ParameterScheduler: t0 = -1, t1 = 0
    S.ctl.periodPIDval = f.Tperiod;
    S.s.center[0] = S.s.com[0] = f.origC[0];
    S.s.center[1] = S.s.com[1] = f.origC[1];
    S.s.orientation = f.origAng;
    S.s.u = f.forcedu; S.s.v = f.forcedv; S.s.omega = f.forcedomega;
    S.ntiles = 0; S.ntilesPrev = 0;
    CK(cudaMemsetAsync(c.tiles[k].slot, 0xff, sizeof(int) * c.g.nblocks, c.stream));
  }
  if ((rc = upload_shapes(ctx))) return rc;
  launch_ic(c);
  launch_set_dt(c, 0.0);
  c.devDt = 0.0;
  launch_objects(c, false);
  if (c.varRho) launch_invrho(c);
  launch_obj_vel_on_grid(c);
  c.udefStale = false;
  launch_apply_obj_vel(c);
  CK(cudaStreamSynchronize(c.stream));
  if ((rc = check_launch(ctx))) return rc;
  c.initialised = true;
  c.midByGraph = false;
  return CUP2D_OK;
}

int cup2d_tuning_get(cup2d_ctx* ctx, cup2d_tuning* out) {
  if (!ctx || !out) return CUP2D_EINVAL;
  poisson_tuning(ctx->c, out);
  return CUP2D_OK;
}

int cup2d_iteration_stats(cup2d_ctx* ctx, int* iterations, double* rel_df) {
  if (!ctx) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  if (!c.initialised) return fail(ctx, CUP2D_ESTATE, "not initialised");
  CK(cudaMemcpyAsync(&c.pin->it, &c.dsc->it, sizeof(IterState), cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  if (iterations) *iterations = c.pin->it.last;
  if (rel_df) *rel_df = c.pin->it.relDF;
  return CUP2D_OK;
}

// Waits for a kernel's signal in mapped host memory: the word reaches want
// (the kernel wrote its data first, behind a system-scope fence).  Spins on
// the word for up to 20 ms -- waking on it costs less than on the event --
// then waits on the event recorded after that kernel, which also reports
// an error of the stream (a kernel that never signals ends up there).
static cudaError_t wait_mapped(const unsigned long long* word, unsigned long long want, cudaEvent_t ev) {
  const volatile unsigned long long* w = word;
  const auto t0 = std::chrono::steady_clock::now();
  for (unsigned it = 0;; it++) {
    if (*w >= want) {
      std::atomic_thread_fence(std::memory_order_acquire);
      return cudaSuccess;
    }
    if ((it & 255) == 255 && std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(20)) break;
  }
  return cudaEventSynchronize(ev);
}

int cup2d_calc_dt(cup2d_ctx* ctx, double* dt_out) {
  if (!ctx || !ctx->c.initialised) return ctx ? fail(ctx, CUP2D_ESTATE, "not initialised") : CUP2D_EINVAL;
  Ctx& c = ctx->c;
  forget_chain(c);                          // sets sc->dt (and overwrites the grid partials)
  c.stateSeq++;
  if (c.dtCarried) {
    // formed by the last step end from this very state
    launch_take_dt_next(c);
    int rc = check_launch(ctx);
    if (rc) return rc;
    c.devDt = NAN;
    if (dt_out) {
      CK(wait_mapped(&c.map->seqDt, c.mapSeqDt, c.evDtNext));
      *dt_out = c.devDt = *(volatile const double*)&c.map->dtNext;
    }
    return CUP2D_OK;
  }
  launch_max_u_dt(c);
  int rc = check_launch(ctx);
  if (rc) return rc;
  c.devDt = NAN;
  if (dt_out) {
    CK(cudaMemcpyAsync(&c.pin->dt, &c.dsc->dt, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    *dt_out = c.devDt = c.pin->dt;
  }
  return CUP2D_OK;
}

// Every stage: the state changes (a carried dt no longer holds) and the
// stage's dt argument becomes sim.dt -- each launched only when the host
// mirrors say the device does not hold it already.  `prologueLaunched`:
// the stage enqueued work of its own before its body.
#define STAGE_PROLOGUE                                                           \
  if (!ctx) return CUP2D_EINVAL;                                                 \
  Ctx& c = ctx->c;                                                               \
  if (!c.initialised) return fail(ctx, CUP2D_ESTATE, "not initialised");         \
  c.shapesAtEvent = false;                                                       \
  c.shapesMapped = false;                                                        \
  c.stateSeq++;                                                                  \
  bool prologueLaunched = c.dtValidMaybe;                                        \
  CK(invalidate_dt_next(c));                                                     \
  if (dt >= 0 && !same_bits(dt, c.devDt)) {                                      \
    launch_set_dt(c, dt);                                                        \
    c.devDt = dt;                                                                \
    c.rhsFresh = false;                         /* the RHS scales with 1/dt */   \
    prologueLaunched = true;                                                     \
  }                                                                              \
  (void)prologueLaunched;

int cup2d_put_objects(cup2d_ctx* ctx, double dt) {
  STAGE_PROLOGUE
  forget_chain(c);
  // advDiff may start beside the obstacle chain once the tiles are placed
  // (with a fish) or right after the body motion (disks only), as in a
  // graph step
  bool anyFishShape = false;
  for (int k = 0; k < c.nshapes; k++) anyFishShape |= c.hshapes[k].cfg.kind != CUP2D_SHAPE_DISK;
  // the next step's midlines (time + dt) need only sim.dt: on the device
  // they may start from here, while the host launches them after this
  // step's chain (so that its first kernels are not delayed)
  if (anyFishShape) CK(cudaEventRecord(c.evFork, c.stream));
  launch_objects_begin(c, false);
  if (c.nshapes > 0) {
    c.recordPlaced = anyFishShape;
    if (!anyFishShape) CK(cudaEventRecord(c.evPlaced, c.stream));
    launch_objects_rest(c);
    c.recordPlaced = false;
  }
  if (c.nshapes == 0) CK(cudaMemsetAsync(&c.dsc->maxNext, 0, sizeof(double), c.stream));
  if (c.varRho) launch_invrho(c);            // PutObjectsOnGrid.cpp:65-73, 197
  if (c.cfg.iterative) {
    // PutObjectsOnGrid.cpp:195, 237-238: the grid's deformation velocity,
    // which the iterated operator's RHS reads
    CK(fill_udef_grid(c));
  } else {
    c.udefStale = c.nshapes > 0;            // filled when read (cup2d_get_field)
  }
  // the next step's midlines on the side stream, beside the rest of this
  // step; the next call takes them if the time matches
  bool anyAhead = false;
  for (int k = 0; k < c.nshapes; k++) anyAhead |= midline_ahead(c, k);
  if (anyAhead) {
    CK(cudaStreamWaitEvent(c.side, c.evFork, 0));
    for (int k = 0; k < c.nshapes; k++)
      if (midline_ahead(c, k)) launch_fish_midline(c, k, c.side, 1);
    CK(cudaEventRecord(c.evSideMid, c.side));
    c.sideMidPending = true;
  }
  c.midByGraph = false;
  c.placedPending = c.nshapes > 0;
  // k_obj_begin reset sc->maxNext: the next step's findMaxU may be formed by
  // this step's own kernels (constant density, PressureSingle)
  c.maxNextState = c.varRho || c.cfg.iterative ? 0 : 1;
  return check_launch(ctx);
}

// advDiff (advDiff.cpp:14-116) with PressureSingle's RHS divergence
// (PressureSingle.cpp:112-128) formed in place, as in a graph step; right
// after PutObjectsOnGrid it runs on side2 beside the obstacle chain (it
// reads no obstacle data) and joins the main stream before returning.
int cup2d_adv_diff(cup2d_ctx* ctx, double dt) {
  STAGE_PROLOGUE
  if (c.varRho) {                           // advDiffGrav reads invRho: after the placement
    c.placedPending = false;
    c.rhsFresh = false;
    launch_advdiff_grav(c);
    return check_launch(ctx);
  }
  const bool beside = c.placedPending && !prologueLaunched;
  c.placedPending = false;
  if (beside) {
    CK(cudaStreamWaitEvent(c.side2, c.evPlaced, 0));
    {
      StreamScope scope(c, c.side2);
      launch_outflow_flux(c);
      launch_advdiff_rhs_div(c);
    }
    CK(cudaEventRecord(c.evObjDone, c.side2));
    CK(cudaStreamWaitEvent(c.stream, c.evObjDone, 0));
  } else {
    launch_outflow_flux(c);
    launch_advdiff_rhs_div(c);
  }
  c.rhsFresh = true;
  return check_launch(ctx);
}

extern "C++" int pressure_single_keep(cup2d_ctx* ctx, double dt, double* keepDiv, double* keepObst) {
  STAGE_PROLOGUE
  c.placedPending = false;
  if (c.varRho) {
    c.rhsFresh = false;
    c.maxNextState = 0;
    return pressure_varrho(ctx);
  }
  if (c.cfg.iterative) {
    c.rhsFresh = false;
    c.maxNextState = 0;
    return pressure_iterative(ctx);
  }
  if (!c.rhsFresh) launch_rhs_div(c);       // else formed by advDiff at this dt
  c.rhsFresh = false;
  const size_t nb = sizeof(double) * c.ncells();
  if (keepDiv) CK(cudaMemcpyAsync(keepDiv, c.rhs, nb, cudaMemcpyDeviceToDevice, c.stream));
  launch_rhs_obstacles(c);
  if (keepObst) CK(cudaMemcpyAsync(keepObst, c.rhs, nb, cudaMemcpyDeviceToDevice, c.stream));
  poisson_solve(c);
  const bool maxNext = c.maxNextState == 1;  // reset by this step's placement
  launch_pressure_tail(c, maxNext);
  c.maxNextState = maxNext ? 2 : 0;
  return check_launch(ctx);
}

int cup2d_pressure_single(cup2d_ctx* ctx, double dt) { return pressure_single_keep(ctx, dt, nullptr, nullptr); }

static double* field_ptr(Ctx& c, int which);

int cup2d_poisson_solve(cup2d_ctx* ctx, int src, int dst) {
  if (!ctx) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  if (!c.initialised) return fail(ctx, CUP2D_ESTATE, "not initialised");
  double* ps = field_ptr(c, src);
  double* pd = field_ptr(c, dst);
  if (!ps || !pd) return fail(ctx, CUP2D_EINVAL, "unknown field (or invRho of a constant-density context)");
  if ((src == CUP2D_FIELD_UDEF_X || src == CUP2D_FIELD_UDEF_Y || dst == CUP2D_FIELD_UDEF_X ||
       dst == CUP2D_FIELD_UDEF_Y) && c.udefStale)
    CK(fill_udef_grid(c));
  forget_chain(c);
  c.shapesAtEvent = c.shapesMapped = false;
  c.stateSeq++;
  CK(invalidate_dt_next(c));
  double* const R = c.rhs;
  double* const P = c.pres;
  c.rhs = ps;                                   // the solver reads c.rhs and writes c.pres
  c.pres = pd;
  launch_fade_sums(c);
  poisson_solve(c);
  c.rhs = R;
  c.pres = P;
  if (dst == CUP2D_FIELD_UDEF_X || dst == CUP2D_FIELD_UDEF_Y) c.udefStale = false;
  return check_launch(ctx);
}

int cup2d_compute_forces(cup2d_ctx* ctx, double dt) {
  STAGE_PROLOGUE
  const bool maxNext = c.maxNextState == 2;  // after this step's pressure correction
  forget_chain(c);
  c.mapSeqForces = ++c.mapSeq;
  launch_forces(c, c.mapDev->shapes, maxNext, c.mapDev->seqShape, c.mapSeqForces);   // the final states also to mapped host memory
  c.maxNextState = maxNext ? 3 : 0;
  CK(cudaEventRecord(c.evForces, c.stream));
  c.shapesMapped = true;
  return check_launch(ctx);
}

// Simulation.cpp:289-290 (t += dt, step += 1), ending like a graph step:
// the next step's calcMaxTimestep is formed on the final velocity and its
// dt copied to pinned host memory, so that cup2d_calc_dt returns it
// without a round trip while nothing changes the state in between.
int cup2d_end_step(cup2d_ctx* ctx) {
  if (!ctx) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  if (!c.initialised) return fail(ctx, CUP2D_ESTATE, "not initialised");
  // the step's own kernels formed the next findMaxU (placement, pressure
  // correction, forces, nothing else in between): the maximum is exact in
  // any order, so the dt is the one a full-grid findMaxU would give
  const bool fused = c.maxNextState == 3;
  forget_chain(c);
  c.stateSeq++;
  // nothing from here on writes the shape states
  CK(cudaEventRecord(c.evShapes, c.stream));
  c.shapesAtEvent = true;
  c.mapSeqDt = ++c.mapSeq;
  // the next dt also to mapped host memory
  if (fused) launch_end_step_dt(c, &c.mapDev->dtNext, &c.mapDev->seqDt, c.mapSeqDt);
  else launch_end_step_max(c, &c.mapDev->dtNext, &c.mapDev->seqDt, c.mapSeqDt);
  CK(cudaEventRecord(c.evDtNext, c.stream));
  c.dtValidMaybe = c.dtCarried = true;
  return check_launch(ctx);
}

} // extern "C"

namespace cup2d {
// Before graph steps: the state they require, and what the first of them
// relies on, enqueued on the context's stream.
int graph_steps_begin(cup2d_ctx* ctx) {
  Ctx& c = ctx->c;
  if (!c.initialised) return fail(ctx, CUP2D_ESTATE, "not initialised");
  if (c.cfg.iterative)
    return fail(ctx, CUP2D_ENOTSUP, "the iterated penalization decides convergence on the host: "
                                    "run it operator by operator");
  forget_chain(c);
  c.shapesAtEvent = c.shapesMapped = false;
  c.stateSeq++;
  c.udefStale = c.nshapes > 0;              // graph steps leave the grid's uDef
  if (c.cur != 0) {
    // a stage was called on its own: finish in eager mode until parity returns
    return fail(ctx, CUP2D_ESTATE, "velocity buffers out of step order");
  }
  if (c.sideMidPending) {                   // a midline formed ahead by the operator path
    CK(cudaStreamWaitEvent(c.stream, c.evSideMid, 0));
    c.sideMidPending = false;
  }
  if (!c.midByGraph) {
    // graph steps form each next step's midline; the first one needs the
    // current step's (formed here unless already present)
    for (int k = 0; k < c.nshapes; k++)
      if (midline_ahead(c, k)) launch_fish_midline(c, k, c.stream, 4);
    c.midByGraph = true;
  }
  return check_launch(ctx);
}

// After graph steps: each set dt on the device and formed the next one.
void graph_steps_end(Ctx& c) {
  c.devDt = NAN;
  c.dtValidMaybe = true;
  c.dtCarried = false;
}
} // namespace cup2d

extern "C" {

int cup2d_advance(cup2d_ctx* ctx, int nsteps) {
  if (!ctx) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  if (!c.initialised) return fail(ctx, CUP2D_ESTATE, "not initialised");
  if (nsteps <= 0) return CUP2D_OK;
  int rc = graph_steps_begin(ctx);
  if (rc) return rc;
  if (!c.graph) {
    const long long before = c.launches;
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
    enqueue_step(c);
    const cudaError_t e = cudaStreamEndCapture(c.stream, &graph);
    if (e != cudaSuccess) return fail(ctx, CUP2D_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    c.launchesInGraph = (int)(c.launches - before);
    c.launches = before;
    const cudaError_t e2 = cudaGraphInstantiate(&c.graph, graph, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) { c.graph = nullptr; return fail(ctx, CUP2D_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e2)); }
  }
  for (int s = 0; s < nsteps; s++) {
    CK(cudaGraphLaunch(c.graph, c.stream));
    c.launches += c.launchesInGraph;
  }
  graph_steps_end(c);
  return CUP2D_OK;
}

int cup2d_sync(cup2d_ctx* ctx) {
  if (!ctx) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  CK(cudaStreamSynchronize(c.stream));
  int rc = check_launch(ctx);
  if (rc) return rc;
  CK(cudaMemcpyAsync(&c.pin->status, &c.dsc->status, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  const int status = c.pin->status;
  // each raised flag is reported once: a context whose state the caller
  // repairs (cup2d_set_field, cup2d_set_shape, checkpoint load) runs on
  if (status) CK(cudaMemsetAsync(&c.dsc->status, 0, sizeof(int), c.stream));
  if (status & ST_NAN) return fail(ctx, CUP2D_ENAN, "non-finite velocity detected");
  if (status & ST_DOMAIN) return fail(ctx, CUP2D_EDOMAIN, "body out of domain");
  if (status & ST_CAPACITY) return fail(ctx, CUP2D_ECAPACITY, "obstacle tiles exceed capacity");
  if (status & ST_TIMEOUT) return fail(ctx, CUP2D_ETIMEOUT, "a kernel's bounded wait for its tile loads gave up");
  return CUP2D_OK;
}

static double* field_ptr(Ctx& c, int which) {
  switch (which) {
    case CUP2D_FIELD_U: return c.u();
    case CUP2D_FIELD_V: return c.v();
    case CUP2D_FIELD_CHI: return c.chi;
    case CUP2D_FIELD_PRES: return c.pres;
    case CUP2D_FIELD_TMP: return c.rhs;
    case CUP2D_FIELD_UDEF_X: return c.udefx;
    case CUP2D_FIELD_UDEF_Y: return c.udefy;
    case CUP2D_FIELD_SDF: return c.sdf;
    case CUP2D_FIELD_INVRHO: return c.invRho;
    default: return nullptr;
  }
}

int cup2d_get_field(cup2d_ctx* ctx, int which, double* host_out) {
  if (!ctx || !host_out) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  double* p = field_ptr(c, which);
  if (!p && which == CUP2D_FIELD_INVRHO) {  // constant density: 1 everywhere
    std::fill(host_out, host_out + c.ncells(), 1.0);
    return CUP2D_OK;
  }
  if (!p) return fail(ctx, CUP2D_EINVAL, "unknown field");
  if ((which == CUP2D_FIELD_UDEF_X || which == CUP2D_FIELD_UDEF_Y) && c.udefStale) CK(fill_udef_grid(c));
  CK(cudaStreamSynchronize(c.stream));
  CK(cudaMemcpy(host_out, p, sizeof(double) * c.ncells(), cudaMemcpyDeviceToHost));
  return CUP2D_OK;
}

int cup2d_set_field(cup2d_ctx* ctx, int which, const double* host_in) {
  if (!ctx || !host_in) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  double* p = field_ptr(c, which);
  if (!p && which == CUP2D_FIELD_INVRHO)
    return fail(ctx, CUP2D_ESTATE, "invRho is 1 without a body of rhoS != 1 (recomputed by every placement)");
  if (!p) return fail(ctx, CUP2D_EINVAL, "unknown field");
  // the other uDef component keeps the values a read would have given
  if ((which == CUP2D_FIELD_UDEF_X || which == CUP2D_FIELD_UDEF_Y) && c.udefStale) CK(fill_udef_grid(c));
  CK(cudaStreamSynchronize(c.stream));
  CK(h2d_sync(p, host_in, sizeof(double) * c.ncells(), c.stream));
  forget_chain(c);
  c.stateSeq++;
  CK(invalidate_dt_next(c));
  return CUP2D_OK;
}

int cup2d_get_shape(cup2d_ctx* ctx, int id, cup2d_shape_state* out) {
  if (!ctx || !out) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  if (id < 0 || id >= c.nshapes) return fail(ctx, CUP2D_EINVAL, "bad shape id");
  if (c.shapesMapped) {
    // written to mapped host memory by the force pass, the last writer
    CK(wait_mapped(&c.map->seqShape[id], c.mapSeqForces, c.evForces));
    const volatile double* src = reinterpret_cast<const volatile double*>(&c.map->shapes[id]);
    double* dst = reinterpret_cast<double*>(&c.hshapes[id].s);
    for (size_t q = 0; q < sizeof(cup2d_shape_state) / sizeof(double); q++) dst[q] = src[q];
    *out = c.hshapes[id].s;
    return CUP2D_OK;
  }
  if (c.shapesAtEvent) {
    // final since the step end began: read beside its kernels
    CK(cudaStreamWaitEvent(c.side2, c.evShapes, 0));
    CK(cudaMemcpyAsync(&c.pin->shape, c.dshapes + id, sizeof(DevShape), cudaMemcpyDeviceToHost, c.side2));
    CK(cudaStreamSynchronize(c.side2));
  } else {
    CK(cudaMemcpyAsync(&c.pin->shape, c.dshapes + id, sizeof(DevShape), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
  }
  c.hshapes[id] = c.pin->shape;
  *out = c.hshapes[id].s;
  return CUP2D_OK;
}

int cup2d_set_shape(cup2d_ctx* ctx, int id, const cup2d_shape_state* in) {
  if (!ctx || !in) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  if (id < 0 || id >= c.nshapes) return fail(ctx, CUP2D_EINVAL, "bad shape id");
  CK(cudaStreamSynchronize(c.stream));
  CK(cudaMemcpy(&c.hshapes[id], c.dshapes + id, sizeof(DevShape), cudaMemcpyDeviceToHost));
  c.hshapes[id].s = *in;
  CK(h2d_sync(c.dshapes + id, &c.hshapes[id], sizeof(DevShape), c.stream));
  forget_chain(c);
  c.shapesAtEvent = c.shapesMapped = false;
  c.stateSeq++;
  CK(invalidate_dt_next(c));
  return CUP2D_OK;
}

int cup2d_get_scalars(cup2d_ctx* ctx, double* time, double* dt, int* step, double* uinfx, double* uinfy) {
  if (!ctx) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  CK(cudaMemcpyAsync(&c.pin->sc, c.dsc, sizeof(Scalars), cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  const Scalars& s = c.pin->sc;
  if (time) *time = s.time;
  if (dt) *dt = s.dt;
  if (step) *step = s.step;
  if (uinfx) *uinfx = s.uinfx;
  if (uinfy) *uinfy = s.uinfy;
  return CUP2D_OK;
}

int cup2d_set_scalars(cup2d_ctx* ctx, double time, double dt, int step, double uinfx, double uinfy) {
  if (!ctx) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  Scalars s;
  CK(cudaStreamSynchronize(c.stream));
  CK(cudaMemcpy(&s, c.dsc, sizeof(Scalars), cudaMemcpyDeviceToHost));
  s.time = time; s.dt = dt; s.step = step; s.uinfx = uinfx; s.uinfy = uinfy;
  s.dtNextValid = 0;
  CK(h2d_sync(c.dsc, &s, sizeof(Scalars), c.stream));
  c.midByGraph = false;
  c.devDt = dt;
  c.dtValidMaybe = c.dtCarried = false;
  c.shapesAtEvent = c.shapesMapped = false;
  c.stateSeq++;
  forget_chain(c);
  return CUP2D_OK;
}

int cup2d_grid_size(const cup2d_ctx* ctx, int* nx, int* ny, double* h) {
  if (!ctx) return CUP2D_EINVAL;
  if (nx) *nx = ctx->c.g.nx;
  if (ny) *ny = ctx->c.g.ny;
  if (h) *h = ctx->c.g.h;
  return CUP2D_OK;
}

int cup2d_kernel_launches(const cup2d_ctx* ctx, long long* count) {
  if (!ctx || !count) return CUP2D_EINVAL;
  *count = ctx->c.launches;
  return CUP2D_OK;
}

namespace {
// Reads n doubles (four per thread and pass), so that the L2 ends up holding
// clean lines of this buffer only: a launch timed after it reads its inputs
// from HBM and evicts nothing that must be written back.  The sum is stored
// only if it is not finite (the buffer holds zeros), which keeps the loads.
__global__ void __launch_bounds__(512) k_l2_evict(const double4* __restrict__ p, size_t n4, double* sink) {
  double a = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x) {
    const double4 q = p[i];
    a += q.x + q.y + q.z + q.w;
  }
  if (!isfinite(a)) *sink = a;
}
} // namespace

int cup2d_time_kernel(cup2d_ctx* ctx, int which, int reps, int flush_l2, double* ms_per_launch) {
  if (!ctx || !ms_per_launch || reps <= 0) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  if (!c.initialised) return fail(ctx, CUP2D_ESTATE, "not initialised");
  if (which < 0 || which > CUP2D_KERNEL_OUTFLOW) return fail(ctx, CUP2D_EINVAL, "unknown kernel");
  constexpr size_t kFlushBytes = (size_t)256 << 20;
  if (flush_l2 && !c.flushBuf) {
    if (cudaMalloc(&c.flushBuf, kFlushBytes + 64) != cudaSuccess) {
      c.flushBuf = nullptr;
      return fail(ctx, CUP2D_ENOMEM, "L2 flush buffer");
    }
    CK(cudaMemsetAsync(c.flushBuf, 0, kFlushBytes + 64, c.stream));
  }
  CK(invalidate_dt_next(c));
  forget_chain(c);
  c.shapesAtEvent = c.shapesMapped = false;
  c.stateSeq++;
  c.devDt = NAN;
  auto one = [&]() {
    switch (which) {
      case CUP2D_KERNEL_ADVDIFF: launch_advdiff_rhs_div(c); launch_advdiff_undo(c); break;
      case CUP2D_KERNEL_RHS_DIV: launch_rhs_div(c); break;
      case CUP2D_KERNEL_PCORR: launch_pcorr(c); launch_pcorr_undo(c); break;
      case CUP2D_KERNEL_FFT_ROWS_FWD: poisson_rows_fwd(c); break;
      case CUP2D_KERNEL_FFT_COLS: poisson_cols(c); break;
      case CUP2D_KERNEL_FFT_ROWS_INV: poisson_rows_inv(c); break;
      case CUP2D_KERNEL_MAX_U: launch_max_u_dt(c); break;
      case CUP2D_KERNEL_OBJECTS: launch_objects(c, false); break;
      case CUP2D_KERNEL_OUTFLOW: launch_outflow_flux(c); break;
    }
  };
  one();   // warm
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0)); CK(cudaEventCreate(&e1));
  double total = 0;
  for (int r = 0; r < reps; r++) {
    if (flush_l2) {
      k_l2_evict<<<4 * c.sms, 512, 0, c.stream>>>(static_cast<const double4*>(c.flushBuf), kFlushBytes / 32,
                                                   reinterpret_cast<double*>(static_cast<char*>(c.flushBuf) + kFlushBytes));
      CK(cudaGetLastError());
    }
    CK(cudaEventRecord(e0, c.stream));
    one();
    CK(cudaEventRecord(e1, c.stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    total += ms;
  }
  cudaEventDestroy(e0); cudaEventDestroy(e1);
  *ms_per_launch = total / reps;
  return check_launch(ctx);
}

int cup2d_advance_timed(cup2d_ctx* ctx, int nsteps, double* ms) {
  if (!ctx || !ms) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0)); CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, c.stream));
  int rc = cup2d_advance(ctx, nsteps);
  if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
  CK(cudaEventRecord(e1, c.stream));
  CK(cudaEventSynchronize(e1));
  float f = 0;
  CK(cudaEventElapsedTime(&f, e0, e1));
  cudaEventDestroy(e0); cudaEventDestroy(e1);
  *ms = f;
  return CUP2D_OK;
}

} // extern "C"

// ---- batched ensemble ------------------------------------------------------
// One graph per ensemble holds one step of every member: each member's step
// is enqueue_step on the member's own streams, forked from the ensemble's
// stream and joined back to it, so the members are independent branches and
// one launch advances them all (their kernels fill the SMs together).
struct cup2d_ensemble {
  std::vector<cup2d_ctx*> m;
  cudaStream_t stream = nullptr;
  cudaEvent_t evRoot = nullptr, evEnd = nullptr, ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> evIn, evOut;      // per member
  std::vector<int> launchesPerStep;          // per member
  std::vector<unsigned> gens;                // members' graphGen at capture
  cudaGraphExec_t graph = nullptr;
  std::string err;
  // every member's final shape states, written by the captured force passes
  // into mapped host memory; first[i]: member i's first shape there;
  // seq[i]: the member's stateSeq after the ensemble's last advance
  cup2d_shape_state* map = nullptr;
  cup2d_shape_state* mapDev = nullptr;
  int mapLen = 0;
  std::vector<int> first;
  std::vector<unsigned long long> seq;
  bool advanced = false;
};

namespace {

#define CKE(call)                                                               \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      ens->err = std::string(#call) + ": " + cudaGetErrorString(e_);            \
      return CUP2D_ECUDA;                                                       \
    }                                                                           \
  } while (0)

int ens_fail(cup2d_ensemble* ens, int code, const std::string& msg) {
  ens->err = msg;
  return code;
}

// capture one step of every member into ens->graph
int ens_capture(cup2d_ensemble* ens) {
  if (ens->graph) { cudaGraphExecDestroy(ens->graph); ens->graph = nullptr; }
  const int n = (int)ens->m.size();
  int total = 0;
  for (int i = 0; i < n; i++) { ens->first[i] = total; total += ens->m[i]->c.nshapes; }
  if (total > ens->mapLen) {
    CKE(cudaStreamSynchronize(ens->stream));  // earlier launches wrote the old block
    if (ens->map) cudaFreeHost(ens->map);
    ens->map = ens->mapDev = nullptr;
    ens->mapLen = 0;
    CKE(cudaHostAlloc(&ens->map, sizeof(cup2d_shape_state) * total, cudaHostAllocMapped));
    CKE(cudaHostGetDevicePointer(&ens->mapDev, ens->map, 0));
    ens->mapLen = total;
  }
  ens->advanced = false;
  CKE(cudaStreamBeginCapture(ens->stream, cudaStreamCaptureModeThreadLocal));
  cudaEventRecord(ens->evRoot, ens->stream);
  for (int i = 0; i < n; i++) {
    Ctx& c = ens->m[i]->c;
    const long long before = c.launches;
    cudaStreamWaitEvent(c.stream, ens->evRoot, 0);
    c.forcesOut = ens->mapDev + ens->first[i];
    enqueue_step(c);
    c.forcesOut = nullptr;
    cudaEventRecord(ens->evOut[i], c.stream);
    cudaStreamWaitEvent(ens->stream, ens->evOut[i], 0);
    ens->launchesPerStep[i] = (int)(c.launches - before);
    c.launches = before;
    ens->gens[i] = c.graphGen;
  }
  cudaGraph_t graph;
  const cudaError_t e = cudaStreamEndCapture(ens->stream, &graph);
  if (e != cudaSuccess) return ens_fail(ens, CUP2D_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  const cudaError_t e2 = cudaGraphInstantiate(&ens->graph, graph, cudaGraphInstantiateFlagUseNodePriority);
  cudaGraphDestroy(graph);
  if (e2 != cudaSuccess) {
    ens->graph = nullptr;
    return ens_fail(ens, CUP2D_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e2));
  }
  return CUP2D_OK;
}

// the members' earlier work -> nsteps ensemble steps -> the members' later work
int ens_advance(cup2d_ensemble* ens, int nsteps, bool timed) {
  const int n = (int)ens->m.size();
  bool stale = !ens->graph;
  for (int i = 0; i < n; i++) {
    cup2d_ctx* ctx = ens->m[i];
    const int rc = graph_steps_begin(ctx);
    if (rc) return ens_fail(ens, rc, "member " + std::to_string(i) + ": " + ctx->c.err);
    stale |= ens->gens[i] != ctx->c.graphGen;
  }
  if (stale) {
    const int rc = ens_capture(ens);
    if (rc) return rc;
  }
  for (int i = 0; i < n; i++) {
    CKE(cudaEventRecord(ens->evIn[i], ens->m[i]->c.stream));
    CKE(cudaStreamWaitEvent(ens->stream, ens->evIn[i], 0));
  }
  if (timed) CKE(cudaEventRecord(ens->ev0, ens->stream));
  for (int s = 0; s < nsteps; s++) {
    CKE(cudaGraphLaunch(ens->graph, ens->stream));
    for (int i = 0; i < n; i++) ens->m[i]->c.launches += ens->launchesPerStep[i];
  }
  if (timed) CKE(cudaEventRecord(ens->ev1, ens->stream));
  CKE(cudaEventRecord(ens->evEnd, ens->stream));
  for (int i = 0; i < n; i++) {
    Ctx& c = ens->m[i]->c;
    CKE(cudaStreamWaitEvent(c.stream, ens->evEnd, 0));
    graph_steps_end(c);
    ens->seq[i] = c.stateSeq;
  }
  ens->advanced = true;
  return CUP2D_OK;
}

} // namespace

extern "C" {

int cup2d_ensemble_create(cup2d_ctx* const* members, int n, cup2d_ensemble** out) {
  if (!members || n <= 0 || !out) return CUP2D_EINVAL;
  *out = nullptr;
  for (int i = 0; i < n; i++) {
    if (!members[i] || !members[i]->c.initialised) return CUP2D_ESTATE;
    if (members[i]->c.device != members[0]->c.device) return CUP2D_EINVAL;
    for (int j = 0; j < i; j++)
      if (members[j] == members[i]) return CUP2D_EINVAL;
  }
  cup2d_ensemble* ens = new (std::nothrow) cup2d_ensemble();
  if (!ens) return CUP2D_ENOMEM;
  ens->m.assign(members, members + n);
  ens->evIn.assign(n, nullptr);
  ens->evOut.assign(n, nullptr);
  ens->launchesPerStep.assign(n, 0);
  ens->gens.assign(n, 0);
  ens->first.assign(n, 0);
  ens->seq.assign(n, 0);
  if (cudaSetDevice(members[0]->c.device) != cudaSuccess) { delete ens; return CUP2D_ECUDA; }
  int prLeast = 0, prGreatest = 0;
  cudaDeviceGetStreamPriorityRange(&prLeast, &prGreatest);
  bool ok = cudaStreamCreateWithPriority(&ens->stream, cudaStreamNonBlocking, prGreatest) == cudaSuccess &&
            cudaEventCreateWithFlags(&ens->evRoot, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&ens->evEnd, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreate(&ens->ev0) == cudaSuccess && cudaEventCreate(&ens->ev1) == cudaSuccess;
  for (int i = 0; ok && i < n; i++)
    ok = cudaEventCreateWithFlags(&ens->evIn[i], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&ens->evOut[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) { cup2d_ensemble_destroy(ens); return CUP2D_ECUDA; }
  *out = ens;
  return CUP2D_OK;
}

int cup2d_ensemble_advance(cup2d_ensemble* ens, int nsteps) {
  if (!ens) return CUP2D_EINVAL;
  if (nsteps <= 0) return CUP2D_OK;
  return ens_advance(ens, nsteps, false);
}

int cup2d_ensemble_advance_timed(cup2d_ensemble* ens, int nsteps, double* ms) {
  if (!ens || !ms) return CUP2D_EINVAL;
  if (nsteps <= 0) { *ms = 0; return CUP2D_OK; }
  const int rc = ens_advance(ens, nsteps, true);
  if (rc) return rc;
  CKE(cudaEventSynchronize(ens->ev1));
  float f = 0;
  CKE(cudaEventElapsedTime(&f, ens->ev0, ens->ev1));
  *ms = f;
  return CUP2D_OK;
}

int cup2d_ensemble_sync(cup2d_ensemble* ens) {
  if (!ens) return CUP2D_EINVAL;
  CKE(cudaStreamSynchronize(ens->stream));
  for (size_t i = 0; i < ens->m.size(); i++) {
    const int rc = cup2d_sync(ens->m[i]);
    if (rc) return ens_fail(ens, rc, "member " + std::to_string(i) + ": " + ens->m[i]->c.err);
  }
  return CUP2D_OK;
}

int cup2d_ensemble_get_shapes(cup2d_ensemble* ens, cup2d_shape_state* out, int capacity, int* count) {
  if (!ens || !count) return CUP2D_EINVAL;
  const int n = (int)ens->m.size();
  int total = 0;
  for (int i = 0; i < n; i++) total += ens->m[i]->c.nshapes;
  *count = total;
  if (!out && capacity == 0) return CUP2D_OK;         // size query
  if (!out || capacity < total) return ens_fail(ens, CUP2D_EINVAL, "shape buffer too small");
  if (ens->advanced) CKE(cudaEventSynchronize(ens->evEnd));
  int o = 0;
  for (int i = 0; i < n; i++) {
    cup2d_ctx* ctx = ens->m[i];
    Ctx& c = ctx->c;
    const bool mapped = ens->advanced && ens->seq[i] == c.stateSeq && ens->map &&
                        ens->first[i] + c.nshapes <= ens->mapLen;
    for (int k = 0; k < c.nshapes; k++, o++) {
      if (mapped) {
        // written by the member's last force pass inside the ensemble's graph
        const volatile double* src = reinterpret_cast<const volatile double*>(&ens->map[ens->first[i] + k]);
        double* dst = reinterpret_cast<double*>(&out[o]);
        for (size_t q = 0; q < sizeof(cup2d_shape_state) / sizeof(double); q++) dst[q] = src[q];
      } else {
        const int rc = cup2d_get_shape(ctx, k, &out[o]);
        if (rc) return ens_fail(ens, rc, "member " + std::to_string(i) + ": " + c.err);
      }
    }
  }
  return CUP2D_OK;
}

const char* cup2d_ensemble_last_error(const cup2d_ensemble* ens) {
  return ens ? ens->err.c_str() : "null ensemble";
}

int cup2d_ensemble_destroy(cup2d_ensemble* ens) {
  if (!ens) return CUP2D_EINVAL;
  if (ens->stream) cudaStreamSynchronize(ens->stream);
  if (ens->graph) cudaGraphExecDestroy(ens->graph);
  for (cudaEvent_t e : ens->evIn) if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : ens->evOut) if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : {ens->evRoot, ens->evEnd, ens->ev0, ens->ev1}) if (e) cudaEventDestroy(e);
  if (ens->stream) cudaStreamDestroy(ens->stream);
  if (ens->map) cudaFreeHost(ens->map);
  delete ens;
  return CUP2D_OK;
}

} // extern "C"

// ---- checkpoint / restart ----------------------------------------------------
// A checkpoint holds every device buffer that carries state from one step to
// the next (scalars, shapes, the current velocity, the other fields, each
// shape's obstacle tiles, each fish's midline buffers and segments), behind
// a header that identifies the configuration.  Derived or per-step data
// (Poisson tables, fade slots, reduction scratch, tickets) is rebuilt by
// cup2d_init and not stored.  Sections are copied with cudaMemcpyDefault, so
// the buffer may be host or device memory.
namespace {

struct CkptHeader {
  char magic[8];
  uint32_t version, nsections;
  int32_t bpdx, bpdy, poisson, precision, nshapes, flags;   // flags: 1 implicit penalization
  double extent, CFL, lambda, dlm, nu, fadeLen;
  uint64_t checksum;              // ckpt_hash over the sections (0 in the comparison copy)
};
constexpr uint32_t CKPT_VERSION = 6;

// The payload checksum: over each section's 8-byte words (the last one
// zero-padded), the sum modulo 2^64 of SplitMix64 of the word mixed with its
// section and word index.  A sum is independent of the order the words are
// added in, so the device (a grid of atomic adds) and the host (a loop) form
// the same value.
__host__ __device__ inline uint64_t ckpt_mix(uint64_t w, uint64_t sec, uint64_t idx) {
  uint64_t z = w ^ ((sec << 40) + idx) * 0x9E3779B97F4A7C15ull;
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__host__ __device__ inline uint64_t ckpt_word(const unsigned char* p, size_t bytes, size_t w) {
  uint64_t v = 0;
  const size_t o = 8 * w, n = bytes - o < 8 ? bytes - o : 8;
  for (size_t k = 0; k < n; k++) v |= (uint64_t)p[o + k] << (8 * k);
  return v;
}
__global__ void k_ckpt_hash(const unsigned char* p, size_t bytes, uint64_t sec, unsigned long long* out) {
  const size_t nw = (bytes + 7) / 8;
  unsigned long long acc = 0;
  for (size_t w = blockIdx.x * (size_t)blockDim.x + threadIdx.x; w < nw; w += (size_t)gridDim.x * blockDim.x)
    acc += ckpt_mix(ckpt_word(p, bytes, w), sec, w);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, acc);
}
uint64_t ckpt_hash_host(const unsigned char* p, size_t bytes, uint64_t sec) {
  uint64_t acc = 0;
  for (size_t w = 0; w < (bytes + 7) / 8; w++) acc += ckpt_mix(ckpt_word(p, bytes, w), sec, w);
  return acc;
}
constexpr char CKPT_MAGIC[8] = {'C', 'U', 'P', '2', 'D', 'C', 'K', 0};

struct CkptSection { void* p; size_t bytes; };

std::vector<CkptSection> ckpt_sections(Ctx& c) {
  std::vector<CkptSection> s;
  const size_t n = c.ncells() * sizeof(double);
  s.push_back({c.dsc, sizeof(Scalars)});
  s.push_back({c.dshapes, sizeof(DevShape) * c.nshapes});
  s.push_back({c.vel[0][0], n});
  s.push_back({c.vel[0][1], n});
  for (double* f : {c.chi, c.pres, c.rhs, c.sdf, c.udefx, c.udefy}) s.push_back({f, n});
  for (int k = 0; k < c.nshapes; k++) {
    const ObstTiles& t = c.tiles[k];
    const size_t tb = (size_t)t.capacity * BS2 * sizeof(double);
    s.push_back({t.tiles, sizeof(int) * t.capacity});
    s.push_back({t.slot, sizeof(int) * c.g.nblocks});
    for (double* a : {t.chi, t.dist, t.udx, t.udy, t.sD, t.sdx, t.sdy}) s.push_back({a, tb});
    if (c.hshapes[k].cfg.kind != CUP2D_SHAPE_DISK) {
      const FishArrays& F = c.fish[k];
      s.push_back({F.pool, sizeof(double) * fish_pool_len(F.nm)});
      s.push_back({F.seg, sizeof(Segment) * F.nseg});
    }
  }
  return s;
}

CkptHeader ckpt_header(const Ctx& c, size_t nsec) {
  CkptHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, CKPT_MAGIC, sizeof(h.magic));
  h.version = CKPT_VERSION;
  h.nsections = (uint32_t)nsec;
  h.bpdx = c.cfg.bpdx; h.bpdy = c.cfg.bpdy; h.poisson = c.cfg.poisson; h.precision = c.cfg.precision;
  h.nshapes = c.nshapes;
  h.flags = c.cfg.implicit_penalization ? 1 : 0;
  h.extent = c.cfg.extent; h.CFL = c.cfg.CFL; h.lambda = c.cfg.lambda; h.dlm = c.cfg.dlm;
  h.nu = c.cfg.nu; h.fadeLen = c.cfg.fadeLen;
  return h;
}

size_t ckpt_total(const Ctx& c, const std::vector<CkptSection>& s) {
  size_t b = sizeof(CkptHeader) + sizeof(ShapeCfg) * c.nshapes + sizeof(uint64_t) * s.size();
  for (const CkptSection& x : s) b += x.bytes;
  return b;
}

// Checksum of sections (device pointers, or host pointers when onHost).
int ckpt_hash(cup2d_ctx* ctx, const std::vector<CkptSection>& secs, bool onHost, uint64_t* out) {
  Ctx& c = ctx->c;
  if (onHost) {
    uint64_t h = 0;
    for (size_t i = 0; i < secs.size(); i++)
      h += ckpt_hash_host(static_cast<const unsigned char*>(secs[i].p), secs[i].bytes, i);
    *out = h;
    return CUP2D_OK;
  }
  if (!c.hashAcc && cudaMalloc(&c.hashAcc, sizeof(unsigned long long)) != cudaSuccess) {
    c.hashAcc = nullptr;
    return fail(ctx, CUP2D_ENOMEM, "checkpoint checksum accumulator");
  }
  unsigned long long* d = c.hashAcc;
  CK(cudaMemsetAsync(d, 0, sizeof(unsigned long long), c.stream));
  for (size_t i = 0; i < secs.size(); i++) {
    const size_t nw = (secs[i].bytes + 7) / 8;
    if (!nw) continue;
    int grid = (int)std::min<size_t>((nw + 255) / 256, (size_t)4 * c.sms);
    k_ckpt_hash<<<grid, 256, 0, c.stream>>>(static_cast<const unsigned char*>(secs[i].p), secs[i].bytes, i, d);
    CK(cudaGetLastError());
  }
  unsigned long long h = 0;
  CK(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  *out = h;
  return CUP2D_OK;
}

// nothing in flight may write the buffers while they are copied
int ckpt_quiesce(cup2d_ctx* ctx) {
  Ctx& c = ctx->c;
  CK(cudaStreamSynchronize(c.stream));
  CK(cudaStreamSynchronize(c.side));
  CK(cudaStreamSynchronize(c.side2));
  return CUP2D_OK;
}

} // namespace

extern "C" {

int cup2d_checkpoint_size(cup2d_ctx* ctx, size_t* bytes) {
  if (!ctx || !bytes) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  if (!c.initialised) return fail(ctx, CUP2D_ESTATE, "not initialised");
  *bytes = ckpt_total(c, ckpt_sections(c));
  return CUP2D_OK;
}

int cup2d_checkpoint_save(cup2d_ctx* ctx, void* buf, size_t bytes) {
  if (!ctx || !buf) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  if (!c.initialised) return fail(ctx, CUP2D_ESTATE, "not initialised");
  if (c.cur != 0) return fail(ctx, CUP2D_ESTATE, "checkpoints are taken between steps");
  const std::vector<CkptSection> secs = ckpt_sections(c);
  if (bytes < ckpt_total(c, secs)) return fail(ctx, CUP2D_EINVAL, "checkpoint buffer too small");
  int rc = ckpt_quiesce(ctx);
  if (rc) return rc;
  char* out = static_cast<char*>(buf);
  CkptHeader h = ckpt_header(c, secs.size());
  if ((rc = ckpt_hash(ctx, secs, false, &h.checksum))) return rc;
  std::vector<ShapeCfg> cfgs(c.nshapes);
  for (int k = 0; k < c.nshapes; k++) cfgs[k] = c.hshapes[k].cfg;
  std::vector<uint64_t> sizes(secs.size());
  for (size_t i = 0; i < secs.size(); i++) sizes[i] = secs[i].bytes;
  // every copy on the context's stream, then a wait: a device buffer's
  // copies (device to device, asynchronous to the host) are complete before
  // the next step's kernels may change the state
  size_t off = 0;
  CK(cudaMemcpyAsync(out + off, &h, sizeof(h), cudaMemcpyDefault, c.stream));
  off += sizeof(h);
  if (c.nshapes)
    CK(cudaMemcpyAsync(out + off, cfgs.data(), sizeof(ShapeCfg) * c.nshapes, cudaMemcpyDefault, c.stream));
  off += sizeof(ShapeCfg) * c.nshapes;
  CK(cudaMemcpyAsync(out + off, sizes.data(), sizeof(uint64_t) * sizes.size(), cudaMemcpyDefault, c.stream));
  off += sizeof(uint64_t) * sizes.size();
  for (const CkptSection& x : secs) {
    CK(cudaMemcpyAsync(out + off, x.p, x.bytes, cudaMemcpyDefault, c.stream));
    off += x.bytes;
  }
  CK(cudaStreamSynchronize(c.stream));
  return CUP2D_OK;
}

int cup2d_checkpoint_load(cup2d_ctx* ctx, const void* buf, size_t bytes) {
  if (!ctx || !buf) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  if (!c.initialised) return fail(ctx, CUP2D_ESTATE, "not initialised");
  const std::vector<CkptSection> secs = ckpt_sections(c);
  const size_t total = ckpt_total(c, secs);
  if (bytes < sizeof(CkptHeader)) return fail(ctx, CUP2D_EINVAL, "checkpoint truncated");
  const char* in = static_cast<const char*>(buf);
  CkptHeader h;
  CK(cudaMemcpy(&h, in, sizeof(h), cudaMemcpyDefault));
  if (std::memcmp(h.magic, CKPT_MAGIC, sizeof(h.magic)) != 0) return fail(ctx, CUP2D_EINVAL, "not a checkpoint");
  if (h.version != CKPT_VERSION) return fail(ctx, CUP2D_ENOTSUP, "checkpoint version not supported");
  const uint64_t stored = h.checksum;
  h.checksum = 0;
  const CkptHeader mine = ckpt_header(c, secs.size());
  if (std::memcmp(&h, &mine, sizeof(h)) != 0)
    return fail(ctx, CUP2D_EINVAL, "checkpoint of another configuration (grid, solver, precision, parameters or shapes)");
  if (bytes < total) return fail(ctx, CUP2D_EINVAL, "checkpoint truncated");
  size_t off = sizeof(h);
  std::vector<ShapeCfg> cfgs(c.nshapes);
  if (c.nshapes) CK(cudaMemcpy(cfgs.data(), in + off, sizeof(ShapeCfg) * c.nshapes, cudaMemcpyDefault));
  off += sizeof(ShapeCfg) * c.nshapes;
  for (int k = 0; k < c.nshapes; k++)
    if (std::memcmp(&cfgs[k], &c.hshapes[k].cfg, sizeof(ShapeCfg)) != 0)
      return fail(ctx, CUP2D_EINVAL, "checkpoint of other shapes (shape " + std::to_string(k) + ")");
  std::vector<uint64_t> sizes(secs.size());
  CK(cudaMemcpy(sizes.data(), in + off, sizeof(uint64_t) * sizes.size(), cudaMemcpyDefault));
  off += sizeof(uint64_t) * sizes.size();
  for (size_t i = 0; i < secs.size(); i++)
    if (sizes[i] != secs[i].bytes) return fail(ctx, CUP2D_EINVAL, "checkpoint section sizes differ");
  int rc = ckpt_quiesce(ctx);
  if (rc) return rc;
  {
    // the payload's checksum, read where the buffer lies, before anything is written
    cudaPointerAttributes pa{};
    const bool onDevice = cudaPointerGetAttributes(&pa, in) == cudaSuccess &&
                          (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged);
    cudaGetLastError();
    std::vector<CkptSection> src(secs.size());
    size_t o = off;
    for (size_t i = 0; i < secs.size(); i++) { src[i] = {const_cast<char*>(in) + o, secs[i].bytes}; o += secs[i].bytes; }
    uint64_t sum = 0;
    if ((rc = ckpt_hash(ctx, src, !onDevice, &sum))) return rc;
    if (sum != stored) return fail(ctx, CUP2D_EINVAL, "checkpoint payload damaged (checksum differs)");
  }
  for (const CkptSection& x : secs) {        // on the context's stream (see the save)
    CK(cudaMemcpyAsync(x.p, in + off, x.bytes, cudaMemcpyDefault, c.stream));
    off += x.bytes;
  }
  CK(cudaStreamSynchronize(c.stream));
  // host state of a context between steps, knowing nothing of the device
  c.cur = 0;
  if (c.nshapes)
    CK(cudaMemcpy(c.hshapes.data(), c.dshapes, sizeof(DevShape) * c.nshapes, cudaMemcpyDeviceToHost));
  c.devDt = NAN;
  c.dtValidMaybe = true;
  c.dtCarried = false;
  c.shapesAtEvent = c.shapesMapped = false;
  c.stateSeq++;
  forget_chain(c);
  c.sideMidPending = false;
  c.midByGraph = false;
  c.udefStale = c.nshapes > 0;              // refilled from the restored tiles when read
  return CUP2D_OK;
}

} // extern "C"

#ifdef CUP2D_TRACE
// Timeline read-back of the optional trace build: out[2*id] / out[2*id+1]
// are the first entry / last exit (%globaltimer, ns) of kernel id since the
// last reset; reset re-arms the slots.
namespace cup2d {
void trace_bind_fluid(unsigned long long*);
void trace_bind_obstacles(unsigned long long*);
void trace_bind_fish(unsigned long long*);
void trace_bind_poisson(unsigned long long*);
}
extern "C" int cup2d_trace(cup2d_ctx* ctx, unsigned long long* out, int reset) {
  using namespace cup2d;
  static unsigned long long* buf = nullptr;
  if (!ctx) return CUP2D_EINVAL;
  cudaSetDevice(ctx->c.device);
  if (!buf) {
    if (cudaMalloc(&buf, sizeof(unsigned long long) * (2 * TR_N + 8 * TRACE_ITEMS)) != cudaSuccess) return CUP2D_ENOMEM;
    trace_bind_fluid(buf); trace_bind_obstacles(buf); trace_bind_fish(buf); trace_bind_poisson(buf);
    reset = 1;
  }
  cudaDeviceSynchronize();
  if (out) cudaMemcpy(out, buf, sizeof(unsigned long long) * (2 * TR_N + 8 * TRACE_ITEMS), cudaMemcpyDeviceToHost);
  if (reset) {
    std::vector<unsigned long long> init(2 * TR_N + 8 * TRACE_ITEMS, 0);
    for (int i = 0; i < TR_N; i++) { init[2 * i] = ~0ULL; init[2 * i + 1] = 0; }
    h2d_sync(buf, init.data(), sizeof(unsigned long long) * init.size(), ctx->c.stream);
  }
  return CUP2D_OK;
}
#endif

// ---- RL actuation of the curvature swimmers ---------------------------------
// StefanFish::act / getLearnTPeriod / getPhase / state
// (StefanFish.cpp:373-577) on the device state.  An action changes the
// midline from its time on, so midlines formed ahead (the operator path's
// side branch, a graph step's next-step branch) are dropped and re-formed.
namespace {

int fish_of(cup2d_ctx* ctx, int id) {
  Ctx& c = ctx->c;
  if (!c.initialised) return fail(ctx, CUP2D_ESTATE, "not initialised");
  if (id < 0 || id >= c.nshapes) return fail(ctx, CUP2D_EINVAL, "bad shape id");
  const int kind = c.hshapes[id].cfg.kind;
  if (kind != CUP2D_SHAPE_STEFANFISH && kind != CUP2D_SHAPE_ENVELOPEFISH)
    return fail(ctx, CUP2D_EINVAL, "shape is not a curvature swimmer (StefanFish)");
  return CUP2D_OK;
}

int quiesce_all(cup2d_ctx* ctx) {
  Ctx& c = ctx->c;
  CK(cudaStreamSynchronize(c.stream));
  CK(cudaStreamSynchronize(c.side));
  CK(cudaStreamSynchronize(c.side2));
  return CUP2D_OK;
}

// StefanFish::getPhase (StefanFish.cpp:385-395)
double fish_phase(const DevShape& S, double t) {
  const double T0 = S.ctl.time0, Ts = S.ctl.timeshift, Tp = S.ctl.periodPIDval;
  const double arg = 2 * M_PI * ((t - T0) / Tp + Ts) + M_PI * S.cfg.phaseShift;
  const double phase = std::fmod(arg, 2 * M_PI);
  return (phase < 0) ? 2 * M_PI + phase : phase;
}

} // namespace

extern "C" {

int cup2d_fish_act(cup2d_ctx* ctx, int id, double t_action, const double* a, int na) {
  if (!ctx || !a || na < 1) return ctx ? fail(ctx, CUP2D_EINVAL, "no action") : CUP2D_EINVAL;
  int rc = fish_of(ctx, id);
  if (rc) return rc;
  Ctx& c = ctx->c;
  if ((rc = quiesce_all(ctx))) return rc;
  CK(cudaMemcpy(&c.hshapes[id], c.dshapes + id, sizeof(DevShape), cudaMemcpyDeviceToHost));
  DevShape& S = c.hshapes[id];
  FishCtl& C = S.ctl;
  // CurvatureFish::execute (StefanFish.cpp:108-131)
  C.oldrCurv = C.lastCurv;
  C.lastCurv = a[0];
  // ParameterSchedulerLearnWave::Turn (FishUtilities.h:377-384): a node at
  // the head of the wave, the oldest two dropped
  C.bendT0 = t_action;
  for (int i = 6; i > 1; --i) C.bend[i] = C.bend[i - 2];
  C.bend[1] = a[0];
  C.bend[0] = 0;
  if (na > 1) {                             // the tail period
    C.lastTact = a[1];
    const double lastArg = (t_action - C.time0) / C.periodPIDval + C.timeshift;
    C.timeshift = lastArg;
    C.time0 = t_action;
    C.periodPIDval = S.cfg.Tperiod * (1 + a[1]);
    C.periodPIDdif = 0;
  }
  CK(h2d_sync(&c.dshapes[id].ctl, &C, sizeof(FishCtl), c.stream));
  // midlines formed ahead are of the old actuation: mark both buffers empty
  // (their time NaN) so that the next placement forms its midline again
  const FishArrays& F = c.fish[id];
  CK(cudaMemsetAsync(F.integ + 7, 0xff, sizeof(double), c.stream));
  CK(cudaMemsetAsync(F.integ + 15, 0xff, sizeof(double), c.stream));
  CK(cudaStreamSynchronize(c.stream));
  c.sideMidPending = false;
  c.midByGraph = false;
  forget_chain(c);
  c.shapesAtEvent = c.shapesMapped = false;
  c.stateSeq++;
  return CUP2D_OK;
}

int cup2d_fish_gait_get(cup2d_ctx* ctx, int id, double* theta) {
  if (!ctx || !theta) return CUP2D_EINVAL;
  int rc = fish_of(ctx, id);
  if (rc) return rc;
  const ShapeCfg& f = ctx->c.hshapes[id].cfg;
  if (f.kind == CUP2D_SHAPE_ENVELOPEFISH) {
    for (int j = 0; j < 8; j++) theta[j] = f.envFourier[j];
    return CUP2D_OK;
  }
  theta[0] = f.ampFac;
  theta[1] = f.phaseShift;
  for (int j = 0; j < 6; j++) theta[2 + j] = f.curvScale[j];
  return CUP2D_OK;
}

int cup2d_fish_gait_set(cup2d_ctx* ctx, int id, const double* theta) {
  if (!ctx || !theta) return CUP2D_EINVAL;
  int rc = fish_of(ctx, id);
  if (rc) return rc;
  Ctx& c = ctx->c;
  if ((rc = quiesce_all(ctx))) return rc;
  CK(cudaMemcpy(&c.hshapes[id], c.dshapes + id, sizeof(DevShape), cudaMemcpyDeviceToHost));
  ShapeCfg& f = c.hshapes[id].cfg;
  if (f.kind == CUP2D_SHAPE_ENVELOPEFISH) {
    for (int j = 0; j < 8; j++) f.envFourier[j] = theta[j];
  } else {
    f.ampFac = theta[0];
    f.phaseShift = theta[1];
    for (int j = 0; j < 6; j++) f.curvScale[j] = theta[2 + j];
  }
  CK(h2d_sync(&c.dshapes[id].cfg, &f, sizeof(ShapeCfg), c.stream));
  const FishArrays& F = c.fish[id];
  std::vector<double> rS(F.nm);
  CK(cudaMemcpy(rS.data(), F.rS, sizeof(double) * F.nm, cudaMemcpyDeviceToHost));
  const std::vector<double> p1f = curvature_profile(f, rS);
  CK(h2d_sync(F.p1f, p1f.data(), sizeof(double) * F.nm, c.stream));
  // midlines formed ahead are of the old gait (as after cup2d_fish_act)
  CK(cudaMemsetAsync(F.integ + 7, 0xff, sizeof(double), c.stream));
  CK(cudaMemsetAsync(F.integ + 15, 0xff, sizeof(double), c.stream));
  CK(cudaStreamSynchronize(c.stream));
  c.sideMidPending = false;
  c.midByGraph = false;
  forget_chain(c);
  c.shapesAtEvent = c.shapesMapped = false;
  c.stateSeq++;
  return CUP2D_OK;
}

int cup2d_fish_period(cup2d_ctx* ctx, int id, double* period) {
  if (!ctx || !period) return CUP2D_EINVAL;
  int rc = fish_of(ctx, id);
  if (rc) return rc;
  Ctx& c = ctx->c;
  CK(cudaStreamSynchronize(c.stream));
  FishCtl C;
  CK(cudaMemcpy(&C, &c.dshapes[id].ctl, sizeof(FishCtl), cudaMemcpyDeviceToHost));
  *period = C.periodPIDval;                 // StefanFish::getLearnTPeriod
  return CUP2D_OK;
}

// StefanFish::state (StefanFish.cpp:397-577) with the head's shear sensors
// that StefanFish.h:12 compiles in (16 values).
int cup2d_fish_state(cup2d_ctx* ctx, int id, int other, double* out, int n) {
  if (!ctx || !out) return CUP2D_EINVAL;
  int rc = fish_of(ctx, id);
  if (rc) return rc;
  Ctx& c = ctx->c;
  if (other < 0 || other >= c.nshapes) return fail(ctx, CUP2D_EINVAL, "bad shape id");
  if (n < 16) return fail(ctx, CUP2D_EINVAL, "the state has 16 values");
  if ((rc = quiesce_all(ctx))) return rc;
  DevShape S, P;
  CK(cudaMemcpy(&S, c.dshapes + id, sizeof(DevShape), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&P, c.dshapes + other, sizeof(DevShape), cudaMemcpyDeviceToHost));
  Scalars sc;
  CK(cudaMemcpy(&sc, c.dsc, sizeof(Scalars), cudaMemcpyDeviceToHost));
  const double L = S.cfg.length, Tp = S.cfg.Tperiod;
  out[0] = (S.s.center[0] - P.s.center[0]) / L;
  out[1] = (S.s.center[1] - P.s.center[1]) / L;
  out[2] = S.s.orientation;
  out[3] = fish_phase(S, sc.time);
  out[4] = S.s.u * Tp / L;
  out[5] = S.s.v * Tp / L;
  out[6] = S.s.omega * Tp;
  out[7] = S.ctl.lastTact;
  out[8] = S.ctl.lastCurv;
  out[9] = S.ctl.oldrCurv;

  // the skin of the last placement in the computational frame:
  // surfaceToCOMFrame (FishLibrary.cpp:259-280), surfaceToComputationalFrame
  // (:282-299), then computeSkinNormals (:196-257) with the midline
  const FishArrays& F = c.fish[id];
  const int Nm = F.nm;
  const FishMidline& M = F.mid[S.f.midBuf & 1];
  std::vector<double> xu(Nm), yu(Nm), xl(Nm), yl(Nm), rX(Nm), rY(Nm), rS(Nm);
  CK(cudaMemcpy(xu.data(), M.uX, sizeof(double) * Nm, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(yu.data(), M.uY, sizeof(double) * Nm, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(xl.data(), M.lX, sizeof(double) * Nm, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(yl.data(), M.lY, sizeof(double) * Nm, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(rX.data(), F.frame.rX, sizeof(double) * Nm, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(rY.data(), F.frame.rY, sizeof(double) * Nm, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(rS.data(), F.rS, sizeof(double) * Nm, cudaMemcpyDeviceToHost));
  auto rotate = [](double c0, double s0, double& x, double& y) {
    const double p0 = x, p1 = y;
    x = c0 * p0 + (-s0) * p1;
    y = s0 * p0 + c0 * p1;
  };
  {
    const double ct = std::cos(S.f.theta_internal), st = std::sin(S.f.theta_internal);
    const double co = std::cos(S.s.orientation), so = std::sin(S.s.orientation);
    for (int i = 0; i < Nm; i++) {
      for (int side = 0; side < 2; side++) {
        double& x = side ? xl[i] : xu[i];
        double& y = side ? yl[i] : yu[i];
        x -= S.f.CoM_internal[0];
        y -= S.f.CoM_internal[1];
        rotate(ct, st, x, y);
        rotate(co, so, x, y);
        x += S.s.com[0];
        y += S.s.com[1];
      }
      rotate(co, so, rX[i], rY[i]);
      rX[i] += S.s.com[0];
      rY[i] += S.s.com[1];
    }
  }
  const int Np = Nm;
  std::vector<double> midX[2], midY[2], nXs[2], nYs[2];
  for (int side = 0; side < 2; side++) {
    const std::vector<double>& xs = side ? xl : xu;
    const std::vector<double>& ys = side ? yl : yu;
    midX[side].resize(Np - 1); midY[side].resize(Np - 1); nXs[side].resize(Np - 1); nYs[side].resize(Np - 1);
    for (int i = 0; i < Np - 1; i++) {
      midX[side][i] = (xs[i] + xs[i + 1]) / 2;
      midY[side][i] = (ys[i] + ys[i + 1]) / 2;
      nXs[side][i] = (ys[i + 1] - ys[i]);
      nYs[side][i] = -(xs[i + 1] - xs[i]);
      const double nrm = std::sqrt(std::pow(nXs[side][i], 2) + std::pow(nYs[side][i], 2));
      nXs[side][i] /= nrm;
      nYs[side][i] /= nrm;
      const int ii = (i < 8) ? 8 : ((i > Np - 9) ? Np - 9 : i);
      const double dir = nXs[side][i] * (midX[side][i] - rX[ii]) + nYs[side][i] * (midY[side][i] - rY[ii]);
      if (dir < 0) { nXs[side][i] *= -1.0; nYs[side][i] *= -1.0; }
    }
  }

  // the obstacle blocks of this fish and the grid's velocity around them
  const GridDesc& g = c.g;
  const double h = g.h, invh = 1 / h;
  std::vector<int> slot(g.nblocks);
  CK(cudaMemcpy(slot.data(), c.tiles[id].slot, sizeof(int) * g.nblocks, cudaMemcpyDeviceToHost));
  auto bmin = [&](int b, int d) {
    const int bi = d == 0 ? b % g.bpdx : b / g.bpdx;
    return (double)(bi * BS) * h + h * (0 + 0.5) - 0.5 * h;
  };
  auto bmax = [&](int b, int d) {
    const int bi = d == 0 ? b % g.bpdx : b / g.bpdx;
    return (double)(bi * BS) * h + h * (BS - 1 + 0.5) + 0.5 * h;
  };
  bool lost = false;
  // the block holding (x, y) that has an obstacle block, else of those the
  // one with the largest outside distance (the order of
  // std::sort + std::reverse over (distance, index) pairs)
  auto holding = [&](double x, double y) {
    std::vector<std::pair<double, int>> d(g.nblocks);
    for (int b = 0; b < g.nblocks; b++) {
      const double mn0 = bmin(b, 0), mn1 = bmin(b, 1), mx0 = bmax(b, 0), mx1 = bmax(b, 1);
      if (x >= mn0 && y >= mn1 && x <= mx0 && y <= mx1 && slot[b] >= 0) return b;
      d[b] = {std::max(std::max(mn0 - x, x - mx0), std::max(mn1 - y, y - mx1)), b};
    }
    std::sort(d.begin(), d.end());
    std::reverse(d.begin(), d.end());
    for (auto& e : d) if (slot[e.second] >= 0) return e.second;
    lost = true;
    return 0;
  };
  auto cell_in = [&](double x, double y, int b, int& ix, int& iy) {
    const double o0 = (double)((b % g.bpdx) * BS) * h + h * 0.5;
    const double o1 = (double)((b / g.bpdx) * BS) * h + h * 0.5;
    ix = std::min(std::max(0, (int)std::round((x - o0) * invh)), BS - 1);
    iy = std::min(std::max(0, (int)std::round((y - o1) * invh)), BS - 1);
  };
  auto skinVel = [&](double x, double y, double* v) -> int {
    const int b = holding(x, y);
    if (slot[b] < 0) { lost = true; return CUP2D_OK; }
    int ix, iy;
    cell_in(x, y, b, ix, iy);
    const size_t o = (size_t)slot[b] * BS2 + iy * BS + ix;
    double ux, uy;
    CK(cudaMemcpy(&ux, c.tiles[id].udx + o, sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&uy, c.tiles[id].udy + o, sizeof(double), cudaMemcpyDeviceToHost));
    // the removed rigid part (Shape.cpp:197-204), as udef_at evaluates it
    const double p0 = cell_x(g, b % g.bpdx, ix) - S.s.com[0], p1 = cell_y(g, b / g.bpdx, iy) - S.s.com[1];
    ux = ux - (S.Iu - S.Ia * p1);
    uy = uy - (S.Iv + S.Ia * p0);
    v[0] = S.s.u - S.s.omega * (y - S.s.com[1]) + ux;
    v[1] = S.s.v + S.s.omega * (x - S.s.com[0]) + uy;
    return CUP2D_OK;
  };
  auto sensVel = [&](double x, double y, double* v) -> int {
    const int b = holding(x, y);
    int ix, iy;
    cell_in(x, y, b, ix, iy);
    const size_t q = (size_t)((b / g.bpdx) * BS + iy) * g.nx + (b % g.bpdx) * BS + ix;
    CK(cudaMemcpy(&v[0], c.u() + q, sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&v[1], c.v() + q, sizeof(double), cudaMemcpyDeviceToHost));
    return CUP2D_OK;
  };
  int iHead = 0;                            // the head side, s = 0.04 L (_width)
  for (int i = 0; i < Nm - 1; ++i)
    if (rS[i] <= 0.04 * L && rS[i + 1] > 0.04 * L) iHead = i;
  double tip[2], low[2], top[2];
  {
    const double pSkin[2] = {xu[0], yu[0]};
    const double nX = (nXs[0][0] + nXs[1][0]) / 2, nY = (nYs[0][0] + nYs[1][0]) / 2;
    const double pSens[2] = {pSkin[0] + h * nX, pSkin[1] + h * nY};
    double vSens[2], vSkin[2];
    if ((rc = sensVel(pSens[0], pSens[1], vSens)) || (rc = skinVel(pSkin[0], pSkin[1], vSkin))) return rc;
    tip[0] = (vSens[0] - vSkin[0]) * invh;
    tip[1] = (vSens[1] - vSkin[1]) * invh;
  }
  for (int side = 0; side < 2; side++) {
    const std::vector<double>& xs = side ? xl : xu;
    const std::vector<double>& ys = side ? yl : yu;
    const double pSkin[2] = {midX[side][iHead], midY[side][iHead]};
    const double nX = nXs[side][iHead], nY = nYs[side][iHead];
    const double pSens[2] = {pSkin[0] + h * nX, pSkin[1] + h * nY};
    double vSens[2], vSkin[2];
    if ((rc = sensVel(pSens[0], pSens[1], vSens)) || (rc = skinVel(pSkin[0], pSkin[1], vSkin))) return rc;
    const double shX = (vSens[0] - vSkin[0]) * invh, shY = (vSens[1] - vSkin[1]) * invh;
    const double dX = xs[iHead + 1] - xs[iHead], dY = ys[iHead + 1] - ys[iHead];
    const double proj = dX * nX - dY * nY;
    const double tX = proj > 0 ? nX : -nX, tY = proj > 0 ? -nY : nY;
    double* r = side == 0 ? top : low;
    r[0] = shX * nX + shY * nY;
    r[1] = shX * tX + shY * tY;
  }
  if (lost) return fail(ctx, CUP2D_ESTATE, "a skin point lies outside the fish's obstacle blocks");
  out[10] = tip[0] * Tp / L; out[11] = tip[1] * Tp / L;
  out[12] = low[0] * Tp / L; out[13] = low[1] * Tp / L;
  out[14] = top[0] * Tp / L; out[15] = top[1] * Tp / L;
  return CUP2D_OK;
}

} // extern "C"

// ---- field dumps --------------------------------------------------------------
// SimulationData::dumpAll (SimulationData.cpp:207-239): velChi (u, v, chi),
// pres and invRho as single-precision fields, named like DumpHDF5's files
// (prefix + name + the step in seven digits).  HDF5 is not available here,
// so each field is a raw little-endian float32 array (Ny x Nx x channels,
// x fastest) described by an XDMF file that visualisation tools read.
namespace {

bool write_file(const std::string& path, const void* data, size_t bytes) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const bool ok = std::fwrite(data, 1, bytes, f) == bytes;
  return std::fclose(f) == 0 && ok;
}

bool write_xmf(const std::string& path, const std::string& raw, const char* attr, int channels,
               int nx, int ny, double h, double time) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return false;
  const char* type = channels == 1 ? "Scalar" : "Vector";
  std::fprintf(f,
      "<?xml version=\"1.0\" ?>\n<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n<Xdmf Version=\"2.0\">\n"
      " <Domain>\n  <Grid GridType=\"Uniform\">\n   <Time Value=\"%.17g\"/>\n"
      "   <Topology TopologyType=\"2DCoRectMesh\" Dimensions=\"%d %d\"/>\n"
      "   <Geometry GeometryType=\"ORIGIN_DXDY\">\n"
      "    <DataItem Dimensions=\"2\" NumberType=\"Float\" Precision=\"8\" Format=\"XML\">0 0</DataItem>\n"
      "    <DataItem Dimensions=\"2\" NumberType=\"Float\" Precision=\"8\" Format=\"XML\">%.17g %.17g</DataItem>\n"
      "   </Geometry>\n"
      "   <Attribute Name=\"%s\" AttributeType=\"%s\" Center=\"Cell\">\n"
      "    <DataItem Dimensions=\"%d %d %d\" NumberType=\"Float\" Precision=\"4\" Endian=\"Little\" "
      "Format=\"Binary\">%s</DataItem>\n"
      "   </Attribute>\n  </Grid>\n </Domain>\n</Xdmf>\n",
      time, ny + 1, nx + 1, h, h, attr, type, ny, nx, channels, raw.c_str());
  return std::fclose(f) == 0;
}

} // namespace

extern "C" int cup2d_dump(cup2d_ctx* ctx, const char* dir, const char* name) {
  if (!ctx || !dir || !name) return CUP2D_EINVAL;
  Ctx& c = ctx->c;
  if (!c.initialised) return fail(ctx, CUP2D_ESTATE, "not initialised");
  Scalars sc;
  CK(cudaStreamSynchronize(c.stream));
  CK(cudaMemcpy(&sc, c.dsc, sizeof(Scalars), cudaMemcpyDeviceToHost));
  const size_t n = c.ncells();
  std::vector<double> u(n), v(n), chi(n), p(n);
  CK(cudaMemcpy(u.data(), c.u(), sizeof(double) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(v.data(), c.v(), sizeof(double) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(chi.data(), c.chi, sizeof(double) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(p.data(), c.pres, sizeof(double) * n, cudaMemcpyDeviceToHost));
  std::vector<double> ir;
  if (c.invRho) {
    ir.resize(n);
    CK(cudaMemcpy(ir.data(), c.invRho, sizeof(double) * n, cudaMemcpyDeviceToHost));
  }
  char step[16];
  std::snprintf(step, sizeof(step), "%07d", sc.step);
  const std::string base = std::string(dir) + (dir[0] && dir[std::strlen(dir) - 1] != '/' ? "/" : "");
  const std::string tag = std::string(name) + step;
  std::vector<float> buf(3 * n);
  for (size_t i = 0; i < n; i++) {                    // StreamerGlue (Definitions.h:210-227)
    buf[3 * i] = (float)u[i]; buf[3 * i + 1] = (float)v[i]; buf[3 * i + 2] = (float)chi[i];
  }
  struct Out { std::string stem; int ch; };
  const Out outs[3] = {{"velChi_" + tag, 3}, {"pres_" + tag, 1}, {"invRho_" + tag, 1}};
  for (int k = 0; k < 3; k++) {
    if (k == 1) for (size_t i = 0; i < n; i++) buf[i] = (float)p[i];
    if (k == 2) for (size_t i = 0; i < n; i++) buf[i] = ir.empty() ? 1.0f : (float)ir[i];
    const std::string raw = outs[k].stem + ".raw";
    if (!write_file(base + raw, buf.data(), sizeof(float) * n * outs[k].ch) ||
        !write_xmf(base + outs[k].stem + ".xmf", raw, k == 0 ? "velChi" : k == 1 ? "pres" : "invRho",
                   outs[k].ch, c.g.nx, c.g.ny, c.g.h, sc.time))
      return fail(ctx, CUP2D_EINVAL, "cannot write " + base + raw);
  }
  return CUP2D_OK;
}
