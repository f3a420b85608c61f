// Host-side launchers of the pipeline kernels (one per reference function).
#pragma once
#include "internal.cuh"

#include <utility>

namespace cup2d {

struct Ctx;

// Kernel launch with programmatic stream serialization (see pdl_begin).
template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                            cudaStream_t stream, Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid; cfg.blockDim = block; cfg.dynamicSmemBytes = smem; cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr; cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// A host-to-device copy ordered on `stream` and complete on return.  A plain
// cudaMemcpy runs on the legacy default stream, which the context's
// non-blocking streams do not wait for: from pageable memory it may return
// before its DMA lands, and a kernel launched next on the context's stream
// could read the old values.
inline cudaError_t h2d_sync(void* dst, const void* src, size_t bytes, cudaStream_t stream) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream);
  return e == cudaSuccess ? cudaStreamSynchronize(stream) : e;
}

// fluid.cu
void launch_max_u_dt(Ctx& c);                        // Helpers.cpp:136-176 + Simulation.cpp:254-277
void launch_set_dt(Ctx& c, double dt);               // Operator::operator()(dt) argument
void launch_outflow_flux(Ctx& c);                     // advDiff.cpp:89-106, before the update
void launch_advdiff_rhs_div(Ctx& c);                  // the update, then PressureSingle.cpp:112-128 in place
void launch_advdiff_undo(Ctx& c);
void launch_pcorr_undo(Ctx& c);
void launch_rhs_div(Ctx& c);                         // PressureSingle.cpp:112-128
void launch_fade_sums(Ctx& c);                       // PoissonSolver.cpp:61-100 sums of c.rhs as it is
void launch_rhs_iter(Ctx& c);                        // PressureIterator_unif.cpp:22-49
void launch_pcorr_from(Ctx& c, const double* ui, const double* vi, double* uo, double* vo);
int build_fade_slots(Ctx& c);                        // PoissonSolver.cpp:71-79, once per grid
// PressureSingle.cpp:216-241; maxNext: with the next step's findMaxU over
// the blocks outside every shape's tiles (graph steps)
void launch_pcorr(Ctx& c, bool maxNext = false);
// Simulation.cpp:289-290 + the next step's calcMaxTimestep from sc->maxNext
// (also to dtOut: mapped host memory, or null)
// dtOut (mapped host memory): the next dt; then seqOut = seqVal behind a
// system-scope fence, the word the host spins on
void launch_end_step_dt(Ctx& c, double* dtOut = nullptr, unsigned long long* seqOut = nullptr,
                        unsigned long long seqVal = 0);
void launch_take_dt_next(Ctx& c);                    // calcMaxTimestep from the carried dt
// findMaxU + Simulation.cpp:289-290 + the next dt (also to dtOut: mapped host memory, or null)
void launch_end_step_max(Ctx& c, double* dtOut = nullptr, unsigned long long* seqOut = nullptr,
                         unsigned long long seqVal = 0);
void launch_ic(Ctx& c);                              // Helpers.cpp:38-82
void launch_apply_obj_vel(Ctx& c);                   // Helpers.cpp:290-307

// obstacles.cu
void launch_objects(Ctx& c, bool midlineReady);     // PutObjectsOnGrid.cpp:186-241
void launch_objects_begin(Ctx& c, bool midlineReady);  // lab velocity + body motion
void launch_objects_rest(Ctx& c);                    // tiles, SDF, chi, moments
void launch_step_begin(Ctx& c);                      // dt + tile reset + body motion, fused
void launch_obj_vel_on_grid(Ctx& c);                 // PutObjectsOnGrid.cpp:149-184
void launch_rhs_obstacles(Ctx& c);                   // PressureSingle.cpp:130-213
void launch_momenta(Ctx& c, const double* ui, const double* vi);  // PressureSingle.cpp:23-67, 362-372
// PressureIterator_unif.cpp (the iterated penalization)
void launch_momenta_iter(Ctx& c, const double* ui, const double* vi);   // :80-135 + updateVelocity
// the variable-density pipeline (varrho.cu; PressureIterator_approx.cpp)
void launch_momenta_varrho(Ctx& c, const double* ui, const double* vi);  // :171-222 + updateVelocity
void launch_invrho(Ctx& c);                          // PutObjectsOnGrid.cpp:65-73, invRho blend
void launch_advdiff_grav(Ctx& c);                    // advDiffGrav.cpp:14-137
void launch_vr_init(Ctx& c);                         // pressureCorrectionInit :81-122
void launch_vr_penalize(Ctx& c);                     // penalize :224-287 -> sc->it.relDF
void launch_vr_rhs(Ctx& c);                          // updatePressureRHS :289-335
void launch_vr_pcorr(Ctx& c, bool final_);           // pressureCorrection / finalizePressure
void launch_penalize_iter(Ctx& c, const double* tu, const double* tv,
                          const double* fu, const double* fv);          // :137-187, residual -> sc->it.relDF
void launch_set_iter_state(Ctx& c, const IterState& st);                // :247-252 state after a call
struct PenalCtas;
// relDF = sqrt((DMX + DMY) / (eps + MX + MY)) from each shape's per-CTA sums
void launch_reldf(Ctx& c, const PenalCtas& nc);
void launch_collide_penalize(Ctx& c);                // PressureSingle.cpp:69-108, 243-344
// ComputeForces.cpp:16-111; out (mapped host memory, or null): each shape's final state
// maxNext: with the next step's findMaxU over the shapes' tiles
// out (mapped host memory, or null): each shape's final state; then
// seqOut[k] = seqVal behind a system-scope fence
void launch_forces(Ctx& c, cup2d_shape_state* out, bool maxNext, unsigned long long* seqOut = nullptr,
                   unsigned long long seqVal = 0);

// poisson.cu
struct Poisson;
Poisson* poisson_create(Ctx& c);
// whether the chosen solver's transforms exist for an nx x ny grid, and the
// limits in words (for the error message)
bool poisson_size_ok(int type, int nx, int ny);
const char* poisson_size_limits(int type);
void poisson_destroy(Poisson* p);
void poisson_solve(Ctx& c);                          // PoissonSolver::solve of the chosen solver
cudaError_t poisson_autotune(Ctx& c);                // the row passes' variants timed on this grid
void poisson_tuning(const Ctx& c, cup2d_tuning* out);
void poisson_rows_fwd(Ctx& c);
void poisson_cols(Ctx& c);
void poisson_rows_inv(Ctx& c);

} // namespace cup2d
