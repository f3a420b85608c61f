/*
 * cup2d.h -- C ABI of the B200-native CubismUP_2D timestep pipeline.
 *
 * The reference has no foreign-function interface: its plugin points are the
 * C++ classes Operator (Operator.h:14-27, one virtual operator()(double dt)
 * per pipeline stage), Shape (Shape.h:15-191) and SimulationData
 * (SimulationData.h:17-116), driven by Simulation::advance
 * (Simulation.cpp:279-305).  Each entry point below replaces one of those
 * calls; thin C++ Operator subclasses forwarding to them plug these into
 * the unchanged Simulation loop.
 *
 * Conventions
 *  - every function returns an int status: CUP2D_OK (0) or a CUP2D_E* code;
 *    cup2d_last_error() gives the message.  Nothing aborts or exits.
 *  - a context owns one grid, its shapes and one CUDA stream; calls on one
 *    context come from one host thread.
 *  - all field and shape state is device-resident; stage calls only enqueue
 *    work on the context's stream.  Host copies happen only in the
 *    cup2d_get_* / cup2d_set_* calls (which synchronise).
 *  - fields cross the ABI as row-major Ny x Nx doubles (x fastest), i.e. the
 *    reference's blocks placed at (index[0]*32, index[1]*32).
 */
#ifndef CUP2D_H
#define CUP2D_H

#include <stddef.h>   /* size_t */

#ifdef __cplusplus
extern "C" {
#endif

#define CUP2D_OK 0
#define CUP2D_EINVAL 1       /* bad argument or configuration               */
#define CUP2D_ECUDA 2        /* CUDA runtime error                          */
#define CUP2D_ENAN 3         /* non-finite value detected (Helpers.cpp:178)  */
#define CUP2D_EDOMAIN 4      /* body left the domain (PutObjectsOnGrid.cpp:214) */
#define CUP2D_ECAPACITY 5    /* obstacle tiles exceed the preallocated slots */
#define CUP2D_ENOTSUP 6      /* feature outside this build                  */
#define CUP2D_ESTATE 7       /* call out of order (e.g. before init)        */
#define CUP2D_ENOMEM 8       /* device allocation failed                    */
#define CUP2D_ETIMEOUT 10    /* a kernel's bounded wait for its tile loads  */
                             /* gave up (the step's results are not valid)  */

/* Poisson solver selection, Poisson/PoissonSolver.cpp:23-59 (makeSolver) */
#define CUP2D_POISSON_FREESPACE 0   /* "freespace": FFTW_freespace.cpp        */
#define CUP2D_POISSON_PERIODIC 1    /* "periodic" : FFTW_periodic.h           */
#define CUP2D_POISSON_COSINE 2      /* "" (default): FFTW_dirichlet.h (DCT)   */

/* arithmetic: FP64 everywhere (the reference's Real = double), or FP32 for
 * the free-space and periodic Poisson transforms only -- fields, stencils,
 * obstacle sums and forces stay FP64, the RHS fade and the pressure written
 * back are FP64 (no counterpart in the reference, which is FP64 throughout;
 * not available with the cosine solver: cup2d_create returns ENOTSUP) */
#define CUP2D_PREC_FP64 0
#define CUP2D_PREC_FP32 1

/* field identifiers for cup2d_get_field / cup2d_set_field
 * (SimulationData.h:21-35) */
#define CUP2D_FIELD_U 0
#define CUP2D_FIELD_V 1
#define CUP2D_FIELD_CHI 2
#define CUP2D_FIELD_PRES 3
#define CUP2D_FIELD_TMP 4       /* pressure RHS after PressureSingle        */
#define CUP2D_FIELD_UDEF_X 5    /* deformation velocity on the grid, as the  */
                                /* last PutObjectsOnGrid leaves it (filled    */
                                /* from the obstacle tiles when read)         */
#define CUP2D_FIELD_UDEF_Y 6
#define CUP2D_FIELD_SDF 7       /* max signed distance of all shapes         */
#define CUP2D_FIELD_INVRHO 8    /* 1/rho (SimulationData::invRho; 1 unless a */
                                /* body has rhoS != 1)                        */

/* Simulation parameters: the runtime arguments parsed by
 * Simulation::parseRuntime (Simulation.cpp:66-104). */
typedef struct cup2d_config {
  int bpdx, bpdy;          /* blocks of 32x32 cells per direction (-bpdx/-bpdy) */
  double extent;           /* -extent (default 1)                               */
  double CFL;              /* -CFL (default 0.1)                                */
  double lambda;           /* -lambda (default 1e3/CFL)                         */
  double dlm;              /* -dlm (default 0)                                  */
  double nu;               /* -nu (default 1e-2)                                */
  double fadeLen;          /* -fadeLen (default 0.01), times extent             */
  int nsteps;              /* -nsteps (0: inactive)                             */
  double tend;             /* -tend (0: inactive)                               */
  int poisson;             /* CUP2D_POISSON_*                                   */
  int precision;           /* CUP2D_PREC_*                                      */
  int device;              /* CUDA device ordinal                               */
  int iterative;           /* -iterativePenalization: PressureIterator_unif     */
                           /* replaces PressureSingle (Simulation.cpp:213-216);  */
                           /* operator-by-operator steps only                    */
  double gravity[2];       /* SimulationData::gravity (SimulationData.h:57,     */
                           /* (0, -9.8)); read by the variable-density pipeline  */
  int implicit_penalization; /* PressureSingle as compiled without           */
                           /* EXPL_INTEGRATE_MOM (PressureSingle.cpp:20): the    */
                           /* lambda-implicit momenta F = h^2 rho X/(1+X) with   */
                           /* X = chi lambda dt, and penalization alpha =        */
                           /* 1/(1 + lambda dt chi) (UpdateObjects.cpp:128-210); */
                           /* 0: the shipped explicit forms                      */
  int autotune;            /* 1: cup2d_create times the FFT row passes' variants */
                           /* (8 or 16 values per thread) on this grid and keeps */
                           /* the faster of each (results differ from the        */
                           /* built-in choice only by rounding); a grid tuned    */
                           /* before in the process reuses that choice, so       */
                           /* contexts of one grid agree bitwise.  0: built-in   */
} cup2d_config;

/* Shape descriptors (the key=value parameters of Shape.cpp:331-345,
 * ShapesSimple.h:19-22, Fish.h:27-29, StefanFish.cpp:246-293). */
typedef struct cup2d_shape_params {
  double xpos, ypos;       /* -xpos/-ypos                                      */
  double angle;            /* -angle in degrees                                */
  double rhoS;             /* -rhoS (1)                                        */
  int bFixed, bFixedx, bFixedy;      /* -1 means "default" as in Shape.cpp     */
  int bForced, bForcedx, bForcedy, bBlockAng;
  double xvel, yvel, angvel;         /* forcedu = -xvel etc (Shape.cpp:342)    */
  double timeForced;       /* default: +inf                                    */
  /* disk */
  double radius;           /* -radius (0.1)                                    */
  double tAccel;           /* -tAccel (-1)                                     */
  /* fish */
  double L, T, phi;        /* -L (0.1), -T (1), -phi (0)                       */
  double amplitudeFactor;  /* -amplitudeFactor (1)                             */
  int pid, pidpos;         /* StefanFish -pid / -pidpos controllers (0)         */
} cup2d_shape_params;

#define CUP2D_SHAPE_DISK 0
#define CUP2D_SHAPE_STEFANFISH 1
#define CUP2D_SHAPE_CARLINGFISH 2
/* A curvature swimmer with the carangiform envelope of the benchmark
 * configurations in place of StefanFish's spline (no counterpart in the
 * reference): the curvature amplitude along the body is
 * 0.82 (s/L + 0.0025) / 1.0025 / L, ramped up over the first period and
 * travelling as in CurvatureFish::computeMidline (StefanFish.cpp:154-206). */
#define CUP2D_SHAPE_ENVELOPEFISH 3

/* Rigid-body state and force sums of one shape, in the order of
 * Shape.h:22-62 (42 doubles). */
typedef struct cup2d_shape_state {
  double center[2], com[2], orientation, u, v, omega, M, J, d_gm[2], lab_com[2];
  double penalM, penalJ, penalDX, penalDY, fluidMomX, fluidMomY, fluidAngMom;
  double perimeter, forcex, forcey, forcex_P, forcey_P, forcex_V, forcey_V;
  double torque, torque_P, torque_V, drag, thrust, circulation;
  double Pout, PoutBnd, defPower, defPowerBnd, Pthrust, Pdrag, EffPDef, EffPDefBnd;
} cup2d_shape_state;

typedef struct cup2d_ctx cup2d_ctx;

/* ---- lifetime --------------------------------------------------------- */
/* Fills *cfg with the defaults of Simulation::parseRuntime. */
int cup2d_config_default(cup2d_config* cfg);
/* SimulationData::allocateGrid (SimulationData.cpp:17-47) + solver setup
 * (PressureSingle ctor -> PoissonSolver::makeSolver).  The Poisson
 * transforms are power-of-two FFTs of lengths 16..4096 in shared memory:
 *  - free space pads the grid to powers of two (the reference pads to
 *    2N - 1; any padding >= 2N - 1 gives the same convolution on the
 *    domain), so any block counts with Nx = 32 bpdx <= 4096 and
 *    Ny = 32 bpdy <= 2048;
 *  - periodic: Nx, Ny powers of two, Nx <= 8192, Ny <= 4096;
 *  - cosine: Nx, Ny powers of two, Nx <= 4096, Ny <= 2048.
 * Other grids return CUP2D_ENOTSUP; cup2d_last_error(NULL) gives the
 * reason of this thread's last failed cup2d_create. */
int cup2d_create(const cup2d_config* cfg, cup2d_ctx** out);
int cup2d_destroy(cup2d_ctx* ctx);
const char* cup2d_last_error(const cup2d_ctx* ctx);
/* Simulation::createShapes (Simulation.cpp:106-173), one shape per call.   */
int cup2d_shape_params_default(cup2d_shape_params* p);
int cup2d_add_shape(cup2d_ctx* ctx, int kind, const cup2d_shape_params* p, int* id);
/* Simulation::init's tail + reset (Simulation.cpp:180-241): IC, objects at
 * t=0, ApplyObjVel.  Must follow the last cup2d_add_shape. */
int cup2d_init(cup2d_ctx* ctx);

/* ---- the pipeline (Simulation::advance order) ------------------------- */
/* The transform variants in use (and, when cup2d_config.autotune was set,
 * the times measured for them: forward rows with 8 and 16 values per
 * thread, inverse rows with 8 and 16, in microseconds; zero otherwise). */
typedef struct cup2d_tuning {
  int fft_rows_fwd_e, fft_rows_inv_e;
  int tuned;
  double us[4];
} cup2d_tuning;
int cup2d_tuning_get(cup2d_ctx* ctx, cup2d_tuning* out);

/* Simulation::calcMaxTimestep (Simulation.cpp:254-277) incl. findMaxU
 * (Helpers.cpp:136-176).  dt stays on the device; if dt_out is non-NULL the
 * call synchronises and returns it.  After cup2d_end_step the dt is already
 * formed: the call then waits for it by spinning on a word the step end
 * writes to mapped host memory (one host thread busy for up to 20 ms), and
 * only then on the stream's event. */
int cup2d_calc_dt(cup2d_ctx* ctx, double* dt_out);
/* One Operator::operator()(dt) each.  dt < 0 means "use the device dt from
 * cup2d_calc_dt"; dt >= 0 overrides it, as the reference's argument does.  */
int cup2d_put_objects(cup2d_ctx* ctx, double dt);      /* PutObjectsOnGrid.cpp:186-241 */
int cup2d_adv_diff(cup2d_ctx* ctx, double dt);         /* advDiff.cpp:36-118            */
int cup2d_pressure_single(cup2d_ctx* ctx, double dt);  /* PressureSingle.cpp:346-373    */
int cup2d_compute_forces(cup2d_ctx* ctx, double dt);   /* ComputeForces.cpp:16-111      */
/* PoissonSolver::solve(BSRC, BDST) (PoissonSolver.h:35-40), the second
 * plug-in point: the context's solver (cup2d_config.poisson) on the RHS in
 * field `src` into field `dst` (CUP2D_FIELD_*, device-resident; src == dst
 * allowed, as in solve(tmp, tmp)).  As cub2rhs does (PoissonSolver.cpp:
 * 101-118), the boundary-strip fade with its mean correction is applied to
 * `src` in place.  The stage calls above run it on their own buffers. */
int cup2d_poisson_solve(cup2d_ctx* ctx, int src, int dst);
/* With cup2d_config.iterative, cup2d_pressure_single runs the iterated
 * penalization and projection of PressureIterator_unif::operator()
 * (PressureIterator_unif.cpp:214-270): it waits for each iteration's
 * residual on the host, as the reference decides convergence there, and
 * cup2d_advance / the ensemble return CUP2D_ENOTSUP.  The iteration count
 * and the last relative momentum change of the latest call: */
int cup2d_iteration_stats(cup2d_ctx* ctx, int* iterations, double* rel_df);
/* time += dt; step++ (Simulation.cpp:289-290). */
int cup2d_end_step(cup2d_ctx* ctx);
/* calc_dt + the four operators + end_step, i.e. one pass of
 * Simulation::simulate's loop; replayed from a captured CUDA graph after the
 * first call.  nsteps steps are enqueued without host synchronisation. */
int cup2d_advance(cup2d_ctx* ctx, int nsteps);
/* Blocks until queued work finished; returns the first device status flag
 * raised (CUP2D_ENAN, CUP2D_EDOMAIN, CUP2D_ECAPACITY, CUP2D_ETIMEOUT) or
 * CUP2D_OK.  The
 * reference aborts or exits on these (Helpers.cpp:178-288,
 * PutObjectsOnGrid.cpp:214-218); here the flags are reported once and
 * cleared, and the context stays usable: a caller that repairs the state
 * (cup2d_set_field, cup2d_set_shape, cup2d_checkpoint_load) runs on.
 * Fault injection on the host: the environment variable
 * CUP2D_FAULT_TILE_CAPACITY=n, read by cup2d_add_shape, caps a shape's
 * obstacle-tile capacity at n, so a larger body raises CUP2D_ECAPACITY;
 * CUP2D_FAULT_TMA_WAIT=1, read by cup2d_create, makes advDiff's tile
 * barrier expect 16 bytes more than its loads bring, so every CTA's bounded
 * wait runs out (after one second) and the step reports CUP2D_ETIMEOUT. */
int cup2d_sync(cup2d_ctx* ctx);

/* ---- state exchange --------------------------------------------------- */
int cup2d_get_field(cup2d_ctx* ctx, int which, double* host_out);
int cup2d_set_field(cup2d_ctx* ctx, int which, const double* host_in);
/* After cup2d_compute_forces the force pass writes the final state to
 * mapped host memory and then a sequence word; cup2d_get_shape spins on that
 * word (up to 20 ms) before it waits on the stream's event. */
int cup2d_get_shape(cup2d_ctx* ctx, int id, cup2d_shape_state* out);
int cup2d_set_shape(cup2d_ctx* ctx, int id, const cup2d_shape_state* in);
/* time, dt, step, uinf (SimulationData.h:45-49) */
int cup2d_get_scalars(cup2d_ctx* ctx, double* time, double* dt, int* step,
                      double* uinfx, double* uinfy);
int cup2d_set_scalars(cup2d_ctx* ctx, double time, double dt, int step,
                      double uinfx, double uinfy);
int cup2d_grid_size(const cup2d_ctx* ctx, int* nx, int* ny, double* h);
/* Number of kernels this context launched since creation (every launch,
 * including those replayed inside CUDA graphs). */
int cup2d_kernel_launches(const cup2d_ctx* ctx, long long* count);

/* Measurement hook (no reference counterpart): launches one pipeline kernel
 * `reps` times on the context's stream and returns the mean milliseconds of
 * one launch, each launch bracketed by its own CUDA events.  With flush_l2,
 * a 256 MB device buffer (allocated by the first such call, kept until
 * cup2d_destroy) is read before every launch, outside the events, so that
 * each launch reads its inputs from HBM, not from the 126 MB L2, and evicts
 * only clean lines (a buffer written instead would leave the L2 dirty, and
 * the timed launch would pay for writing it back).  The
 * kernels re-read and re-write the context's own buffers (the column pass,
 * for one, multiplies the spectrum by the Green's function at every launch),
 * so afterwards the fields hold no physical state: re-initialise the context
 * or load a checkpoint before stepping on.  which: CUP2D_KERNEL_*. */
#define CUP2D_KERNEL_ADVDIFF 0      /* advDiff update + RHS divergence (one kernel) */
#define CUP2D_KERNEL_RHS_DIV 1
#define CUP2D_KERNEL_PCORR 2
#define CUP2D_KERNEL_FFT_ROWS_FWD 3
#define CUP2D_KERNEL_FFT_COLS 4
#define CUP2D_KERNEL_FFT_ROWS_INV 5
#define CUP2D_KERNEL_MAX_U 6
#define CUP2D_KERNEL_OBJECTS 7
#define CUP2D_KERNEL_OUTFLOW 8      /* advDiff's boundary outflow flux */
int cup2d_time_kernel(cup2d_ctx* ctx, int which, int reps, int flush_l2, double* ms_per_launch);
/* Measurement hook (no reference counterpart): cup2d_advance(ctx, nsteps)
 * bracketed by CUDA events on the context's stream; returns the elapsed
 * milliseconds (synchronises). */
int cup2d_advance_timed(cup2d_ctx* ctx, int nsteps, double* ms);

/* ---- field dumps ------------------------------------------------------- */
/* SimulationData::dumpAll (SimulationData.cpp:207-239) as the constant-
 * density pipeline calls it (Simulation.cpp:229, 282-297): velChi (u, v,
 * chi), pres and invRho in single precision into directory `dir`, named
 * "velChi_" name step (seven digits) and so on, as DumpHDF5 names its
 * files.  HDF5 is not available to this library: each field is a raw
 * little-endian float32 array (Ny x Nx x channels, x fastest, ".raw") with
 * an XDMF description (".xmf": cell-centred 2DCoRectMesh, spacing h) that
 * visualisation tools read.  Synchronises. */
int cup2d_dump(cup2d_ctx* ctx, const char* dir, const char* name);

/* ---- checkpoint / restart ---------------------------------------------- */
/* The reference parses -restart but restores nothing (Simulation.cpp:68);
 * these calls save and restore the whole state a step carries to the next:
 * scalars (time, dt, step, ...), shape states, velocity and the other
 * fields, the obstacle tiles and the fish midlines.  Continuing from a
 * restored checkpoint is bitwise the same as continuing the saved run.
 *  - the buffer may be host or device memory (copied with
 *    cudaMemcpyDefault); cup2d_checkpoint_size gives its size;
 *  - save: between steps only (CUP2D_ESTATE after a lone advDiff);
 *    synchronises the context;
 *  - the header carries a 64-bit checksum of the payload (formed on the
 *    device at save, checked where the buffer lies at load);
 *  - load: into an initialised context of the same configuration and
 *    shapes (the saved one, or a new one built alike); anything else, a
 *    truncated, damaged (checksum) or foreign buffer returns CUP2D_EINVAL
 *    (another format version CUP2D_ENOTSUP) without changing the context;
 *    synchronises. */
int cup2d_checkpoint_size(cup2d_ctx* ctx, size_t* bytes);
int cup2d_checkpoint_save(cup2d_ctx* ctx, void* buf, size_t bytes);
int cup2d_checkpoint_load(cup2d_ctx* ctx, const void* buf, size_t bytes);

/* ---- discrete adjoint ---------------------------------------------------- */
/* No counterpart in the reference.  Runs nsteps steps of Simulation::advance
 * (PutObjectsOnGrid, advDiff, PressureSingle, ComputeForces) from the
 * current state and returns the time-averaged objective
 *   J = (1/nsteps) sum_{n=1..nsteps} [ w_energy (h^2/2) sum_box (u^2 + v^2)
 *                                      + w_force . (forcex, forcey)
 *                                      + w_torque |torque|
 *                                      + w_body . (u_b, v_b, omega) ]
 * of each step's final velocity, ComputeForces' force on the body and the
 * body's velocity
 * (box = {x0, x1, y0, y1} in domain units: the cells whose index ranges
 * [floor(x0/h), ceil(x1/h)) etc. cover), and, by the transposed steps, its
 * gradient with respect to the initial velocity (grad_u, grad_v: host
 * arrays of Nx*Ny, row-major, or null) and to the body's velocity
 * (grad_body: 3 values, u_b, v_b, omega, or null: a forced body's held
 * velocity, or a free body's initial one), each step's operators linearized about
 * its forward values and applied in reverse order, the forward recomputed
 * from device checkpoints taken every `every` steps.
 *  - grad_gait (CUP2D_GAIT_PARAMS values, or null): for a tethered curvature
 *    swimmer, dJ/dtheta of its gait parameters (cup2d_fish_gait_get): the
 *    flow part by the adjoint (each step's sensitivity to the body's chi,
 *    target velocity and surface normals on the grid), the geometry's
 *    dependence on theta by central differences of the placement alone
 *    (which the flow does not move for a held body), replayed from the
 *    run's first checkpoint;
 *  - dt_in: the step sizes (nsteps values), or null for calcMaxTimestep's;
 *    dt_out (nsteps values, or null) receives the schedule used.  dt is not
 *    differentiated (a frozen schedule);
 *  - ms (2 values, 3 with grad_gait, or null): device time of the forward
 *    (with its checkpoints), of the backward (recomputation and transposed
 *    steps), and host time of the gait's placement replays (run side by
 *    side on contexts of the same configuration, made on the first call and
 *    kept until cup2d_destroy; one after another on ctx if they cannot be
 *    made);
 *  - covered: FP64, any of the three solvers, explicit penalization
 *    without the iterated or variable-density pipelines, one disk fixed on
 *    the grid (bFixed: its chi does not move; the lab velocity is minus the
 *    body's), either forced in x, y and angle for the whole run and past
 *    its tAccel ramp (its velocity is held), or free in all three (its
 *    velocity solved each step from the momentum integrals, Shape.cpp:25-59,
 *    and differentiated through them); or a curvature swimmer held the same
 *    way (forced in all three, no PID: its chi and udef move with its gait
 *    alone, each step's kept by the recomputation); anything else
 *    CUP2D_ENOTSUP;
 *  - the context ends in the forward's final state (as after nsteps
 *    steps), its gait as it was; synchronises.  After an error its state is
 *    unspecified: load a checkpoint taken before the call. */
typedef struct cup2d_adjoint_objective {
  double box[4];          /* the kinetic-energy probe: x0, x1, y0, y1      */
  double w_energy;        /* its weight (0: no energy term, box unused)    */
  double w_force[2];      /* weights of the body's forcex and forcey       */
  double w_body[3];       /* weights of the body's velocity u, v, omega    */
  double w_torque;        /* weight of |torque| (ComputeForces' torque)    */
  double gait_step;       /* the gait gradient's central-difference step   */
                          /* of the placement (0: 1e-7); the forward is     */
                          /* piecewise smooth (raster switches), so a      */
                          /* whole-simulation difference compares at the    */
                          /* same step                                      */
} cup2d_adjoint_objective;
int cup2d_adjoint_run(cup2d_ctx* ctx, int nsteps, int every, const cup2d_adjoint_objective* obj,
                      const double* dt_in, double* dt_out, double* J, double* grad_u, double* grad_v,
                      double* grad_body, double* grad_gait, double* ms);

/* ---- batched ensemble --------------------------------------------------- */
/* No counterpart in the reference (it runs one Simulation per process):
 * n independent simulations on one device, of any grid sizes and shapes,
 * advanced together.  One step of every member is captured into one CUDA
 * graph, each member an independent branch on its own streams, so one
 * launch advances the whole ensemble by a step and the members' kernels
 * share the SMs.  Each member ends bitwise where cup2d_advance(member,
 * nsteps) would leave it.
 *  - members: distinct, initialised contexts on one device (CUP2D_ESTATE /
 *    CUP2D_EINVAL otherwise), each with its velocity in step order, as
 *    cup2d_advance requires;
 *  - the ensemble keeps the member pointers: advance it only while they
 *    exist; destroying it leaves them untouched;
 *  - after an advance the members may be used on their own (their streams
 *    are ordered after the ensemble's work); a member re-initialised since
 *    the last advance is re-captured;
 *  - cup2d_ensemble_advance_timed: the graph launches alone bracketed by
 *    CUDA events (synchronises); cup2d_ensemble_sync: waits and reports the
 *    first member whose status is not CUP2D_OK (cup2d_sync). */
typedef struct cup2d_ensemble cup2d_ensemble;
int cup2d_ensemble_create(cup2d_ctx* const* members, int n, cup2d_ensemble** out);
int cup2d_ensemble_advance(cup2d_ensemble* ens, int nsteps);
int cup2d_ensemble_advance_timed(cup2d_ensemble* ens, int nsteps, double* ms);
int cup2d_ensemble_sync(cup2d_ensemble* ens);
/* Every member's shape states, member by member (*count of them; CUP2D_EINVAL
 * when capacity is smaller; out == NULL with capacity 0 only sets *count),
 * as cup2d_get_shape returns them.  After an
 * ensemble advance the graph's force passes have written them to mapped host
 * memory: one wait for all members; a member used on its own since is read
 * through cup2d_get_shape. */
int cup2d_ensemble_get_shapes(cup2d_ensemble* ens, cup2d_shape_state* out, int capacity, int* count);
const char* cup2d_ensemble_last_error(const cup2d_ensemble* ens);
int cup2d_ensemble_destroy(cup2d_ensemble* ens);

/* ---- RL actuation of the curvature swimmers ---------------------------- */
/* StefanFish::act (StefanFish.cpp:373-377, CurvatureFish::execute :108-131):
 * a[0] turns the body (a node at the head of the learn-wave bending
 * scheduler, FishUtilities.h:377-384, timed t_action); with na > 1, a[1]
 * sets the tail period to Tperiod (1 + a[1]) from t_action on, keeping the
 * undulation's phase.  Between steps; the midline is re-formed from the next
 * placement.  Only for StefanFish / envelope swimmers. */
int cup2d_fish_act(cup2d_ctx* ctx, int id, double t_action, const double* a, int na);
/* The gait parameters of a curvature swimmer (no counterpart in the
 * reference as one set).  StefanFish: theta[0] = amplitudeFactor (the
 * -amplitudeFactor of the shape descriptor), theta[1] = phi (-phi),
 * theta[2..7] = scales of its six curvature control values
 * (StefanFish.cpp:187-193; 1 as built).  The envelope swimmer: the Fourier
 * coefficients f_0..f_7 of its curvature amplitude, the envelope times
 * f_0 + sum_{k=1..7} (f_k - 1) cos(k pi s / L) (1 as built: the envelope).
 * set: between steps; the midline is re-formed from the next placement; a
 * checkpoint loads only into a context of the same gait. */
#define CUP2D_GAIT_PARAMS 8
int cup2d_fish_gait_get(cup2d_ctx* ctx, int id, double* theta);
int cup2d_fish_gait_set(cup2d_ctx* ctx, int id, const double* theta);
/* StefanFish::getLearnTPeriod (StefanFish.cpp:379-383): the current period. */
int cup2d_fish_period(cup2d_ctx* ctx, int id, double* period);
/* StefanFish::state (StefanFish.cpp:397-577) relative to shape `other`, with
 * the head's shear sensors that StefanFish.h:12 compiles in: 16 values
 * (n >= 16): relative centre / L (2), orientation, undulation phase,
 * u T/L, v T/L, omega T, the last period and curvature actions, the one
 * before, then the shear at the tip, lower and upper head side times T/L
 * (normal, tangential each).  Reads the state after the last placement. */
int cup2d_fish_state(cup2d_ctx* ctx, int id, int other, double* out, int n);

/* ---- allocation-free advDiff ------------------------------------------ */
/* This entry point has no counterpart in the reference.  It is advDiff
 * (advDiff.cpp:36-118: explicit Euler step of central advection and 5-point
 * diffusion, inflow-fade ghosts, boundary outflow correction) applied to
 * device buffers the caller owns, for callers that cannot allocate device
 * memory: hosts whose own pool or caching allocator owns the GPU's memory,
 * and latency-critical loops that must not call cudaMalloc/cudaFree (they
 * synchronise the device).  It allocates nothing; its reduction scratch is
 * one fixed device array inside the library (about 128 KB, held on every GPU
 * that loads the library until exit).
 *  - u, v: current velocity, u_out, v_out: result; row-major
 *    (32 bpdy) x (32 bpdx) doubles on the current device; the outputs must
 *    not alias the inputs.  h, nu, dt, uinf as in SimulationData.
 *  - grids of more than CUP2D_NOALLOC_MAX_BLOCKS blocks return
 *    CUP2D_ETOOLARGE without launching anything.
 *  - the first call on a device looks up the scratch address on that device
 *    (cudaGetSymbolAddress); make that first call before any stream capture.
 *    The address is kept for the life of the process: after a
 *    cudaDeviceReset of that device it is stale, so do not call this entry
 *    point on a device that was reset.
 *  - calls share the scratch: calls that overlap on the GPU race and give
 *    wrong results; serialise them (one stream, or events).
 *  - stream: a cudaStream_t (NULL = legacy default stream); the call only
 *    enqueues work. */
#define CUP2D_ETOOLARGE 9
#define CUP2D_NOALLOC_MAX_BLOCKS 16384
int cup2d_adv_diff_noalloc(const double* u, const double* v, double* u_out, double* v_out,
                           int bpdx, int bpdy, double h, double nu, double dt,
                           double uinfx, double uinfy, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CUP2D_H */
