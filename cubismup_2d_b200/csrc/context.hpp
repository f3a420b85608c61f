// Host-side context: the device-resident counterpart of the reference's
// SimulationData (SimulationData.h:17-116) plus its shapes and solver.
#pragma once
#include <string>
#include <vector>
#include "internal.cuh"
#include "launch.hpp"
#include "tma.cuh"

namespace cup2d {

struct Ctx {
  cup2d_config cfg{};
  GridDesc g{};
  int device = 0;
  int sms = 148;                // streaming multiprocessors of the device
  cudaStream_t stream = nullptr;
  bool initialised = false;

  // dense fields (fp64 planes, Ny x Nx)
  double* vel[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [buffer][component]
  int cur = 0;                  // buffer holding the current velocity
  // TMA maps of the velocity planes, boxes of the 32x32 block plus a
  // two-cell halo (advDiff's staged tiles); advTx: the bytes advDiff's tile
  // barrier expects (its two boxes, unless fault injection adds to it)
  CUtensorMap tmVel[2][2];
  unsigned advTx = 0;
  double* chi = nullptr;        // SimulationData::chi
  double* pres = nullptr;       // SimulationData::pres
  double* rhs = nullptr;        // SimulationData::tmp as used by PressureSingle
  double* sdf = nullptr;        // SimulationData::tmp as used by PutObjectsOnGrid
  double* udefx = nullptr;      // SimulationData::uDef
  double* udefy = nullptr;
  // iterated penalization only: SimulationData::tmpV (the velocity before
  // the operator) and vFluid (the fluid velocity of an iteration)
  double* itmp[2] = {nullptr, nullptr};
  double* ifluid[2] = {nullptr, nullptr};
  // variable density (a body with rhoS != 1, with the iterated
  // penalization): SimulationData::invRho and pRHS; rho0 = minRho()
  // (SimulationData.cpp:116-121).  itmp then holds the penalization force
  // (tmpV) and ifluid the pressure-corrected velocity (vFluid).
  bool varRho = false;
  double rho0 = 1.0;
  double* invRho = nullptr;
  double* prhs = nullptr;

  Scalars* dsc = nullptr;       // device scalars
  DevShape* dshapes = nullptr;  // device shape array [MAX_SHAPES]
  std::vector<DevShape> hshapes;
  std::vector<ObstTiles> tiles;
  std::vector<FishArrays> fish;
  int nshapes = 0;
  int maxCapacity = 0;

  // reduction scratch: per-CTA partial sums and "last CTA" tickets
  double* partials = nullptr;
  size_t npartials = 0;
  // blocks that reach the fade strip: fadeSlot[block] = rank among them in
  // block order, or -1 ([nblocks] = their number nfade); their fade sums sit
  // at fade_partials(c)[3 slot ..]
  int* fadeSlot = nullptr;
  int nfade = 0;

  unsigned* counters = nullptr;
  static constexpr int NCOUNTERS = 256;

  Poisson* poisson = nullptr;
  cudaStream_t side = nullptr;  // branch for the next step's fish midlines
  cudaStream_t side2 = nullptr; // branch for the obstacle chain, beside advDiff
  cudaEvent_t evFork = nullptr, evJoin = nullptr, evObj = nullptr, evObjDone = nullptr;
  cudaEvent_t evStart = nullptr;   // the start of a graph step (fork of its first side launches)
  cudaEvent_t evPres = nullptr, evMom = nullptr;
  cudaEvent_t evPlaced = nullptr;   // recorded after the obstacle tiles are placed
  bool recordPlaced = false;
  bool graphStep = false;           // enqueue_step is recording a graph step
  // the operator-by-operator path forms the next step's fish midlines on
  // `side` (evSideMid after them), checked by the next call; midByGraph:
  // the current step's midlines came from a graph step's side branch
  cudaEvent_t evSideMid = nullptr;
  bool sideMidPending = false;
  bool midByGraph = false;

  // Host mirrors of device state, valid in stream order (what the device
  // holds once the work enqueued so far has run), kept by the ABI calls so
  // that the operator-by-operator path launches nothing redundant:
  //   devDt        sc->dt (NaN: not known on the host)
  //   dtValidMaybe sc->dtNextValid may be 1 (a step end formed the next dt)
  //   dtCarried    sc->dtNextValid is 1 and map->dtNext holds sc->dtNext
  //                once evDtNext has completed
  //   rhsFresh     rhs and the fade partials hold the RHS divergence of the
  //                current velocity at sc->dt (formed in place by advDiff)
  //   placedPending evPlaced marks the placed tiles of the last
  //                PutObjectsOnGrid and nothing was enqueued after its chain
  //   shapesAtEvent the shape states are final at evShapes (recorded at a
  //                step end, before kernels that only read them)
  //   udefStale    the grid's deformation velocity (uDef) is not filled for
  //                the tiles of the last PutObjectsOnGrid: PressureSingle
  //                never reads it, so plain and graph steps leave it and
  //                cup2d_get_field fills it from the tiles on demand
  //   maxNextState the next step's findMaxU formed by the operator path's
  //                own kernels, as in a graph step: 1 sc->maxNext reset by
  //                this step's PutObjectsOnGrid, 2 and the pressure
  //                correction's part (the blocks outside the tiles) added, 3
  //                and the force pass's part (the tiles, penalized) added --
  //                the step end then takes dt from it instead of a full-grid
  //                findMaxU; 0 otherwise (any other call in between)
  double devDt = 0.0;
  int maxNextState = 0;
  bool dtValidMaybe = false, dtCarried = false, rhsFresh = false, placedPending = false;
  bool udefStale = false;
  bool shapesAtEvent = false;
  cudaEvent_t evDtNext = nullptr, evShapes = nullptr;
  // pinned host staging of the small read-backs (one copy + one wait each)
  struct HostPin { double dt; int status; IterState it; Scalars sc; DevShape shape; };
  HostPin* pin = nullptr;
  // mapped pinned memory the operator path's kernels write directly (no copy
  // engine): the next dt (step end) and each shape's final state (force
  // pass).  shapesMapped: map->shapes is current once evForces completes.
  // seqDt / seqShape[k]: written by the step end / the force pass after
  // dtNext / shapes[k] (behind a system-scope fence) with the value of
  // mapSeq at that launch; the host spins on them (wait_mapped)
  struct HostMapped {
    double dtNext;
    cup2d_shape_state shapes[MAX_SHAPES];
    unsigned long long seqDt, seqShape[MAX_SHAPES];
  };
  HostMapped* map = nullptr;      // host address
  HostMapped* mapDev = nullptr;   // its device address
  cudaEvent_t evForces = nullptr;
  bool shapesMapped = false;
  // a graph step's force pass also writes the final shape states here when
  // an ensemble captures it (null otherwise)
  cup2d_shape_state* forcesOut = nullptr;
  // bumped by every call that may change the state; an ensemble compares it
  // with the value after its own advance to know a member's read-back is current
  unsigned long long stateSeq = 0;
  // launches that signal the host through HostMapped, counted; the values
  // the last step end and the last force pass were given
  unsigned long long mapSeq = 0, mapSeqDt = 0, mapSeqForces = 0;

  // the Poisson solve of the adjoint: the convolution alone, without
  // cub2rhs's fade (the adjoint applies the fade's transpose itself)
  bool solveNoFade = false;

  // the shape descriptors as given to cup2d_add_shape, and contexts of the
  // same configuration kept for the adjoint's gait replays (created on
  // first use, destroyed with this context)
  std::vector<cup2d_shape_params> shapeParams;
  std::vector<int> shapeKinds;
  std::vector<struct cup2d_ctx*> gaitShadows;

  cudaGraphExec_t graph = nullptr;
  void* flushBuf = nullptr;      // cup2d_time_kernel's L2 flush (256 MB, allocated on demand)
  unsigned long long* hashAcc = nullptr;   // checkpoint checksum accumulator (on demand)
  unsigned graphGen = 0;        // bumped whenever what a step captures changes
  long long launches = 0;
  int launchesInGraph = 0;
  std::string err;

  double* u() const { return vel[cur][0]; }
  double* v() const { return vel[cur][1]; }
  double* uo() const { return vel[1 - cur][0]; }
  double* vo() const { return vel[1 - cur][1]; }
  size_t ncells() const { return (size_t)g.nx * g.ny; }
};

// A swimmer whose midline depends on time only is formed a step ahead (on a
// side branch); one under PID control depends on the body's state at the
// step's start and is formed within the step, after the controller.
inline bool midline_in_step(const Ctx& c, int k) {
  return c.hshapes[k].cfg.pid || c.hshapes[k].cfg.pidpos;
}
inline bool midline_ahead(const Ctx& c, int k) {
  return c.hshapes[k].cfg.kind != CUP2D_SHAPE_DISK && !midline_in_step(c, k);
}

// doubles behind one fish's arrays (FishArrays::pool): the static profile,
// two midline buffers, the frame midline, the integrals, then the skins of
// the two midline buffers
inline size_t fish_pool_len(int nm) { return 36 * (size_t)nm + 16; }

// counter slots used by the kernels (each last-CTA reduction owns one)
enum CounterSlot : int {
  CNT_MAXU = 0, CNT_ADV = 1,
  CNT_CHI = 8,          // + shape
  CNT_RHSOBST = 24,     // + shape
  CNT_FORCES = 40,      // + shape
  CNT_MOMENTS = 56,     // + shape
  CNT_MOMENTA = 72,     // + shape
};
// partials: [0, 3 nblocks) the grid reductions (findMaxU, advDiff's outflow,
// the fade sums: three per strip block), then 4096 spare, then the
// per-shape tile reductions
inline double* fade_partials(const Ctx& c) { return c.partials; }

// every shape's obstacle tiles, by value (a kernel argument)
struct AllTiles { ObstTiles t[MAX_SHAPES]; };
inline AllTiles all_tiles(const Ctx& c) {
  AllTiles a{};
  for (int k = 0; k < c.nshapes; k++) a.t[k] = c.tiles[k];
  return a;
}
// CTAs of each shape's per-tile kernel (a kernel argument)
struct PenalCtas { int n[MAX_SHAPES]; };
// doubles of one shape's tile-reduction region
inline size_t shape_region(const Ctx& c) { return (size_t)c.maxCapacity * 24; }
// CTAs per shape of the per-tile kernels: one wave at most; each CTA loops
// over tiles s = blockIdx.x, blockIdx.x + gridDim.x, ... < ntiles
inline int tile_ctas(const Ctx& c, int capacity) { return capacity < c.sms ? capacity : c.sms; }
inline double* shape_partials(const Ctx& c) { return c.partials + (size_t)3 * c.g.nblocks + 4096; }

#define CUP2D_LAUNCHED(c) ((c).launches++)

} // namespace cup2d

// the opaque handle of the C ABI
struct cup2d_ctx { cup2d::Ctx c; };

// cup2d_pressure_single, keeping copies of the RHS before the obstacle
// terms (keepDiv) and before the fade (keepObst) when these are non-null
// (the adjoint's recomputation; a constant-density context without the
// iterated penalization)
int pressure_single_keep(cup2d_ctx* ctx, double dt, double* keepDiv, double* keepObst);
