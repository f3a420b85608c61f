// Oracle test infrastructure (never shipped, never on the product path).
//
// An MPI-free harness around the reference's OWN operator sources, compiled
// unmodified from the reference tree against the project-written shims in
// oracle/shim (Cubism grid/lab/parser, FFTW API, 3x3 GSL LU).  It replaces
// main.cpp / Simulation.cpp, whose include set drags in the HYPRE-only
// variable-density operators; the steps below restate Simulation.cpp for the
// constant-density pipeline (PressureSingle, or PressureIterator_unif under
// -iterativePenalization 1):
//   parseRuntime        Simulation.cpp:66-104
//   createShapes        Simulation.cpp:106-173
//   init (pipeline)     Simulation.cpp:175-230 (bVariableDensity == false
//                       branch, :205-221)
//   reset               Simulation.cpp:232-241
//   calcMaxTimestep     Simulation.cpp:254-277
//   advance             Simulation.cpp:279-305
// and exposes fields/shape state through a C ABI for ctypes-based tests.
#include "Definitions.h"
#include "SimulationData.h"
#include "Shape.h"
#include "Operators/Helpers.h"
#include "Operators/PutObjectsOnGrid.h"
#include "Operators/advDiff.h"
#include "Operators/PressureSingle.h"
#include "Operators/PressureIterator_unif.h"
#include "Operators/advDiffGrav.h"
#include "Operators/PressureIterator_approx.h"
#include "Operators/UpdateObjects.h"
#include "Poisson/PoissonSolver.h"
#include "Operators/ComputeForces.h"
#include "Obstacles/ShapesSimple.h"
#include "Obstacles/StefanFish.h"
#include "Obstacles/CarlingFish.h"
#include "Utils/FactoryFileLineParser.h"

#include <omp.h>
#include <algorithm>
#include <cstring>
#include <sstream>
#include <string>
#include <unistd.h>
#include <vector>

using namespace cubism;

namespace {

std::vector<std::string> split(const std::string& s, const char dlm) {
  std::stringstream ss(s); std::string item; std::vector<std::string> tokens;
  while (std::getline(ss, item, dlm)) tokens.push_back(item);
  return tokens;
}

struct Argv {
  std::vector<std::string> store;
  std::vector<char*> ptrs;
  explicit Argv(const std::string& line) {
    store.push_back("cup2d_ref");
    // tokens separated by spaces; a token in single quotes may hold spaces
    std::string cur; bool q = false;
    for (char c : line) {
      if (c == '\'') { q = !q; continue; }
      if (c == ' ' && !q) { if (!cur.empty()) store.push_back(cur); cur.clear(); }
      else cur += c;
    }
    if (!cur.empty()) store.push_back(cur);
    for (auto& s : store) ptrs.push_back(&s[0]);
    ptrs.push_back(nullptr);
  }
  int argc() const { return (int)store.size(); }
  char** argv() { return ptrs.data(); }
};

// The iterated operators keep their iteration count (oldNsteps, the
// iterations of the last call) private, PressureSingle its steps.  An explicit template instantiation
// may name a private member (access is not checked there), which hands the
// harness a pointer to it without touching the reference's sources.
struct IterCountTag { typedef int PressureIterator_unif::*type; };
IterCountTag::type member_of(IterCountTag);
template <class Tag, typename Tag::type M>
struct MemberPtr { friend typename Tag::type member_of(Tag) { return M; } };
template struct MemberPtr<IterCountTag, &PressureIterator_unif::oldNsteps>;
struct VarRhoCountTag { typedef int PressureVarRho_approx::*type; };
VarRhoCountTag::type member_of(VarRhoCountTag);
template struct MemberPtr<VarRhoCountTag, &PressureVarRho_approx::oldNsteps>;

struct PsRhsTag { typedef void (PressureSingle::*type)(const double) const; };
PsRhsTag::type member_of(PsRhsTag);
template struct MemberPtr<PsRhsTag, &PressureSingle::updatePressureRHS>;
struct PsCorrTag { typedef void (PressureSingle::*type)(const double) const; };
PsCorrTag::type member_of(PsCorrTag);
template struct MemberPtr<PsCorrTag, &PressureSingle::pressureCorrection>;
struct PsSolverTag { typedef PoissonSolver* const PressureSingle::*type; };
PsSolverTag::type member_of(PsSolverTag);
template struct MemberPtr<PsSolverTag, &PressureSingle::pressureSolver>;

// PressureSingle as compiled without EXPL_INTEGRATE_MOM (a #define at
// PressureSingle.cpp:20): its RHS, solve and pressure correction
// (PressureSingle.cpp:346-360), then the lambda-implicit momenta, velocity
// update, collisions and penalization, which UpdateObjects::operator()
// (UpdateObjects.cpp:213-224) runs in the same order with that switch off
// (UpdateObjects.cpp:19); harness option -implicitPenalization 1.
struct PressureSingleImplicit : public Operator {
  PressureSingle ps;
  UpdateObjects uo;
  explicit PressureSingleImplicit(SimulationData& s) : Operator(s), ps(s), uo(s) {}
  void operator()(const double dt) override {
    (ps.*member_of(PsRhsTag()))(dt);
    (ps.*member_of(PsSolverTag()))->solve(sim.tmp->getBlocksInfo(), sim.pres->getBlocksInfo());
    (ps.*member_of(PsCorrTag()))(dt);
    uo(dt);
  }
  std::string getName() override { return "PressureSingle(implicit penalization)"; }
};

struct RefSim
{
  Argv args;
  ArgumentParser parser;
  SimulationData sim;
  std::vector<Operator*> pipeline;
  std::string workdir;
  bool implicitPenalization = false;

  explicit RefSim(const std::string& line)
    : args(line), parser(args.argc(), args.argv()) {}

  ~RefSim() {
    for (auto* g : pipeline) delete g;
  }

  void parseRuntime() {  // Simulation.cpp:66-104
    sim.bRestart = parser("-restart").asBool(false);
    parser.set_strict_mode();
    sim.bpdx = parser("-bpdx").asInt();
    sim.bpdy = parser("-bpdy").asInt();
    parser.unset_strict_mode();
    sim.extent = parser("-extent").asDouble(1);
    sim.allocateGrid();
    sim.nsteps = parser("-nsteps").asInt(0);
    sim.endTime = parser("-tend").asDouble(0);
    sim.dumpFreq = parser("-fdump").asInt(0);
    sim.dumpTime = parser("-tdump").asDouble(0);
    sim.path2file = parser("-file").asString("./");
    sim.path4serialization = parser("-serialization").asString(sim.path2file);
    sim.poissonType = parser("-poissonType").asString("");
    sim.CFL = parser("-CFL").asDouble(.1);
    sim.lambda = parser("-lambda").asDouble(1e3 / sim.CFL);
    sim.dlm = parser("-dlm").asDouble(0);
    sim.nu = parser("-nu").asDouble(1e-2);
    sim.fadeLenX = parser("-fadeLen").asDouble(0.01) * sim.extent;
    sim.fadeLenY = parser("-fadeLen").asDouble(0.01) * sim.extent;
    sim.verbose = parser("-verbose").asInt(1);
    sim.iterativePenalization = parser("-iterativePenalization").asInt(0);
    implicitPenalization = parser("-implicitPenalization").asInt(0) != 0;   // harness option
    sim.muteAll = parser("-muteAll").asInt(0);
    if (sim.muteAll) sim.verbose = 0;
  }

  void createShapes() {  // Simulation.cpp:106-173
    const std::string shapeArg = parser("-shapes").asString("");
    std::stringstream descriptors(shapeArg);
    std::string lines;
    unsigned k = 0;
    while (std::getline(descriptors, lines)) {
      std::replace(lines.begin(), lines.end(), '_', ' ');
      for (const auto& line : split(lines, ',')) {
        std::istringstream line_stream(line);
        std::string objectName;
        line_stream >> objectName;
        if (objectName.empty() or objectName[0] == '#') continue;
        FactoryFileLineParser ffparser(line_stream);
        double center[2] = {ffparser("-xpos").asDouble(.5 * sim.extents[0]),
                            ffparser("-ypos").asDouble(.5 * sim.extents[1])};
        Shape* shape = nullptr;
        if (objectName == "disk") shape = new Disk(sim, ffparser, center);
        else if (objectName == "halfDisk") shape = new HalfDisk(sim, ffparser, center);
        else if (objectName == "ellipse") shape = new Ellipse(sim, ffparser, center);
        else if (objectName == "stefanfish") shape = new StefanFish(sim, ffparser, center);
        else if (objectName == "carlingfish") shape = new CarlingFish(sim, ffparser, center);
        else throw std::runtime_error("shape not supported by the oracle harness: " + objectName);
        shape->obstacleID = k++;
        sim.shapes.push_back(shape);
      }
    }
    if (sim.shapes.empty()) throw std::runtime_error("no shapes");
    sim.checkVariableDensity();
    // Simulation.cpp:194-199: without -iterativePenalization the variable-
    // density branch needs HYPRE (PressureVarRho_proper), absent here
    if (sim.bVariableDensity && !sim.iterativePenalization)
      throw std::runtime_error("variable density without -iterativePenalization needs HYPRE");
  }

  void init() {  // Simulation.cpp:175-230, constant-density branch
    parseRuntime();
    createShapes();
    { IC ic(sim); ic(0); }
    sim.bStaggeredGrid = false;
    pipeline.push_back(new PutObjectsOnGrid(sim));
    if (sim.bVariableDensity) {
      // Simulation.cpp:183-192: the variable-density branch with the
      // iterated penalization
      pipeline.push_back(new advDiffGrav(sim));
      pipeline.push_back(new PressureVarRho_approx(sim));
    } else {
      pipeline.push_back(new advDiff(sim));
      // Simulation.cpp:213-216: -iterativePenalization selects the iterated
      // penalization/projection operator in place of PressureSingle
      if (sim.iterativePenalization) pipeline.push_back(new PressureIterator_unif(sim));
      else if (implicitPenalization) pipeline.push_back(new PressureSingleImplicit(sim));
      else pipeline.push_back(new PressureSingle(sim));
    }
    pipeline.push_back(new ComputeForces(sim));
    reset();
    sim.dt = 0;
  }

  void reset() {  // Simulation.cpp:232-241
    sim.resetAll();
    IC ic(sim); ic(0);
    (*pipeline[0])(0);
    ApplyObjVel initVel(sim); initVel(0);
  }

  double calcMaxTimestep() {  // Simulation.cpp:254-277
    const auto findMaxU_op = findMaxU(sim);
    const Real maxU = findMaxU_op.run();
    const double h = sim.getH();
    const double dtFourier = h * h / sim.nu, dtCFL = maxU < 2.2e-16 ? 1 : h / maxU;
    const double maxUb = sim.maxRelSpeed(), dtBody = maxUb < 2.2e-16 ? 1 : h / maxUb;
    sim.dt = sim.CFL * std::min({dtCFL, dtFourier, dtBody});
    if (sim.step < 100) {
      const double x = (sim.step + 1.0) / 100;
      const double rampCFL = std::exp(std::log(1e-3) * (1 - x) + std::log(sim.CFL) * x);
      sim.dt = rampCFL * std::min({dtCFL, dtFourier, dtBody});
    }
    if (sim.dlm > 0) sim.lambda = sim.dlm / sim.dt;
    return sim.dt;
  }

  bool advance(const double dt) {  // Simulation.cpp:279-305 (dumps are no-ops)
    (void)dt;
    for (size_t c = 0; c < pipeline.size(); c++) (*pipeline[c])(sim.dt);
    sim.time += sim.dt;
    sim.step++;
    return sim.bOver();
  }
};

// field accessors: row-major Ny x Nx planes, x fastest
template <typename F>
void for_cells(RefSim* r, F&& f) {
  auto& infos = r->sim.vel->getBlocksInfo();
  const int Nx = r->sim.bpdx * _BS_;
  for (size_t b = 0; b < infos.size(); b++) {
    const int bx = infos[b].index[0], by = infos[b].index[1];
    for (int iy = 0; iy < _BS_; iy++)
    for (int ix = 0; ix < _BS_; ix++) {
      const long g = (long)(by * _BS_ + iy) * Nx + (bx * _BS_ + ix);
      f(b, ix, iy, g);
    }
  }
}

Real* field_ptr(RefSim* r, int which, size_t b, int ix, int iy) {
  SimulationData& s = r->sim;
  switch (which) {
    case 0: return &(*(VectorBlock*)s.vel->getBlocksInfo()[b].ptrBlock)(ix, iy).u[0];
    case 1: return &(*(VectorBlock*)s.vel->getBlocksInfo()[b].ptrBlock)(ix, iy).u[1];
    case 2: return &(*(ScalarBlock*)s.chi->getBlocksInfo()[b].ptrBlock)(ix, iy).s;
    case 3: return &(*(ScalarBlock*)s.pres->getBlocksInfo()[b].ptrBlock)(ix, iy).s;
    case 4: return &(*(ScalarBlock*)s.tmp->getBlocksInfo()[b].ptrBlock)(ix, iy).s;
    case 5: return &(*(VectorBlock*)s.uDef->getBlocksInfo()[b].ptrBlock)(ix, iy).u[0];
    case 6: return &(*(VectorBlock*)s.uDef->getBlocksInfo()[b].ptrBlock)(ix, iy).u[1];
    case 7: return &(*(ScalarBlock*)s.invRho->getBlocksInfo()[b].ptrBlock)(ix, iy).s;
    case 8: return &(*(VectorBlock*)s.tmpV->getBlocksInfo()[b].ptrBlock)(ix, iy).u[0];
    case 9: return &(*(VectorBlock*)s.tmpV->getBlocksInfo()[b].ptrBlock)(ix, iy).u[1];
    default: return nullptr;
  }
}

thread_local std::string g_err;


} // namespace

extern "C" {

// Number of doubles written by ref_get_shape (same order as cup2d_shape_state).
int ref_shape_nfields(void) { return 42; }

const char* ref_last_error(void) { return g_err.c_str(); }

void* ref_create(const char* argline) {
  try {
    RefSim* r = new RefSim(argline);
    char cwd[4096];
    const bool haveCwd = getcwd(cwd, sizeof(cwd)) != nullptr;
    // fish constructors write "initialCheck" midline files into the cwd
    if (chdir("/tmp") != 0) { /* keep going in the current directory */ }
    r->init();
    if (haveCwd && chdir(cwd) != 0) { /* ignore */ }
    return r;
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}
void ref_destroy(void* h) { delete (RefSim*)h; }
int ref_nx(void* h) { return ((RefSim*)h)->sim.bpdx * _BS_; }
int ref_ny(void* h) { return ((RefSim*)h)->sim.bpdy * _BS_; }
double ref_h(void* h) { return ((RefSim*)h)->sim.getH(); }
double ref_time(void* h) { return ((RefSim*)h)->sim.time; }
int ref_stepid(void* h) { return ((RefSim*)h)->sim.step; }
double ref_dt(void* h) { return ((RefSim*)h)->sim.dt; }
double ref_lambda(void* h) { return ((RefSim*)h)->sim.lambda; }
void ref_uinf(void* h, double* out) { out[0] = ((RefSim*)h)->sim.uinfx; out[1] = ((RefSim*)h)->sim.uinfy; }
void ref_set_uinf(void* h, double ux, double uy) { ((RefSim*)h)->sim.uinfx = ux; ((RefSim*)h)->sim.uinfy = uy; }
void ref_set_time(void* h, double t, int step, double dt) {
  RefSim* r = (RefSim*)h; r->sim.time = t; r->sim.step = step; r->sim.dt = dt;
}

double ref_calc_dt(void* h) { return ((RefSim*)h)->calcMaxTimestep(); }
int ref_advance(void* h) { return ((RefSim*)h)->advance(((RefSim*)h)->sim.dt) ? 1 : 0; }
double ref_max_u(void* h) { const auto op = findMaxU(((RefSim*)h)->sim); return op.run(); }

// Iterations of the last PressureIterator_unif or PressureVarRho_approx
// call (its oldNsteps), or -1 when the pipeline runs PressureSingle.
int ref_iterations(void* h) {
  Operator* p = ((RefSim*)h)->pipeline[2];
  if (auto* op = dynamic_cast<PressureIterator_unif*>(p)) return op->*member_of(IterCountTag());
  if (auto* op = dynamic_cast<PressureVarRho_approx*>(p)) return op->*member_of(VarRhoCountTag());
  return -1;
}
// SimulationData::gravity (SimulationData.h:57), fixed at (0, -9.8) there
void ref_set_gravity(void* h, double gx, double gy) {
  ((RefSim*)h)->sim.gravity[0] = gx; ((RefSim*)h)->sim.gravity[1] = gy;
}
int ref_variable_density(void* h) { return ((RefSim*)h)->sim.bVariableDensity ? 1 : 0; }
// OpenMP threads of the reference's parallel loops (returns the previous
// count): one thread gives the order-dependent loops their sequential result
int ref_set_threads(int n) { const int old = omp_get_max_threads(); omp_set_num_threads(n); return old; }
// PoissonSolver::solve(BSRC, BDST) of a solver made by the reference's own
// factory (PoissonSolver.cpp:23-59) on scalar fields (2 chi, 3 pres, 4 tmp,
// 7 invRho); returns -1 for a non-scalar field
int ref_poisson_solve(void* h, int src, int dst) {
  SimulationData& s = ((RefSim*)h)->sim;
  auto grid = [&](int w) -> ScalarGrid* {
    switch (w) { case 2: return s.chi; case 3: return s.pres; case 4: return s.tmp; case 7: return s.invRho;
                 default: return nullptr; }
  };
  ScalarGrid *gs = grid(src), *gd = grid(dst);
  if (!gs || !gd) return -1;
  PoissonSolver* solver = PoissonSolver::makeSolver(s);
  solver->solve(gs->getBlocksInfo(), gd->getBlocksInfo());
  delete solver;
  return 0;
}

// The RL actuation of a StefanFish (StefanFish.cpp:373-577): act, the
// learn period, and its state relative to another shape (16 values with the
// sensors StefanFish.h:12 compiles in).  Return -1 if `id` is no StefanFish.
int ref_fish_act(void* h, int id, double t, const double* a, int na) {
  auto* f = dynamic_cast<StefanFish*>(((RefSim*)h)->sim.shapes[id]);
  if (!f) return -1;
  f->act(t, std::vector<double>(a, a + na));
  return 0;
}
void ref_set_pose(void* h, int id, double cx, double cy, double px, double py, double ang) {
  Shape* s = ((RefSim*)h)->sim.shapes[id];
  double com[2] = {cx, cy};
  s->setCenterOfMass(com);
  s->center[0] = px; s->center[1] = py;
  s->setOrientation(ang);
}
// Shape::u, v, omega (Shape.h:45-47): a forced body keeps them (Shape.cpp:52-59)
void ref_set_shape_velocity(void* h, int id, double u, double v, double omega) {
  Shape* s = ((RefSim*)h)->sim.shapes[id];
  s->u = u; s->v = v; s->omega = omega;
}
double ref_fish_period(void* h, int id) {
  auto* f = dynamic_cast<StefanFish*>(((RefSim*)h)->sim.shapes[id]);
  return f ? f->getLearnTPeriod() : -1;
}
int ref_fish_state(void* h, int id, int other, double* out) {
  RefSim* r = (RefSim*)h;
  auto* f = dynamic_cast<StefanFish*>(r->sim.shapes[id]);
  if (!f) return -1;
  const std::vector<double> s = f->state(r->sim.shapes[other]);
  for (size_t i = 0; i < s.size(); i++) out[i] = s[i];
  return (int)s.size();
}

// op: 0 PutObjectsOnGrid, 1 advDiff, 2 PressureSingle, 3 ComputeForces
void ref_run_op(void* h, int op, double dt) { (*((RefSim*)h)->pipeline[op])(dt); }
void ref_reset(void* h) { ((RefSim*)h)->reset(); ((RefSim*)h)->sim.dt = 0; }

// which: 0 u, 1 v, 2 chi, 3 pres, 4 tmp, 5 uDef x, 6 uDef y, 7 invRho, 8/9 tmpV
void ref_get_field(void* h, int which, double* out) {
  RefSim* r = (RefSim*)h;
  for_cells(r, [&](size_t b, int ix, int iy, long g) { out[g] = *field_ptr(r, which, b, ix, iy); });
}
void ref_set_field(void* h, int which, const double* in) {
  RefSim* r = (RefSim*)h;
  for_cells(r, [&](size_t b, int ix, int iy, long g) { *field_ptr(r, which, b, ix, iy) = in[g]; });
}

int ref_nshapes(void* h) { return (int)((RefSim*)h)->sim.shapes.size(); }

void ref_get_shape(void* h, int id, double* o) {
  const Shape* s = ((RefSim*)h)->sim.shapes[id];
  const double v[] = {
    s->center[0], s->center[1], s->centerOfMass[0], s->centerOfMass[1],
    s->orientation, s->u, s->v, s->omega, s->M, s->J,
    s->d_gm[0], s->d_gm[1], s->labCenterOfMass[0], s->labCenterOfMass[1],
    s->penalM, s->penalJ, s->penalDX, s->penalDY,
    s->fluidMomX, s->fluidMomY, s->fluidAngMom,
    s->perimeter, s->forcex, s->forcey, s->forcex_P, s->forcey_P,
    s->forcex_V, s->forcey_V, s->torque, s->torque_P, s->torque_V,
    s->drag, s->thrust, s->circulation, s->Pout, s->PoutBnd,
    s->defPower, s->defPowerBnd, s->Pthrust, s->Pdrag, s->EffPDef, s->EffPDefBnd};
  std::memcpy(o, v, sizeof(v));
}

// Per-block obstacle data of one shape: for every touched block, the block
// index followed by chi, dist, udef_x, udef_y (BS*BS each, row-major) and the
// surface list count + (ix, iy, dchidx, dchidy, delta) tuples.  Returns the
// number of doubles written (or needed when out == nullptr).
long ref_get_obstacle(void* h, int id, double* out) {
  const Shape* s = ((RefSim*)h)->sim.shapes[id];
  long n = 0;
  auto put = [&](double x) { if (out) out[n] = x; n++; };
  for (size_t b = 0; b < s->obstacleBlocks.size(); b++) {
    const ObstacleBlock* o = s->obstacleBlocks[b];
    if (o == nullptr) continue;
    put((double)b);
    for (int iy = 0; iy < _BS_; iy++) for (int ix = 0; ix < _BS_; ix++) put(o->chi[iy][ix]);
    for (int iy = 0; iy < _BS_; iy++) for (int ix = 0; ix < _BS_; ix++) put(o->dist[iy][ix]);
    for (int iy = 0; iy < _BS_; iy++) for (int ix = 0; ix < _BS_; ix++) put(o->udef[iy][ix][0]);
    for (int iy = 0; iy < _BS_; iy++) for (int ix = 0; ix < _BS_; ix++) put(o->udef[iy][ix][1]);
    put((double)o->n_surfPoints);
    for (size_t k = 0; k < o->n_surfPoints; k++) {
      put(o->surface[k]->ix); put(o->surface[k]->iy);
      put(o->surface[k]->dchidx); put(o->surface[k]->dchidy); put(o->surface[k]->delta);
    }
  }
  return n;
}

// Per-stage wall seconds accumulated by the Profiler stand-in.
int ref_profile(void* h, char* names, int names_len, double* secs, int max_n) {
  auto* p = ((RefSim*)h)->sim.profiler;
  int i = 0; std::string all;
  for (auto& kv : p->seconds) {
    if (i >= max_n) break;
    secs[i++] = kv.second;
    all += kv.first; all += ";";
  }
  if (names && names_len > 0) {
    std::strncpy(names, all.c_str(), names_len - 1);
    names[names_len - 1] = 0;
  }
  return i;
}
void ref_profile_reset(void* h) {
  auto* p = ((RefSim*)h)->sim.profiler;
  p->seconds.clear(); p->calls.clear();
}

} // extern "C"
