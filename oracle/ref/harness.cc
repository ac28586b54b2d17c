// Driver for HemePure's own solver built as the CPU oracle (test infrastructure only).
//
// It wires the reference's objects together the way SimulationMaster::Initialise
// does (src/SimulationMaster.cc:126-285) — GeometryReader, LatticeData,
// NeighbouringDataManager, LBM, StabilityTester, the two BoundaryValues and the
// phased StepManager — without colloids, images or reports, runs a number of
// time steps as SimulationMaster::DoTimeStep does (src/SimulationMaster.cc:335-375),
// and writes the distributions and the macroscopic caches of the last step to a
// binary dump in the reference's contiguous site order.
//
// usage: hemepure_ref <config.xml> <output-dir> <steps> <dump-file | -> [warm-up steps]
//
// Warm-up steps run before the timed loop (and before the start barrier below)
// and count toward the step total.
//
// Dump layout (little-endian): char[8] "HBREFDMP", int64 n_sites, int64 steps_done,
// int64 stability, then int64 coords[n][3], double f_old[n][19], double rho[n],
// double u[n][3], double wss[n].  A dump file of "-" writes nothing (timing runs).
//
// For timing several copies side by side: with HB_REF_READY=<dir> set, the run
// creates <dir>/ready.<pid> once set up and waits (at most ten minutes) for
// <dir>/go before its first step.  The last stderr line gives the stepping
// loop's start and end on CLOCK_MONOTONIC, comparable across processes.
#include <time.h>
#include <unistd.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "configuration/CommandLine.h"
#include "configuration/SimConfig.h"
#include "geometry/GeometryReader.h"
#include "geometry/LatticeData.h"
#include "geometry/neighbouring/NeighbouringDataManager.h"
#include "lb/StabilityTester.h"
#include "lb/iolets/BoundaryValues.h"
#include "lb/lattices/Lattices.h"
#include "lb/lb.hpp"
#include "log/Logger.h"
#include "net/IOCommunicator.h"
#include "net/mpi.h"
#include "net/net.h"
#include "net/phased/NetConcern.h"
#include "net/phased/StepManager.h"
#include "net/BuildInfo.h"
#include "io/PathManager.h"
#include "reporting/Timers.h"
#include "util/UnitConverter.h"

// SimulationMaster.cc defines this global; the LES sponge-layer kernel reads it.
double hemelb::tau_;

namespace {

typedef hemelb::lb::lattices::HEMELB_LATTICE Lattice;

double monotonic() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

// Start barrier between copies timed side by side (see the header comment).
void wait_for_go() {
  const char* dir = std::getenv("HB_REF_READY");
  if (!dir || !*dir) return;
  const std::string ready = std::string(dir) + "/ready." + std::to_string((long)getpid());
  if (FILE* f = std::fopen(ready.c_str(), "w")) std::fclose(f);
  const std::string go = std::string(dir) + "/go";
  const double until = monotonic() + 600.0;
  while (access(go.c_str(), F_OK) != 0 && monotonic() < until) usleep(1000);
}

template <class T>
void put(FILE* f, const T* p, size_t n) {
  if (std::fwrite(p, sizeof(T), n, f) != n) {
    std::perror("write");
    std::exit(3);
  }
}

int run(int argc, char** argv) {
  using namespace hemelb;
  if (argc < 5) {
    std::fprintf(stderr, "usage: %s config.xml outdir steps dump\n", argv[0]);
    return 2;
  }
  const long steps = std::atol(argv[3]);
  const std::string dump = argv[4];
  const long warmup = argc > 5 ? std::atol(argv[5]) : 0;

  net::MpiCommunicator commWorld = net::MpiCommunicator::World();
  net::IOCommunicator ioComms(commWorld);

  const char* cl[] = {argv[0], "-in", argv[1], "-out", argv[2]};
  configuration::CommandLine options(5, cl);
  io::PathManager fileManager(options, ioComms.OnIORank(), ioComms.Size());
  configuration::SimConfig* simConfig = configuration::SimConfig::New(fileManager.GetInputFile());
  const util::UnitConverter* unitConverter = &simConfig->GetUnitConverter();
  const configuration::SimConfig::MonitoringConfig* monitoring = simConfig->GetMonitoringConfiguration();

  reporting::Timers timings(ioComms);
  net::Net communicationNet(ioComms);

  lb::SimulationState* simulationState =
      new lb::SimulationState(simConfig->GetTimeStepLength(), simConfig->GetTotalTimeSteps());

  geometry::GeometryReader reader(Lattice::GetLatticeInfo(), timings, ioComms);
  geometry::Geometry readGeometryData = reader.LoadAndDecompose(simConfig->GetDataFilePath());
  geometry::LatticeData* latticeData =
      new geometry::LatticeData(Lattice::GetLatticeInfo(), readGeometryData, ioComms);

  geometry::neighbouring::NeighbouringDataManager* neighbouringDataManager =
      new geometry::neighbouring::NeighbouringDataManager(*latticeData, latticeData->GetNeighbouringData(),
                                                          communicationNet);

  lb::LBM<Lattice>* lbm = new lb::LBM<Lattice>(simConfig, &communicationNet, latticeData, simulationState,
                                               timings, neighbouringDataManager);
  hemelb::tau_ = lbm->GetLbmParams()->GetTau();

  lb::StabilityTester<Lattice>* stabilityTester =
      new lb::StabilityTester<Lattice>(latticeData, &communicationNet, simulationState, timings, monitoring);

  lb::iolets::BoundaryValues* inletValues = new lb::iolets::BoundaryValues(
      geometry::INLET_TYPE, latticeData, simConfig->GetInlets(), simulationState, ioComms, *unitConverter);
  lb::iolets::BoundaryValues* outletValues = new lb::iolets::BoundaryValues(
      geometry::OUTLET_TYPE, latticeData, simConfig->GetOutlets(), simulationState, ioComms, *unitConverter);

  lbm->Initialise(inletValues, outletValues, unitConverter);
  lbm->SetInitialConditions(ioComms);
  neighbouringDataManager->ShareNeeds();
  neighbouringDataManager->TransferNonFieldDependentInformation();

  net::phased::StepManager stepManager(2, &timings, net::separate_communications);
  net::phased::NetConcern netConcern(communicationNet);
  stepManager.RegisterIteratedActorSteps(*neighbouringDataManager, 0);
  stepManager.RegisterIteratedActorSteps(*lbm, 1);
  stepManager.RegisterIteratedActorSteps(*inletValues, 1);
  stepManager.RegisterIteratedActorSteps(*outletValues, 1);
  stepManager.RegisterIteratedActorSteps(*stabilityTester, 1);
  stepManager.RegisterCommsForAllPhases(netConcern);

  lb::MacroscopicPropertyCache& cache = lbm->GetPropertyCache();
  for (long s = 0; s < warmup && simulationState->GetStability() != lb::Unstable; ++s) {
    cache.ResetRequirements();
    stepManager.CallActions();
    simulationState->Increment();
  }
  long done = 0;
  wait_for_go();
  double t0 = monotonic();
  for (long s = 0; s < steps; ++s) {
    cache.ResetRequirements();
    if (s == steps - 1) {
      cache.densityCache.SetRefreshFlag();
      cache.velocityCache.SetRefreshFlag();
      cache.wallShearStressMagnitudeCache.SetRefreshFlag();
    }
    stepManager.CallActions();
    ++done;
    if (simulationState->GetStability() == lb::Unstable) break;
    simulationState->Increment();
  }
  double t1 = monotonic();

  const int64_t n = latticeData->GetLocalFluidSiteCount();
  std::fprintf(stderr, "hemepure_ref: %lld sites, %ld steps, %.3f s, loop %.6f %.6f, %.2f MLUPS\n", (long long)n,
               done, t1 - t0, t0, t1, (double)n * (double)done / (t1 - t0) / 1e6);

  if (dump == "-") return 0;
  FILE* out = std::fopen(dump.c_str(), "wb");
  if (!out) {
    std::perror(dump.c_str());
    return 3;
  }
  const int64_t head[3] = {n, (int64_t)done, (int64_t)simulationState->GetStability()};
  put(out, "HBREFDMP", 8);
  put(out, head, 3);
  std::vector<int64_t> coords(3 * n);
  std::vector<double> f(19 * n), rho(n), u(3 * n), wss(n);
  for (int64_t i = 0; i < n; ++i) {
    const geometry::Site<const geometry::LatticeData> site =
        static_cast<const geometry::LatticeData*>(latticeData)->GetSite(i);
    const util::Vector3D<site_t>& c = site.GetGlobalSiteCoords();
    coords[3 * i] = c.x;
    coords[3 * i + 1] = c.y;
    coords[3 * i + 2] = c.z;
    const distribn_t* fi = site.GetFOld<Lattice>();
    for (int d = 0; d < Lattice::NUMVECTORS; ++d) f[19 * i + d] = fi[d];
    rho[i] = cache.densityCache.Get(i);
    const util::Vector3D<distribn_t>& v = cache.velocityCache.Get(i);
    u[3 * i] = v.x;
    u[3 * i + 1] = v.y;
    u[3 * i + 2] = v.z;
    wss[i] = cache.wallShearStressMagnitudeCache.Get(i);
  }
  put(out, coords.data(), coords.size());
  put(out, f.data(), f.size());
  put(out, rho.data(), rho.size());
  put(out, u.data(), u.size());
  put(out, wss.data(), wss.size());
  std::fclose(out);

  delete outletValues;
  delete inletValues;
  delete stabilityTester;
  delete lbm;
  delete neighbouringDataManager;
  delete latticeData;
  delete simulationState;
  delete simConfig;
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  hemelb::net::MpiEnvironment mpi(argc, argv);
  hemelb::log::Logger::Init();
  try {
    return run(argc, argv);
  } catch (std::exception& e) {
    std::fprintf(stderr, "hemepure_ref: %s\n", e.what());
    return 1;
  }
}
