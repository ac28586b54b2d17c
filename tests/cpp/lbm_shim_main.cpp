// Drives the C++ class of include/hemeb200_lbm.hpp the way HemePure's
// SimulationMaster drives lb::LBM: the five phases per step, the property
// and stress caches on the last step, then GetFOld, GetPropertyCache and the
// stress tensor and traction caches.  Writes the
// results as raw little-endian doubles for the test to compare.
//
//   lbm_shim_main <case.xml> <steps> <kernel 0|1|2> <wall 0|1|2> <out.bin>
//
// Exit status: 0 on success, 1 on a usage error, 2 when the library reports an
// error (the message goes to stderr), 3 when the run went unstable.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <vector>

#include "hemeb200_lbm.hpp"

int main(int argc, char** argv) {
  if (argc != 6) {
    std::fprintf(stderr, "usage: %s case.xml steps kernel wall out.bin\n", argv[0]);
    return 1;
  }
  const long steps = std::atol(argv[2]);
  hb_options opt;
  hb_default_options(&opt);
  opt.kernel = std::atoi(argv[3]);
  opt.wall = std::atoi(argv[4]);
  try {
    hemeb200::LBM lbm(argv[1], opt);
    for (long t = 0; t < steps; t++) {
      lbm.RequestComms();
      lbm.PreSend();
      lbm.PreReceive(t == steps - 1, true);
      lbm.PostReceive();
      lbm.EndIteration();
    }
    if (lbm.IsUnstable()) return 3;
    const std::vector<double> f = lbm.GetFOld();
    std::vector<double> rho, u, wss;
    lbm.GetPropertyCache(rho, u, wss);
    const int64_t n = lbm.GetLocalFluidSiteCount();
    const uint64_t t = lbm.GetTimeStep();
    std::ofstream out(argv[5], std::ios::binary);
    out.write(reinterpret_cast<const char*>(&n), sizeof n);
    out.write(reinterpret_cast<const char*>(&t), sizeof t);
    const std::vector<double> tensor = lbm.GetStressCache(HB_STRESS_TENSOR);
    const std::vector<double> traction = lbm.GetStressCache(HB_STRESS_TRACTION);
    const std::vector<double>* fields[] = {&f, &rho, &u, &wss, &tensor, &traction};
    for (const std::vector<double>* v : fields)
      out.write(reinterpret_cast<const char*>(v->data()), (std::streamsize)(v->size() * sizeof(double)));
    return out ? 0 : 2;
  } catch (const hemeb200::Error& e) {
    std::fprintf(stderr, "hemeb200 error %d: %s\n", e.code(), e.what());
    return 2;
  }
}
