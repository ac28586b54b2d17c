// hemeb200_lbm.hpp -- C++ host class with the method set of the reference's
// lb::LBM<LatticeType> (src/lb/lb.h:32-148), implemented over the C ABI in
// hemeb200.h.  A HemePure build replaces the body of its LBM with this class:
// the construction takes the tables LatticeData already holds, the per-step
// phases keep their names and order, and errors surface as exceptions the way
// hemelb::Exception does (an instability sets a flag instead, as
// SimulationState::SetStability(Unstable) does).
#ifndef HEMEB200_LBM_HPP
#define HEMEB200_LBM_HPP

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "hemeb200.h"

namespace hemeb200 {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

class LBM {
 public:
  // The constructor + Initialise + SetInitialConditions of the reference.
  LBM(const hb_lattice_desc& lattice, const hb_params& params, const hb_options& options) {
    check_create(hb_create(&lattice, &params, &options, &h_));
  }
  // The same from a case file (SimConfig + GeometryReader + LatticeData inside).
  LBM(const std::string& xml_path, const hb_options& options) {
    check_create(hb_create_from_xml(xml_path.c_str(), &options, &h_));
  }
  LBM(const LBM&) = delete;
  LBM& operator=(const LBM&) = delete;
  ~LBM() {
    if (h_) hb_destroy(h_);
  }

  // Per-step phases, in the order net::phased::StepManager calls them.
  void RequestComms() { check(hb_request_comms(h_)); }
  void PreSend() { check(hb_pre_send(h_)); }
  // `fill_property_cache` fills density, velocity and wall shear stress; with
  // `fill_stress_caches` also the von Mises, shear-rate, stress-tensor and traction caches.
  void PreReceive(bool fill_property_cache = false, bool fill_stress_caches = false) {
    check(hb_pre_receive(h_, (fill_property_cache ? HB_STEP_MACRO : 0u) |
                                 (fill_property_cache && fill_stress_caches ? HB_STEP_STRESS : 0u)));
  }
  void PostReceive() { check(hb_post_receive(h_)); }
  void EndIteration() { check(hb_end_iteration(h_)); }

  hb_params GetLbmParams() const {
    hb_params p;
    check(hb_get_params(h_, &p));
    return p;
  }
  int64_t GetLocalFluidSiteCount() const {
    int64_t n = 0;
    check(hb_site_count(h_, &n));
    return n;
  }
  uint64_t GetTimeStep() const {
    uint64_t t = 0;
    check(hb_time_step(h_, &t));
    return t;
  }
  // LatticeData::GetFOld over all sites, AoS in contiguous site order.
  std::vector<double> GetFOld() const {
    std::vector<double> f(19 * (size_t)GetLocalFluidSiteCount());
    check(hb_get_fs(h_, f.data()));
    return f;
  }
  void SetFs(const std::vector<double>& f) { check(hb_set_fs(h_, f.data())); }
  // MacroscopicPropertyCache: density, velocity (x,y,z per site), wall shear stress.
  void GetPropertyCache(std::vector<double>& density, std::vector<double>& velocity, std::vector<double>& wss) const {
    const size_t n = (size_t)GetLocalFluidSiteCount();
    density.resize(n);
    velocity.resize(3 * n);
    wss.resize(n);
    check(hb_get_macro(h_, density.data(), velocity.data(), wss.data()));
  }
  // One stress cache (HB_STRESS_*) of the last step run with the stress caches:
  // 1, 6 (xx, xy, xz, yy, yz, zz) or 3 values per site, contiguous site order.
  std::vector<double> GetStressCache(int field) const {
    const size_t per = field == HB_STRESS_TENSOR ? 6 : (field >= HB_STRESS_TRACTION ? 3 : 1);
    std::vector<double> out(per * (size_t)GetLocalFluidSiteCount());
    check(hb_get_stress(h_, field, out.data()));
    return out;
  }
  // BoundaryValues::GetBoundaryDensity from the caller's own iolets, per inlet and
  // outlet, for the cosine and file pressure iolets from the next step on.
  void SetIoletDensities(const std::vector<double>& inlets, const std::vector<double>& outlets) {
    check(hb_set_iolet_densities(h_, inlets.data(), (int)inlets.size(), outlets.data(), (int)outlets.size()));
  }
  void ClearIoletDensities() { check(hb_set_iolet_densities(h_, nullptr, 0, nullptr, 0)); }
  bool IsUnstable() const { return unstable_; }
  hb_handle* handle() const { return h_; }

 private:
  void check(int rc) const {
    if (rc == HB_OK) return;
    if (rc == HB_UNSTABLE) {
      unstable_ = true;
      return;
    }
    char msg[512];
    hb_last_error(h_, msg, sizeof msg);
    throw Error(rc, msg);
  }
  void check_create(int rc) {
    if (rc == HB_OK) return;
    char msg[512];
    hb_last_error(nullptr, msg, sizeof msg);
    throw Error(rc, msg);
  }
  hb_handle* h_ = nullptr;
  mutable bool unstable_ = false;
};

}  // namespace hemeb200

#endif  // HEMEB200_LBM_HPP
