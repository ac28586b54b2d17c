// config.h -- case-file reader (the reference's configuration::SimConfig) and the
// lattice tables of one rank (the reference's geometry::LatticeData).
#pragma once

#include <algorithm>
#include <complex>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/hemeb200.h"
#include "hb_common.h"

namespace hb {

// What SimConfig::DoIO extracts for the collide-and-stream path, converted to
// lattice units by the reference's UnitConverter (src/util/UnitConverter.cc:15-118).
struct CaseConfig {
  std::string gmy_path;
  double dt = 0, dx = 0;
  double origin[3] = {0, 0, 0};
  uint64_t total_steps = 0;       // <steps> + <extra_warmup_steps>
  uint64_t warmup = 0;
  hb_params params{};
  struct PropertyOutput {
    std::string file;
    uint64_t period = 0;
    std::string geometry;
    std::vector<std::string> fields;
  };
  std::vector<PropertyOutput> outputs;
  std::vector<double> tables[32];  // file iolets' tables (inlets 0-15, outlets 16-31)
  std::string checkpoint_file;    // <initialconditions><checkpoint file=...>
  bool has_time = false;          // <initialconditions><time> present
};

// SimConfig::New + DoIO (src/configuration/SimConfig.cc:41-121).  `kernel` decides
// which kernel-specific elements are required, as HEMELB_KERNEL does.
CaseConfig read_case(const std::string& xml_path, int kernel);

// A host array of plain values whose resize leaves new elements unset: the
// large site tables (coordinates, cut distances, normals: 124 bytes a site) are
// written in full by whoever fills them, and a zero fill first would cost as
// much as the copy from the device.  Large arrays are aligned to 2 MiB and
// advised as huge-page candidates, so that first touching them takes a few
// hundred page faults instead of a hundred thousand.  The subset of std::vector
// the tables use.
void* host_table_alloc(size_t bytes);
void host_table_free(void* p);

template <class T>
class HostArray {
 public:
  using value_type = T;
  HostArray() = default;
  HostArray(const HostArray& o) { assign(o.begin(), o.end()); }
  HostArray(HostArray&& o) noexcept : p_(o.p_), n_(o.n_) {
    o.p_ = nullptr;
    o.n_ = 0;
  }
  HostArray& operator=(const HostArray& o) {
    if (this != &o) assign(o.begin(), o.end());
    return *this;
  }
  HostArray& operator=(HostArray&& o) noexcept {
    if (this != &o) {
      host_table_free(p_);
      p_ = o.p_;
      n_ = o.n_;
      o.p_ = nullptr;
      o.n_ = 0;
    }
    return *this;
  }
  ~HostArray() { host_table_free(p_); }

  size_t size() const { return n_; }
  bool empty() const { return n_ == 0; }
  T* data() { return p_; }
  const T* data() const { return p_; }
  T* begin() { return p_; }
  T* end() { return p_ + n_; }
  const T* begin() const { return p_; }
  const T* end() const { return p_ + n_; }
  T& operator[](size_t k) { return p_[k]; }
  const T& operator[](size_t k) const { return p_[k]; }
  void clear() {
    host_table_free(p_);
    p_ = nullptr;
    n_ = 0;
  }
  // New elements are left unset; old ones are kept.
  void resize(size_t n) {
    if (n == n_) return;
    T* q = n ? static_cast<T*>(host_table_alloc(n * sizeof(T))) : nullptr;
    for (size_t k = 0; k < std::min(n, n_); k++) q[k] = p_[k];
    host_table_free(p_);
    p_ = q;
    n_ = n;
  }
  template <class It>
  void assign(It first, It last) {
    const size_t n = (size_t)(last - first);
    T* q = n ? static_cast<T*>(host_table_alloc(n * sizeof(T))) : nullptr;
    for (size_t k = 0; k < n; k++) q[k] = (T)first[k];
    host_table_free(p_);
    p_ = q;
    n_ = n;
  }
  void assign(size_t n, T v) {
    clear();
    resize(n);
    for (size_t k = 0; k < n; k++) p_[k] = v;
  }

 private:
  T* p_ = nullptr;
  size_t n_ = 0;
};

// Lattice tables in the reference's contiguous order
// (src/geometry/LatticeData.cc:69-285, 366-443; LatticeData.h:375-436).
struct LatticeTables {
  int64_t n = 0;
  int64_t dims[3] = {0, 0, 0};
  int64_t block_size = 0;
  int64_t blocks[3] = {0, 0, 0};
  int64_t type_counts[6] = {0, 0, 0, 0, 0, 0};
  HostArray<int64_t> coords;        // [n*3]
  std::vector<uint32_t> wall;       // [n]
  std::vector<uint32_t> iolet;      // [n]
  std::vector<int32_t> stype;       // [n] 0 fluid 1 inlet 2 outlet
  std::vector<int32_t> iolet_id;    // [n]
  HostArray<float> q;               // [n*18] cut distances as the .gmy stores them (float; -1 no wall link)
  HostArray<float> normal;          // [n*3] wall normal, normalised in float (HUGE_VALF without one)
  std::vector<int64_t> nbr;         // [n*19] neighbourIndices, or empty: derived from the coordinates
                                    // when asked for (neighbour_table)
  // One slab of a sharded lattice: sites [0, n_owned) are this shard's own, in
  // the reference's order; sites [n_owned, n) are halo sites of the neighbouring
  // slabs, whose post-collision values arrive every step.  -1: all sites owned.
  int64_t n_owned = -1;
  std::vector<int64_t> gid;         // [n] global contiguous index of each site (shards only)

  int64_t owned() const { return n_owned >= 0 ? n_owned : n; }

  int collision_type(int64_t i) const {
    const bool w = wall[i] != 0;
    const int st = stype[i];
    return !w ? (st == 0 ? 0 : (st == 1 ? 2 : 3)) : (st == 0 ? 1 : (st == 1 ? 4 : 5));
  }
};

// InOutLetVelocity::GetVelocity on the host for the velocity iolets (parabolic,
// file velocity, Womersley) at lattice position x and 1-based step t.  Returns 0,
// or HB_ERR_IOLET_RADIUS for a parabolic or file-velocity point outside the radius.
int iolet_velocity(const hb_iolet& io, const double x[3], uint64_t t, double v[3]);
// The Womersley profile split into its time-independent factor at x,
// A(x) = G / (rho omega) (1 - J0(i^(3/2) alpha r / R) / J0(i^(3/2) alpha)), and
// its phase exp(i omega t); the speed is Re(A exp(i omega t)) along -normal.
std::complex<double> womersley_amplitude(const hb_iolet& io, const double x[3]);
std::complex<double> womersley_phase(const hb_iolet& io, uint64_t t);
// util::BesselJ0ComplexArgument (src/util/Bessel.cc:17-43).
std::complex<double> bessel_j0(const std::complex<double>& z, double tol_sq = 1e-12);

// GeometryReader::LoadAndDecompose on one rank + LatticeData construction.
LatticeTables read_gmy(const std::string& path);
// neighbourIndices from coordinates (LatticeData::InitialiseNeighbourLookup), into
// out[n*19]; t.nbr itself when the tables carry one.
void neighbour_table(const LatticeTables& t, int64_t* out);
// Fills t.nbr.
void build_neighbours(LatticeTables& t);

// The same tables with the site records decoded, binned and linked on the GPU
// (gmy_device.cu); wall-clock milliseconds of its phases in `timing`.
struct GmyTiming {
  double read_ms = 0, inflate_ms = 0, h2d_ms = 0, device_ms = 0, d2h_ms = 0;
};
// With `layout`, the storage layout for `params` and `wall` is built on the
// device from the decoded tables while they are copied back to the host.
struct Layout;
LatticeTables read_gmy_device(const std::string& path, int device, GmyTiming* timing = nullptr,
                              const hb_params* params = nullptr, int wall = 0, Layout* layout = nullptr);

}  // namespace hb
