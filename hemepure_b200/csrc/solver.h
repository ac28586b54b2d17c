// solver.h -- one lattice resident on one GPU (the state behind an hb_handle).
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "../../include/hemeb200.h"
#include "config.h"
#include "device.h"
#include "layout.h"

namespace hb {

struct DeviceBuffer {
  void* p = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer();
  void alloc(size_t b);
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

// The checks of a case's parameters and options that need no lattice (the
// solver's constructor runs them first); throws hb::Error.
void validate_case(const hb_params& p, const hb_options& o);

class Solver {
 public:
  // `layout`, when given, is the storage layout already built for these tables,
  // parameters and wall rule (moved from); otherwise it is built here.
  Solver(LatticeTables tables, const hb_params& params, const hb_options& opt, Layout* layout = nullptr);
  ~Solver();

  // lb::LBM phases.
  void request_comms();
  // `stress` (with `macro`) also stores the momentum flux tensor for the stress caches.
  void pre_receive(bool macro, int which = 3, bool stress = false);
  void end_iteration();
  int step(int64_t n, uint32_t flags);
  // `n` steps with CUDA events around each launch: ms[0] plain bulk kernel,
  // ms[1] general kernel, ms[2] Windkessel kernel (summed over the steps).
  int profile(int64_t n, double ms[3]);
  // Total density and momentum of the distributions entering the next step.
  void moment_sums(double out[4]);

  void get_fs(double* f);
  void set_fs(const double* f);
  void get_macro(double* rho, double* u, double* wss);
  // Stress cache HB_STRESS_* of the last stress step, AoS in reference order.
  void get_stress(int field, double* out);
  static int stress_len(int field);
  void get_wk3(int group, int index, double st[4]);
  // Densities of the pressure iolets (cosine and file) supplied by the caller,
  // replacing the ones computed from the case from the next step on; null clears.
  void set_iolet_densities(const double* inlets, int n_inlets, const double* outlets, int n_outlets);

  const LatticeTables& tables() const { return t_; }
  const Layout& layout() const { return L_; }
  const hb_params& params() const { return p_; }
  uint64_t time_step() const { return t_step_; }
  double last_ms() const { return last_ms_; }
  int64_t last_launches() const { return last_launches_; }
  int64_t device_bytes() const { return dev_bytes_; }
  int read_status();

  // Physical scales for output (UnitConverter): time step, voxel size, origin.
  void set_units(double dt, double dx, const double origin[3]);
  double dt() const { return dt_; }
  double dx() const { return dx_; }
  const double* origin() const { return origin_; }
  bool macro_valid() const { return macro_valid_; }
  bool stress_valid() const { return stress_valid_; }
  // Pre-collision f of the last completed step (what the reference's GetFNew
  // returns after EndIteration), AoS in reference order.  False if no step has
  // run since the last set_fs / get_fs.
  bool get_previous_fs(double* f);
  void set_time_step(uint64_t t) { t_step_ = t; }

  // Exact FP64 restart: the distributions entering the next step, the time
  // step, and the Windkessel state with the coupling contributions the next
  // step's flow sum reads (FP64 storage only).
  void write_state(const std::string& path);
  void read_state(const std::string& path);

  // The sites a geometry selector takes (reference order) and the requested
  // data of those sites only, selected and gathered on the device so that only
  // they cross to the host: density, velocity, WSS of the last output step
  // [m], [m*3], [m]; stress caches [m*k]; pre-collision f of the last step [m*19].
  struct Selection {
    std::vector<int> idx;
    std::vector<double> rho, u, wss, fd;
    std::vector<double> stress[6];
  };
  Selection select(const hb_selector& sel, bool macro, const bool stress[6], bool distributions);

  // Sharded form (tables cut by cut_shard): the halo lists of the slab
  // [lo, hi) along `axis`; then, after every step, pack the values the two
  // neighbours pull and, before the next, unpack theirs.  Both run on the
  // solver's stream, ordered against the caller's stream by events.
  void attach_shard(int axis, int64_t lo, int64_t hi);
  bool sharded() const { return shard_; }
  // Elements sent to the lower / upper neighbour, received from them.
  void shard_sizes(int64_t counts[4]) const;
  int elem_size() const { return (int)elem_bytes(); }
  void shard_pack(void* to_lower, void* to_upper, cudaStream_t caller);
  void shard_unpack(const void* from_lower, const void* from_upper, cudaStream_t caller);

 private:
  void upload();
  void materialise();
  void ensure_macro();
  void fill_density_rows(uint64_t t_first, int count);
  // Index of step t's iolet row in the device table, refilling the table with
  // the rows of steps t .. t + 1023 when t lies outside the resident window.
  int density_row(uint64_t t, int64_t steps_ahead);
  StepArgs args() const;
  void check(cudaError_t e, const char* what);
  bool mixed() const { return opt_.precision != HB_STORE_FP64; }
  size_t elem_bytes() const { return opt_.precision == HB_STORE_FP64 ? 8 : (opt_.precision == HB_STORE_FP32 ? 4 : 2); }
  void launch(const StepArgs& a, bool macro, int which, cudaStream_t st);
  void to_aos(bool use_prev, double* dev_aos);

  LatticeTables t_;
  hb_params p_;
  std::vector<double> tables_[32];  // file iolets' tables (p_ points into them)
  hb_options opt_;
  Layout L_;
  cudaStream_t stream_ = nullptr;
  cudaStream_t side_ = nullptr;   // boundary kernel, concurrent with the bulk kernel
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  cudaStream_t side2_ = nullptr;  // the boundary records with iolet links, beside the others
  cudaEvent_t fork_ = nullptr, join_ = nullptr, join2_ = nullptr;

  DeviceBuffer f_[2];
  DeviceBuffer ghost_[2];         // iolet ghost values, paired with f_
  int cur_ = 0;
  bool direct_ = true;            // f_[cur_] holds pre-collision f (else post-collision f*)
  DeviceBuffer meta_, run_off_, run_po_, st2ref_;
  DeviceBuffer g_run_;
  DeviceBuffer g_site_, g_wall_, g_iolet_, g_src_, g_q_, g_nrm_, g_io_, g_cpl_, g_xyz_;
  DeviceBuffer g_wom_, wom_amp_;     // Womersley link factors (allocated only with such an iolet)
  DeviceBuffer vtau_, iolets_, dens_, cpl_buf_, wk3_, status_;
  DeviceBuffer rho_, u_, wss_;
  DeviceBuffer pi_, stress_out_;  // allocated at the first stress step
  DeviceBuffer sum_scratch_, sum_out_;
  int dens_rows_ = 0;
  int row_ = 0;                   // row of the density table used by the current step
  // Pinned, so a step's row upload is a direct asynchronous copy; rows_ev_ marks
  // when the last upload has read it, before the next fill rewrites it.
  double* host_rows_ = nullptr;
  cudaEvent_t rows_ev_ = nullptr;
  bool rows_pending_ = false;
  bool rows_valid_ = false;         // the device table holds the rows of steps rows_first_ ...
  uint64_t rows_first_ = 0;
  int rows_count_ = 0;              // rows uploaded at rows_first_
  bool dens_override_ = false;
  double dens_override_v_[32] = {};  // inlets 0-15, outlets 16-31
  int nwk3_ = 0;
  bool macro_valid_ = false;
  bool phase_open_ = false;
  bool phase_macro_ = false;
  bool stress_valid_ = false;
  bool phase_stress_ = false;
  uint64_t t_step_ = 1;
  double omega_ = 0, omega_minus_ = 0;
  double last_ms_ = 0;
  int64_t last_launches_ = 0;
  int64_t dev_bytes_ = 0;
  int status_sticky_ = 0;
  int* status_host_ = nullptr;    // pinned host copy of the status word
  bool prev_valid_ = false;
  bool prev_direct_ = false;
  double dt_ = 1.0, dx_ = 1.0;
  double origin_[3] = {0, 0, 0};
  // Device copies of the tables a selector reads (made at the first selection).
  DeviceBuffer sel_coords_, sel_wall_, sel_stype_, ref2st_;
  // Pre-collision f of the last completed step, AoS in reference order, into a device buffer.
  bool previous_aos_device(double* aos);
  // Sharded form.
  bool shard_ = false;
  int64_t send_n_[2] = {0, 0}, recv_n_[2] = {0, 0};
  DeviceBuffer send_idx_[2], recv_idx_[2];
  cudaEvent_t xev_ = nullptr;
};

}  // namespace hb
