// batch.h -- many independent lattices resident on one GPU, stepped together.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <vector>

#include "../../include/hemeb200.h"
#include "config.h"
#include "device.h"
#include "layout.h"
#include "solver.h"

namespace hb {

// One block of the begin kernel serves every lattice slot.
constexpr int kMaxBatchLattices = 1024;

// First-fit allocator of index ranges [0, capacity).
class RangeAlloc {
 public:
  explicit RangeAlloc(int64_t capacity = 0) { reset(capacity); }
  void reset(int64_t capacity);
  int64_t take(int64_t n);   // start, or -1 when no free range fits
  void give(int64_t start, int64_t n);
  int64_t high_water() const;  // one past the highest allocated index
  int64_t capacity() const { return cap_; }

 private:
  int64_t cap_ = 0;
  std::map<int64_t, int64_t> free_;  // start -> length
  std::map<int64_t, int64_t> used_;
};

// A lattice checked and laid out on the host, ready for upload.
struct PreparedLattice {
  LatticeTables t;
  hb_params p;
  int kernel = 0, wall = 0;
  uint64_t steps = 0;
  Layout L;
  bool taken = false;
};

// Host-only: validate the physics the batched form supports and build the layout.
// The checks of a batched case that need no lattice; throws hb::Error.
void validate_batch_case(const hb_params& p, int kernel, int wall);
// `layout`, when given, is the layout already built for these tables (moved from).
std::unique_ptr<PreparedLattice> prepare_lattice(LatticeTables t, const hb_params& p, int kernel, int wall, uint64_t steps,
                                                 Layout* layout = nullptr);

struct BatchMember {
  int slot = -1;
  Layout L;
  LatticeTables t;
  hb_params p;
  int kernel = 0, wall = 0;
  int64_t site_base = 0, site_len = 0;
  int64_t run_base = 0, gen_base = 0;
  int64_t iol_base = 0, iol_len = 0;  // entries of the iolet-link lists
  int buffer_at_admission = 0;
  uint64_t steps = 0, t_first = 1;
  bool finished = false;
};

class Batch {
 public:
  Batch(int64_t site_capacity, int64_t general_capacity, int max_lattices, int precision, int device);
  ~Batch();

  // Admit a lattice; returns its slot.  Throws Error(HB_ERR_OOM) when it does not fit.
  int add(LatticeTables t, const hb_params& p, int kernel, int wall, uint64_t steps);
  // Admit a prepared lattice; its contents move into the batch only on success.
  int add(PreparedLattice& prep);
  void remove(int slot);
  // Run `k` steps of every active member (a captured CUDA graph per block
  // length); returns the slots that finished during the block: reached their
  // step count, or went unstable (then stopped, their fields not filled).
  std::vector<int> run(int k);
  // Macroscopic fields of a finished member's last step, reference order.
  void get_macro(int slot, double* rho, double* u, double* wss);
  int status(int slot);
  uint64_t time_step(int slot);
  int64_t member_sites(int slot) const;
  int members() const { return (int)members_.size(); }
  int64_t active_sites() const;
  void set_tuning(int spt, int bulk_block);
  // HB_BATCH_STEP_PERSISTENT or HB_BATCH_STEP_SPLIT.
  void set_step_form(int form);
  int step_form() const { return form_; }
  int spt() const { return spt_; }
  int bulk_block() const { return bulk_block_; }
  double last_ms() const { return last_ms_; }
  int64_t device_bytes() const { return dev_bytes_; }
  int precision() const { return precision_; }
  // Bytes of device memory a batch of these capacities holds.
  static int64_t bytes_for(int64_t site_capacity, int64_t general_capacity, int max_lattices, int precision);

 private:
  void check(cudaError_t e, const char* what);
  void write_member_tables(const BatchMember& m);
  void clear_member_tables(const BatchMember& m);
  void capture(int k);
  void* batch_args_blob(int parity);

  int device_, precision_;
  int64_t cap_sites_, np_, cap_gen_;
  int max_lat_;
  int64_t run_cap_;
  RangeAlloc sites_, gens_, runs_, iols_;
  std::vector<int> free_slots_;
  std::map<int, std::unique_ptr<BatchMember>> members_;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  cudaStream_t side_ = nullptr;               // boundary tiles of the split form
  cudaEvent_t fork_ = nullptr, join_ = nullptr;
  DeviceBuffer f_[2], ghost_[2];
  DeviceBuffer meta_, run_off_;
  DeviceBuffer g_site_, g_run_, g_wall_, g_iolet_, g_src_, g_q_, g_nrm_, g_io_, g_cpl_, g_xyz_, g_lat_;
  DeviceBuffer lat_, cos_, iolets_, dens_, lat_status_, macro_list_, macro_count_, io_moments_, iol_list_, iol_link_, rho_, u_, wss_;
  int cur_ = 0;
  int spt_ = 2, bulk_block_ = 256;
  int form_ = HB_BATCH_STEP_PERSISTENT;
  int sm_count_ = 148;
  cudaGraphExec_t graph_ = nullptr;
  int graph_k_ = 0;
  bool dirty_ = true;
  double last_ms_ = 0;
  int64_t dev_bytes_ = 0;
};

}  // namespace hb
