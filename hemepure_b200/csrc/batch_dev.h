// batch_dev.h -- device records of the batched form (kernels_batch.cu, batch.cpp).
#pragma once

#include <cstdint>

#include "device.h"

namespace hb {

struct BatchLatDev {
  double tau, omega, omega_minus;
  uint64_t t;          // 1-based step of the next step
  uint64_t t_first;    // time step at admission
  uint64_t t_end;      // the lattice stops once t reaches t_end
  int64_t site_base;   // the lattice's sites are [site_base, site_base + n_sites)
  int n_sites;
  int kernel, wall;
  int io_base;         // 32 iolet entries per lattice
  int active;          // this step runs
  int macro;           // this step is the last: k_batch_macro runs it and fills the outputs
  int ran_prev;        // the previous step ran (its t is still to be advanced)
  int pad;
};

struct BatchCosDev {   // cosine iolet parameters (InOutLetCosine) per iolet entry
  double mean, amp, phase, period, min_density;
  uint64_t warmup;
  int kind;
  int pad;
};

struct BatchArgs {
  StepArgs base;        // arena-wide tables; per-lattice fields patched per site
  const void* fin;
  void* fout;
  const float* gin;
  float* gout;
  BatchLatDev* lat;
  const int* g_lat;     // lattice of each general site
  double* dens;         // [L][32] iolet densities of this step
  int* lat_status;      // [L] StatusBits per lattice
  int* macro_list;      // lattices in their last step this step (written by k_batch_begin)
  int* macro_count;
  float* io_moments;    // [4][G] pre-collision density and velocity of records with iolet links
  int n_lat;
  int bulk_tiles;       // tiles of block*spt sites
  int gen_tiles;        // tiles of block boundary records
  const int* iol_list;  // record of each iolet link (-1: free entry)
  const uint8_t* iol_link;  // the link (1..18)
  int iol_count;        // entries of iol_list in use (high-water mark)
};

struct Row19f {
  float v[19];
};

// One block (n_lat <= 1024): advances time, iolet densities, and the list of
// lattices in their last step.
void launch_batch_begin(void* lat, const void* cos_tab, double* dens, int* macro_list, int* macro_count, int n_lat,
                        void* stream);
// Iolet ghosts of the records the step kernel relaxed (after it, same stream).
void launch_batch_ghosts(const BatchArgs& b, int precision, int grid, void* stream);
// The last step of the listed lattices, with the macroscopic outputs.
void launch_batch_macro(const BatchArgs& b, int precision, int grid, void* stream);
// Iolet ghosts of general slots [base, base + n) set to vals[d-1] for link d.
void launch_fill_ghost(float* ghost, int64_t pitch, int64_t base, int64_t n, const float vals[18], void* stream);
// One step of all running lattices not in their last step (persistent kernel).
void launch_batch_step(const BatchArgs& b, int precision, int spt, int block, int grid, void* stream);
// Split form: bulk tiles (grid b.bulk_tiles of `block` threads) and boundary tiles
// (grid b.gen_tiles of kBatchGenBlock records), launched on two streams.
constexpr int kBatchGenBlock = 128;
void launch_batch_bulk(const BatchArgs& b, int precision, int spt, int block, void* stream);
void launch_batch_gen(const BatchArgs& b, int precision, void* stream);
int batch_occupancy(int precision, int spt, int block, int* blocks_per_sm);
void launch_fill_shift(void* out, int64_t np, int64_t base, int64_t n, const float vals[19], int precision, void* stream);

}  // namespace hb
