// batch_dev.h -- device records of the batched form (kernels_batch.cu, batch.cpp).
#pragma once

#include <cstdint>

#include "device.h"

namespace hb {

struct BatchLatDev {
  double tau, omega, omega_minus;
  uint64_t t;          // 1-based step of the next step
  uint64_t t_first;    // the first step after admission reads f directly
  uint64_t t_end;      // the lattice stops once t reaches t_end
  int kernel, wall;
  int io_base;         // 32 iolet entries per lattice
  int active;          // this step runs
  int direct;          // this step reads pre-collision f
  int macro;           // this step fills the macroscopic outputs (the last step)
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
  float inv_scale;
  BatchLatDev* lat;
  const int* run_lat;   // lattice of each run
  const int* g_lat;     // lattice of each general site
  double* dens;         // [L][32] iolet densities of this step
  int* lat_status;      // [L] StatusBits per lattice
  int n_lat;
  int bulk_tiles;       // tiles of bulk_block*spt sites
  int gen_tiles;
};

struct Row19f {
  float v[19];
};

void launch_batch_begin(void* lat, const void* cos_tab, double* dens, int n_lat, void* stream);
void launch_batch_step(const BatchArgs& b, int precision, int spt, int bulk_block, int bulk_grid, int gen_grid,
                       void* bulk_stream, void* gen_stream);
int batch_occupancy(int precision, int spt, int bulk_block, int* bulk_blocks_per_sm, int* gen_blocks_per_sm);
void launch_fill_shift(void* out, int64_t np, int64_t base, int64_t n, const float vals[19], int precision, float inv_scale,
                       void* stream);

}  // namespace hb
