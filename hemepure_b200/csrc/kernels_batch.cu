// kernels_batch.cu -- many independent lattices of uneven size per launch.
//
// The member lattices share one storage arena: each owns a contiguous range of
// sites (its runs and general records are concatenated with shifted indices),
// so the single-lattice gather rules apply unchanged.  Per-lattice parameters
// (relaxation times, time step, iolets, flags) live in device memory and are
// advanced by k_batch_begin, so a captured CUDA graph of a block of steps can be
// replayed without host involvement.  The step is two persistent kernels over
// the whole arena, one for plain bulk sites (bandwidth-bound) and one for
// boundary sites (latency-bound), launched side by side; each loops over tiles
// of the arena with a grid sized to the SM count.  A lattice's last step, which
// also fills its macroscopic outputs, is run instead by k_batch_macro over the
// short list k_batch_begin builds, so the step kernels carry no output path.
// A newly admitted lattice starts from equilibrium in both its distributions and
// its iolet ghosts, so its first step gathers like every other.
//
// Supported per lattice: LBGK or TRT; bounce-back or BFL walls; Nash cosine
// pressure and Ladd parabolic velocity iolets (the serving mix).
#include "batch_dev.h"
#include "mixed_site.cuh"

namespace hb {

namespace {

__device__ __forceinline__ void patch(StepArgs& a, const BatchLatDev& d, int l, const BatchArgs& b) {
  a.tau = d.tau;
  a.omega = d.omega;
  a.omega_minus = d.omega_minus;
  a.t = d.t;
  a.dens_row = b.dens + 32 * (int64_t)l;
  a.iolets = b.base.iolets + 32 * (int64_t)l;
  a.status = b.lat_status + l;
}

template <class S, int SPT>
__global__ void __launch_bounds__(256) k_batch_bulk(const BatchArgs b) {
  const MixArgs m{b.fin, b.fout, b.gin, b.gout};
  const int span = blockDim.x * SPT;
  for (int tile = blockIdx.x; tile < b.bulk_tiles; tile += gridDim.x) {
    // All SPT sites are gathered before any collides, so their loads overlap.
    int s[SPT], l[SPT];
    float g[SPT][Q];
#pragma unroll
    for (int k = 0; k < SPT; k++) {
      s[k] = tile * span + k * blockDim.x + threadIdx.x;
      l[k] = -1;
      if (s[k] >= b.base.n) continue;
      const int r = __ldg(b.base.meta + s[k]);
      if (r < 0) continue;
      const int lk = __ldg(b.run_lat + r);
      if (!b.lat[lk].active || b.lat[lk].macro) continue;
      l[k] = lk;
      gather_bulk_m<S>(b.base, m, s[k], r, g[k]);
    }
#pragma unroll
    for (int k = 0; k < SPT; k++) {
      if (l[k] < 0) continue;
      const BatchLatDev d = b.lat[l[k]];
      StepArgs a = b.base;
      patch(a, d, l[k], b);
      if (d.kernel == kTRT) bulk_collide_m<S, kTRT, false>(a, m, s[k], g[k]);
      else bulk_collide_m<S, kLBGK, false>(a, m, s[k], g[k]);
    }
  }
}

template <class S>
__global__ void __launch_bounds__(128) k_batch_general(const BatchArgs b) {
  const MixArgs m{b.fin, b.fout, b.gin, b.gout};
  for (int tile = blockIdx.x; tile < b.gen_tiles; tile += gridDim.x) {
    const int gi = tile * blockDim.x + threadIdx.x;
    if (gi >= b.base.gen.G) continue;
    const int l = __ldg(b.g_lat + gi);
    if (l < 0) continue;  // a free general slot
    const BatchLatDev d = b.lat[l];
    if (!d.active || d.macro) continue;
    StepArgs a = b.base;
    patch(a, d, l, b);
    if (d.kernel == kTRT) {
      if (d.wall == kBFL) general_site_m<S, kTRT, kBFL, true, false>(a, m, gi);
      else general_site_m<S, kTRT, kSBB, true, false>(a, m, gi);
    } else {
      if (d.wall == kBFL) general_site_m<S, kLBGK, kBFL, true, false>(a, m, gi);
      else general_site_m<S, kLBGK, kSBB, true, false>(a, m, gi);
    }
  }
}

// The last step of each listed lattice, over its whole site range, with outputs.
template <class S>
__global__ void __launch_bounds__(128) k_batch_macro(const BatchArgs b) {
  const MixArgs m{b.fin, b.fout, b.gin, b.gout};
  const int count = *b.macro_count;
  for (int j = 0; j < count; j++) {
    const int l = b.macro_list[j];
    const BatchLatDev d = b.lat[l];
    StepArgs a = b.base;
    patch(a, d, l, b);
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < d.n_sites; k += (int64_t)gridDim.x * blockDim.x) {
      const int s = (int)(d.site_base + k);
      const int r = __ldg(b.base.meta + s);
      if (r >= 0) {
        if (d.kernel == kTRT) bulk_site_m<S, kTRT, true, true>(a, m, s, r);
        else bulk_site_m<S, kLBGK, true, true>(a, m, s, r);
      } else {
        const int gi = -r - 1;
        if (d.kernel == kTRT) {
          if (d.wall == kBFL) general_site_m<S, kTRT, kBFL, true, true>(a, m, gi);
          else general_site_m<S, kTRT, kSBB, true, true>(a, m, gi);
        } else {
          if (d.wall == kBFL) general_site_m<S, kLBGK, kBFL, true, true>(a, m, gi);
          else general_site_m<S, kLBGK, kSBB, true, true>(a, m, gi);
        }
      }
    }
  }
}

// One block, one thread per lattice: advance the time of lattices that ran,
// decide which run this step, compute their cosine iolet densities for this step
// (InOutLetCosine::GetDensity at the 0-indexed step, BoundaryValues.cc:211-214),
// and list the lattices whose last step this is.
__global__ void __launch_bounds__(1024) k_batch_begin(BatchLatDev* lat, const BatchCosDev* cos_tab, double* dens,
                                                      int* macro_list, int* macro_count, int n_lat) {
  __shared__ int listed;
  if (threadIdx.x == 0) listed = 0;
  __syncthreads();
  const int l = threadIdx.x;
  if (l < n_lat) {
    BatchLatDev d = lat[l];
    if (d.ran_prev) d.t++;
    d.active = d.t < d.t_end;
    d.macro = d.active && (d.t + 1 == d.t_end);
    d.ran_prev = d.active;
    if (d.active) {
      const uint64_t t0 = d.t - 1;
      for (int k = 0; k < 32; k++) {
        const BatchCosDev c = cos_tab[32 * (int64_t)l + k];
        double v = 1.0;
        if (c.kind == kCosine) {
          const double w = 2.0 * kPi / c.period;
          const double target = c.mean + c.amp * cos(w * (double)t0 + c.phase);
          if (t0 >= c.warmup) v = target;
          else {
            const double fac = (double)t0 / (double)c.warmup;
            v = fac * target + (1. - fac) * c.min_density;
          }
        }
        dens[32 * (int64_t)l + k] = v;
      }
    }
    if (d.macro) macro_list[atomicAdd(&listed, 1)] = l;
    lat[l] = d;
  }
  __syncthreads();
  if (threadIdx.x == 0) *macro_count = listed;
}

__global__ void k_fill_ghost(float* ghost, int64_t pitch, int64_t base, int64_t n, Row19f vals) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
#pragma unroll
  for (int d = 0; d < 18; d++) ghost[(int64_t)d * pitch + base + g] = vals.v[d];
}

// Shifted equilibrium g_i = f_i - w_i into sites [base, base + n) of one buffer.
template <class S>
__global__ void k_fill_shift(void* out, int64_t np, int64_t base, int64_t n, Row19f vals) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
#pragma unroll
  for (int i = 0; i < Q; i++) Store<S>::store(out, (int64_t)i * np + base + s, vals.v[i]);
}

}  // namespace

void launch_fill_shift(void* out, int64_t np, int64_t base, int64_t n, const float vals[19], int precision,
                       void* stream) {
  Row19f r;
  for (int i = 0; i < Q; i++) r.v[i] = vals[i];
  if (n <= 0) return;
  const unsigned g = (unsigned)((n + 255) / 256);
  if (precision == HB_STORE_FP16) k_fill_shift<__half><<<g, 256, 0, (cudaStream_t)stream>>>(out, np, base, n, r);
  else k_fill_shift<float><<<g, 256, 0, (cudaStream_t)stream>>>(out, np, base, n, r);
}

void launch_batch_begin(void* lat, const void* cos_tab, double* dens, int* macro_list, int* macro_count, int n_lat,
                        void* stream) {
  if (n_lat > 0)
    k_batch_begin<<<1, 1024, 0, (cudaStream_t)stream>>>(static_cast<BatchLatDev*>(lat), static_cast<const BatchCosDev*>(cos_tab),
                                                        dens, macro_list, macro_count, n_lat);
}

void launch_batch_macro(const BatchArgs& b, int precision, int grid, void* stream) {
  if (precision == HB_STORE_FP16) k_batch_macro<__half><<<grid, 128, 0, (cudaStream_t)stream>>>(b);
  else k_batch_macro<float><<<grid, 128, 0, (cudaStream_t)stream>>>(b);
}

void launch_fill_ghost(float* ghost, int64_t pitch, int64_t base, int64_t n, const float vals[18], void* stream) {
  Row19f r;
  for (int d = 0; d < 18; d++) r.v[d] = vals[d];
  r.v[18] = 0.0f;
  if (n > 0) k_fill_ghost<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(ghost, pitch, base, n, r);
}

void launch_batch_step(const BatchArgs& b, int precision, int spt, int bulk_block, int bulk_grid, int gen_grid,
                       void* bulk_stream, void* gen_stream) {
  cudaStream_t sb = (cudaStream_t)bulk_stream, sg = (cudaStream_t)gen_stream;
  if (b.gen_tiles > 0) {
    if (precision == HB_STORE_FP16) k_batch_general<__half><<<gen_grid, 128, 0, sg>>>(b);
    else k_batch_general<float><<<gen_grid, 128, 0, sg>>>(b);
  }
  if (b.bulk_tiles > 0) {
    if (precision == HB_STORE_FP16) {
      if (spt == 2) k_batch_bulk<__half, 2><<<bulk_grid, bulk_block, 0, sb>>>(b);
      else k_batch_bulk<__half, 1><<<bulk_grid, bulk_block, 0, sb>>>(b);
    } else {
      if (spt == 2) k_batch_bulk<float, 2><<<bulk_grid, bulk_block, 0, sb>>>(b);
      else k_batch_bulk<float, 1><<<bulk_grid, bulk_block, 0, sb>>>(b);
    }
  }
}

int batch_occupancy(int precision, int spt, int bulk_block, int* bulk_blocks_per_sm, int* gen_blocks_per_sm) {
  cudaError_t e;
  if (precision == HB_STORE_FP16) {
    e = spt == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(bulk_blocks_per_sm, k_batch_bulk<__half, 2>, bulk_block, 0)
                 : cudaOccupancyMaxActiveBlocksPerMultiprocessor(bulk_blocks_per_sm, k_batch_bulk<__half, 1>, bulk_block, 0);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(gen_blocks_per_sm, k_batch_general<__half>, 128, 0);
  } else {
    e = spt == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(bulk_blocks_per_sm, k_batch_bulk<float, 2>, bulk_block, 0)
                 : cudaOccupancyMaxActiveBlocksPerMultiprocessor(bulk_blocks_per_sm, k_batch_bulk<float, 1>, bulk_block, 0);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(gen_blocks_per_sm, k_batch_general<float>, 128, 0);
  }
  return e == cudaSuccess ? 0 : -1;
}

}  // namespace hb
