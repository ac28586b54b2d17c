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
// of the arena with a grid sized to the SM count.
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

template <class S, int K>
__device__ __forceinline__ void bulk_dispatch(const StepArgs& a, const MixArgs& m, int s, int r, bool direct, bool macro) {
  if (direct) {
    if (macro) bulk_site_m<S, K, false, true>(a, m, s, r);
    else bulk_site_m<S, K, false, false>(a, m, s, r);
  } else {
    if (macro) bulk_site_m<S, K, true, true>(a, m, s, r);
    else bulk_site_m<S, K, true, false>(a, m, s, r);
  }
}

template <class S, int K, int WALL>
__device__ __forceinline__ void general_dispatch(const StepArgs& a, const MixArgs& m, int gi, bool direct, bool macro) {
  if (direct) {
    if (macro) general_site_m<S, K, WALL, false, true>(a, m, gi);
    else general_site_m<S, K, WALL, false, false>(a, m, gi);
  } else {
    if (macro) general_site_m<S, K, WALL, true, true>(a, m, gi);
    else general_site_m<S, K, WALL, true, false>(a, m, gi);
  }
}

template <class S, int SPT>
__global__ void __launch_bounds__(256) k_batch_bulk(const BatchArgs b) {
  const MixArgs m{b.fin, b.fout, b.gin, b.gout, b.inv_scale};
  const int span = blockDim.x * SPT;
  for (int tile = blockIdx.x; tile < b.bulk_tiles; tile += gridDim.x) {
#pragma unroll
    for (int k = 0; k < SPT; k++) {
      const int s = tile * span + k * blockDim.x + threadIdx.x;
      if (s >= b.base.n) continue;
      const int r = __ldg(b.base.meta + s);
      if (r < 0) continue;
      const int l = __ldg(b.run_lat + r);
      const BatchLatDev d = b.lat[l];
      if (!d.active) continue;
      StepArgs a = b.base;
      patch(a, d, l, b);
      if (d.kernel == kTRT) bulk_dispatch<S, kTRT>(a, m, s, r, d.direct, d.macro);
      else bulk_dispatch<S, kLBGK>(a, m, s, r, d.direct, d.macro);
    }
  }
}

template <class S>
__global__ void __launch_bounds__(128) k_batch_general(const BatchArgs b) {
  const MixArgs m{b.fin, b.fout, b.gin, b.gout, b.inv_scale};
  for (int tile = blockIdx.x; tile < b.gen_tiles; tile += gridDim.x) {
    const int gi = tile * blockDim.x + threadIdx.x;
    if (gi >= b.base.gen.G) continue;
    const int l = __ldg(b.g_lat + gi);
    if (l < 0) continue;  // a free general slot
    const BatchLatDev d = b.lat[l];
    if (!d.active) continue;
    StepArgs a = b.base;
    patch(a, d, l, b);
    if (d.kernel == kTRT) {
      if (d.wall == kBFL) general_dispatch<S, kTRT, kBFL>(a, m, gi, d.direct, d.macro);
      else general_dispatch<S, kTRT, kSBB>(a, m, gi, d.direct, d.macro);
    } else {
      if (d.wall == kBFL) general_dispatch<S, kLBGK, kBFL>(a, m, gi, d.direct, d.macro);
      else general_dispatch<S, kLBGK, kSBB>(a, m, gi, d.direct, d.macro);
    }
  }
}

// One thread per lattice: advance the time of lattices that ran, decide which
// run this step, and compute their cosine iolet densities for this step
// (InOutLetCosine::GetDensity at the 0-indexed step, BoundaryValues.cc:211-214).
__global__ void k_batch_begin(BatchLatDev* lat, const BatchCosDev* cos_tab, double* dens, int n_lat) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n_lat) return;
  BatchLatDev d = lat[l];
  if (d.ran_prev) d.t++;
  d.active = d.t < d.t_end;
  d.direct = d.t == d.t_first;
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
  lat[l] = d;
}

// Shifted equilibrium g_i = f_i - w_i into sites [base, base + n) of one buffer.
template <class S>
__global__ void k_fill_shift(void* out, int64_t np, int64_t base, int64_t n, Row19f vals, float inv_scale) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
#pragma unroll
  for (int i = 0; i < Q; i++) Store<S>::store(out, (int64_t)i * np + base + s, vals.v[i], inv_scale);
}

}  // namespace

void launch_fill_shift(void* out, int64_t np, int64_t base, int64_t n, const float vals[19], int precision, float inv_scale,
                       void* stream) {
  Row19f r;
  for (int i = 0; i < Q; i++) r.v[i] = vals[i];
  if (n <= 0) return;
  const unsigned g = (unsigned)((n + 255) / 256);
  if (precision == HB_STORE_FP16) k_fill_shift<__half><<<g, 256, 0, (cudaStream_t)stream>>>(out, np, base, n, r, inv_scale);
  else k_fill_shift<float><<<g, 256, 0, (cudaStream_t)stream>>>(out, np, base, n, r, inv_scale);
}

void launch_batch_begin(void* lat, const void* cos_tab, double* dens, int n_lat, void* stream) {
  if (n_lat > 0)
    k_batch_begin<<<(n_lat + 127) / 128, 128, 0, (cudaStream_t)stream>>>(static_cast<BatchLatDev*>(lat),
                                                                          static_cast<const BatchCosDev*>(cos_tab), dens, n_lat);
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
