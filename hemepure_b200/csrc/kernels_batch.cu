// kernels_batch.cu -- many independent lattices of uneven size per launch.
//
// The member lattices share one storage arena: each owns a contiguous range of
// sites (its runs and general records are concatenated with shifted indices),
// so the single-lattice gather rules apply unchanged.  Per-lattice parameters
// (relaxation times, time step, iolets, flags) live in device memory and are
// advanced by k_batch_begin, so a captured CUDA graph of a block of steps can be
// replayed without host involvement.  The step is one persistent kernel over the
// whole arena whose blocks interleave tiles of plain bulk sites (bandwidth-bound)
// with tiles of boundary records (latency-bound), so both kinds of work share
// every SM.  A lattice's last step, which
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

// Relax the gathered shifted distributions g in place (LBGK, or TRT by pairs of
// opposite directions, in the arithmetic of collide_one_f), flagging instability
// in the lattice's status word.  Returns the pre-collision moments.
__device__ __forceinline__ void relax_inplace(float* g, int* status, bool trt, float om, float omm, float& drho,
                                              float& mx, float& my, float& mz) {
  flag_unstable_status(g, status);
  moments_g(g, drho, mx, my, mz);
  float eq[Q];
  GeqF(drho, mx, my, mz).all(eq);  // the same values as GeqF::operator(), by pairs
  if (trt) {
    g[0] = g[0] + om * (g[0] - eq[0]);
#pragma unroll
    for (int i = 1; i < Q; i += 2) {
      const int j = i + 1;  // inv(i) for odd i
      const float fi = g[i] - eq[i], fj = g[j] - eq[j];
      const float gi = g[i] + 0.5f * om * (fi + fj) + 0.5f * omm * (fi - fj);
      const float gj = g[j] + 0.5f * om * (fj + fi) + 0.5f * omm * (fj - fi);
      g[i] = gi;
      g[j] = gj;
    }
  } else {
#pragma unroll
    for (int i = 0; i < Q; i++) g[i] = g[i] + (g[i] - eq[i]) * om;
  }
}

// Gather of a boundary record with the wall rule chosen at run time (SBB or
// BFL); the rules are those of gather_general_m.  Every load depends only on
// the record's metadata and run offsets, and its address is chosen without a
// branch (records of small vessels side by side in a warp have different link
// masks), so all are in flight together; the BFL cut distances and own-site
// values follow in one batch before any arithmetic.
template <class S>
__device__ __forceinline__ void gather_general_rt(const StepArgs& a, const MixArgs& m, int gi, int s, uint32_t wm,
                                                  uint32_t im, int run, const int* off, bool bfl, float* g) {
  const GeneralDev& G = a.gen;
  g[0] = ldg_s<S>(m, s);
#pragma unroll
  for (int i = 1; i < Q; i++) {
    const int d = inv(i);
    const bool bw = (wm >> (d - 1)) & 1u, bi = (im >> (d - 1)) & 1u;
    const int src = run >= 0 ? s + off[i] : __ldg(G.src + (int64_t)(i - 1) * G.G + gi);
    const int64_t k = bw ? (int64_t)d * a.np + s : (int64_t)i * a.np + src;
    g[i] = bi ? __ldg(m.gin + (int64_t)(d - 1) * G.G + gi) : ldg_s<S>(m, k);
  }
  if (bfl && wm) {
    float qv[18], fo[18];
#pragma unroll
    for (int i = 1; i < Q; i++) {
      const int d = inv(i);
      const bool corr = ((wm >> (d - 1)) & 1u) && !((wm >> (i - 1)) & 1u);
      qv[i - 1] = corr ? __ldg(G.q + (int64_t)(d - 1) * G.G + gi) : 1.0f;
      fo[i - 1] = corr ? ldg_s<S>(m, (int64_t)i * a.np + s) : 0.0f;
    }
#pragma unroll
    for (int i = 1; i < Q; i++) {
      const int d = inv(i);
      const bool corr = ((wm >> (d - 1)) & 1u) && !((wm >> (i - 1)) & 1u);
      if (corr) {
        const float q = qv[i - 1];
        if (!(q < 0.5f)) g[i] = (g[i] + (2.0f * q - 1.0f) * fo[i - 1]) / (2.0f * q);
        else g[i] = 2.0f * q * g[i] + (1.0f - 2.0f * q) * g[d];
      }
    }
  }
}

__device__ __forceinline__ bool lattice_steps(const BatchArgs& b, int l) {
  return b.lat[l].active && !b.lat[l].macro;
}

// A tile of boundary records, one per thread (walls SBB/BFL, LBGK/TRT).  A
// record with iolet links also leaves its pre-collision density and velocity
// for k_batch_ghosts, which produces its iolet ghosts after the step: kept out
// of the step kernel, that rarely taken path does not set its register budget.
template <class S>
__device__ __forceinline__ void batch_general_tile(const BatchArgs& b, const MixArgs& m, int tile) {
  const int gi = tile * blockDim.x + threadIdx.x;
  if (gi >= b.base.gen.G) return;
  const GeneralDev& G = b.base.gen;
  const int l = __ldg(b.g_lat + gi);
  if (l < 0) return;  // a free boundary slot
  const int s = __ldg(G.site + gi);
  const uint32_t wm = __ldg(G.wall + gi), im = __ldg(G.iolet + gi);
  const int run = __ldg(G.run + gi);
  int off[20];
  if (run >= 0) run_offsets(b.base, run, off);
  if (!lattice_steps(b, l)) return;
  const BatchLatDev& d = b.lat[l];
  float g[Q];
  gather_general_rt<S>(b.base, m, gi, s, wm, im, run, off, d.wall == kBFL, g);
  float drho, mx, my, mz;
  relax_inplace(g, b.lat_status + l, d.kernel == kTRT, (float)d.omega, (float)d.omega_minus, drho, mx, my, mz);
#pragma unroll
  for (int i = 0; i < Q; i++) Store<S>::store(m.fout, (int64_t)i * b.base.np + s, g[i]);
  if (im) {
    const float rho = 1.0f + drho;
    b.io_moments[gi] = rho;
    b.io_moments[G.G + gi] = mx / rho;
    b.io_moments[2 * (int64_t)G.G + gi] = my / rho;
    b.io_moments[3 * (int64_t)G.G + gi] = mz / rho;
  }
}

// A tile of SPT * blockDim sites, plain bulk ones taken.  The run row carries
// the lattice slot in its spare last entry, so the site's run offsets and its
// lattice come in one load.  The gather is issued together with the load of
// the lattice's flags rather than after it: the loads stay inside the lattice's
// own range, and one that is not stepping (finished, awaiting retirement at the
// end of the block) only wastes them.  All SPT sites of a thread are gathered
// before any relaxes, so their loads are in flight together.
template <class S, int SPT>
__device__ __forceinline__ void batch_bulk_tile(const BatchArgs& b, const MixArgs& m, int tile) {
  int s[SPT], l[SPT];
  float g[SPT][Q];
#pragma unroll
  for (int k = 0; k < SPT; k++) {
    s[k] = (tile * SPT + k) * blockDim.x + threadIdx.x;
    l[k] = -1;
    if (s[k] >= b.base.n) continue;
    const int r = __ldg(b.base.meta + s[k]);
    if (r < 0) continue;
    int off[20];
    run_offsets(b.base, r, off);
    g[k][0] = ldg_s<S>(m, s[k]);
#pragma unroll
    for (int i = 1; i < Q; i++) g[k][i] = ldg_s<S>(m, (int64_t)i * b.base.np + (s[k] + off[i]));
    if (lattice_steps(b, off[19])) l[k] = off[19];
  }
#pragma unroll
  for (int k = 0; k < SPT; k++) {
    if (l[k] < 0) continue;
    const BatchLatDev& d = b.lat[l[k]];
    float drho, mx, my, mz;
    relax_inplace(g[k], b.lat_status + l[k], d.kernel == kTRT, (float)d.omega, (float)d.omega_minus, drho, mx, my, mz);
#pragma unroll
    for (int i = 0; i < Q; i++) Store<S>::store(m.fout, (int64_t)i * b.base.np + s[k], g[k][i]);
  }
}

// One time step of every running lattice except those in their last step: a
// persistent kernel.  Block j takes boundary tiles j, j + grid, ... and bulk
// tiles j, j + grid, ..., interleaving the two in proportion, so at any moment
// the SMs mix latency-bound boundary work with bandwidth-bound bulk work (the
// assignment is static: no counter, no block-wide barrier).  The kernel is
// latency-bound, so warps per SM set its speed: with one site per thread it is
// held to 64 registers (four 256-thread blocks per SM; the boundary path spills
// ~100 bytes to L1, measured 6-11% faster than 80 registers and three blocks),
// with two sites per thread to 80 registers (tighter bounds spill the second
// site's values).
template <class S, int SPT>
__global__ void __launch_bounds__(256, SPT == 1 ? 4 : 3) k_batch_step(const BatchArgs b) {
  const MixArgs m{b.fin, b.fout, b.gin, b.gout};
  const int j = blockIdx.x, grid = gridDim.x;
  const int n_gen = j < b.gen_tiles ? (b.gen_tiles - j + grid - 1) / grid : 0;
  const int n_bulk = j < b.bulk_tiles ? (b.bulk_tiles - j + grid - 1) / grid : 0;
  int done_gen = 0, done_bulk = 0;
  while (done_gen < n_gen || done_bulk < n_bulk) {
    // the boundary share so far stays at or below its proportion
    const bool gen_next =
        done_gen < n_gen && (done_bulk >= n_bulk || (int64_t)done_gen * n_bulk <= (int64_t)done_bulk * n_gen);
    if (gen_next) {
      batch_general_tile<S>(b, m, j + done_gen * grid);
      done_gen++;
    } else {
      batch_bulk_tile<S, SPT>(b, m, j + done_bulk * grid);
      done_bulk++;
    }
  }
}

// The split form of the step: the same tiles as two ordinary (non-persistent)
// kernels that the graph runs side by side, so each gets its own register
// budget and the hardware balances the blocks.  Boundary tiles are 128 records;
// that kernel is latency-bound and held to 48 registers (ten blocks per SM, no
// spills; 1.6-2% faster on the probe below than at its own 54).  The bulk kernel
// alone needs 56 registers; held to
// 40 (six 256-thread blocks per SM, 8 bytes spilled) it ran the serving probe
// (11 requests, 8.1M sites) at 28.1-28.5k MLUPS against 26.4-27.9k at 56 and
// 22.9k for the persistent kernel.
template <class S, int SPT>
__global__ void __launch_bounds__(256, SPT == 1 ? 6 : 3) k_batch_bulk(const BatchArgs b) {
  const MixArgs m{b.fin, b.fout, b.gin, b.gout};
  batch_bulk_tile<S, SPT>(b, m, blockIdx.x);
}

// Eight blocks of 128 per SM (64 registers, ~60 bytes spilled): with the
// batched BFL loads, ten blocks (48 registers) spilled ~160 bytes; six (80
// registers, none spilled) measured the same as eight.  Serving probe (11
// requests, 8.1M sites): 28.9k -> 30.3k MLUPS for the split step form.
template <class S>
__global__ void __launch_bounds__(128, 8) k_batch_gen(const BatchArgs b) {
  const MixArgs m{b.fin, b.fout, b.gin, b.gout};
  batch_general_tile<S>(b, m, blockIdx.x);
}

// Iolet ghosts of the boundary records stepped by k_batch_step: the Nash
// zeroth-order pressure and Ladd velocity rules of general_site_m, from the
// record's post-collision values (in fout) and its pre-collision density and
// velocity (io_moments).  One thread per iolet link (record and link from two
// parallel lists), so the FP64 profile arithmetic of a record's links runs in
// parallel.
template <class S>
__global__ void __launch_bounds__(128) k_batch_ghosts(const BatchArgs b) {
  const GeneralDev& G = b.base.gen;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < b.iol_count; k += gridDim.x * blockDim.x) {
    const int gi = __ldg(b.iol_list + k);
    if (gi < 0) continue;
    const int link = b.iol_link[k];
    const int l = __ldg(b.g_lat + gi);
    if (l < 0) continue;
    const BatchLatDev& d = b.lat[l];
    if (!d.active || d.macro) continue;
    const int io = __ldg(G.io + gi);
    const IoletDev& I = b.base.iolets[32 * (int64_t)l + io];
    const float rho = b.io_moments[gi];
    float v;
    if (I.kind == kParabolic) {
      const int s = __ldg(G.site + gi);
      const double hw[3] = {(double)__ldg(G.xyz + gi) + 0.5 * cx(link), (double)__ldg(G.xyz + G.G + gi) + 0.5 * cy(link),
                            (double)__ldg(G.xyz + 2 * G.G + gi) + 0.5 * cz(link)};
      float w[3];
      if (!parabolic_f(I, hw, (uint64_t)(unsigned int)d.t, w)) {
        atomicOr(b.lat_status + l, kStatusIoletRadius);
        w[0] = w[1] = w[2] = 0.0f;
      }
      const float corr = 2.0f * wf(link) * rho * (w[0] * cx(link) + w[1] * cy(link) + w[2] * cz(link)) * 3.0f;
      v = Store<S>::load(b.fout, (int64_t)link * b.base.np + s) - corr;
    } else {
      const float ux = b.io_moments[G.G + gi], uy = b.io_moments[2 * (int64_t)G.G + gi],
                  uz = b.io_moments[3 * (int64_t)G.G + gi];
      const double rb = b.dens[32 * (int64_t)l + io];
      const float drb = (float)(rb - 1.0);
      const float rbf = (float)rb;
      const float nx = (float)I.nrm_f[0], ny = (float)I.nrm_f[1], nz = (float)I.nrm_f[2];
      const float comp = ux * nx + uy * ny + uz * nz;
      const GeqF gq(drb, nx * comp * rbf, ny * comp * rbf, nz * comp * rbf);
      v = gq(inv(link));
    }
    b.gout[(int64_t)(link - 1) * G.G + gi] = v;
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

// One block, one warp per lattice: advance the time of lattices that ran,
// decide which run this step, list the lattices whose last step this is, and
// compute their cosine iolet densities for this step, one lane per iolet entry
// (InOutLetCosine::GetDensity at the 0-indexed step, BoundaryValues.cc:211-214).
__global__ void __launch_bounds__(1024) k_batch_begin(BatchLatDev* lat, const BatchCosDev* cos_tab, double* dens,
                                                      int* macro_list, int* macro_count, int n_lat) {
  __shared__ int listed;
  if (threadIdx.x == 0) listed = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
  for (int l = threadIdx.x >> 5; l < n_lat; l += warps) {
    unsigned long long t = 0;
    int active = 0;
    if (lane == 0) {
      BatchLatDev d = lat[l];
      if (d.ran_prev) d.t++;
      d.active = d.t < d.t_end;
      d.macro = d.active && (d.t + 1 == d.t_end);
      d.ran_prev = d.active;
      lat[l] = d;
      t = d.t;
      active = d.active;
      if (d.macro) macro_list[atomicAdd(&listed, 1)] = l;
    }
    t = __shfl_sync(0xffffffffu, t, 0);
    active = __shfl_sync(0xffffffffu, active, 0);
    if (!active) continue;
    const uint64_t t0 = t - 1;
    const BatchCosDev c = cos_tab[32 * (int64_t)l + lane];
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
    dens[32 * (int64_t)l + lane] = v;
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
  k_batch_begin<<<1, 1024, 0, (cudaStream_t)stream>>>(static_cast<BatchLatDev*>(lat), static_cast<const BatchCosDev*>(cos_tab),
                                                      dens, macro_list, macro_count, n_lat);
}

void launch_batch_ghosts(const BatchArgs& b, int precision, int grid, void* stream) {
  if (b.iol_count <= 0) return;
  if (precision == HB_STORE_FP16) k_batch_ghosts<__half><<<grid, 128, 0, (cudaStream_t)stream>>>(b);
  else k_batch_ghosts<float><<<grid, 128, 0, (cudaStream_t)stream>>>(b);
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

void launch_batch_step(const BatchArgs& b, int precision, int spt, int block, int grid, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if ((int64_t)b.gen_tiles + b.bulk_tiles <= 0) return;
  if (precision == HB_STORE_FP16) {
    if (spt == 2) k_batch_step<__half, 2><<<grid, block, 0, st>>>(b);
    else k_batch_step<__half, 1><<<grid, block, 0, st>>>(b);
  } else {
    if (spt == 2) k_batch_step<float, 2><<<grid, block, 0, st>>>(b);
    else k_batch_step<float, 1><<<grid, block, 0, st>>>(b);
  }
}

void launch_batch_bulk(const BatchArgs& b, int precision, int spt, int block, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (b.bulk_tiles <= 0) return;
  if (precision == HB_STORE_FP16) {
    if (spt == 2) k_batch_bulk<__half, 2><<<b.bulk_tiles, block, 0, st>>>(b);
    else k_batch_bulk<__half, 1><<<b.bulk_tiles, block, 0, st>>>(b);
  } else {
    if (spt == 2) k_batch_bulk<float, 2><<<b.bulk_tiles, block, 0, st>>>(b);
    else k_batch_bulk<float, 1><<<b.bulk_tiles, block, 0, st>>>(b);
  }
}

void launch_batch_gen(const BatchArgs& b, int precision, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (b.gen_tiles <= 0) return;
  if (precision == HB_STORE_FP16) k_batch_gen<__half><<<b.gen_tiles, kBatchGenBlock, 0, st>>>(b);
  else k_batch_gen<float><<<b.gen_tiles, kBatchGenBlock, 0, st>>>(b);
}

int batch_occupancy(int precision, int spt, int block, int* blocks_per_sm) {
  cudaError_t e;
  if (precision == HB_STORE_FP16)
    e = spt == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_batch_step<__half, 2>, block, 0)
                 : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_batch_step<__half, 1>, block, 0);
  else
    e = spt == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_batch_step<float, 2>, block, 0)
                 : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_batch_step<float, 1>, block, 0);
  return e == cudaSuccess ? 0 : -1;
}

}  // namespace hb
