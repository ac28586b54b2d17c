// kernels_f64.cu -- FP64 collide-and-stream kernels for sm_100a.
//
// Compiled with -fmad=false: every product and sum is rounded separately, in
// the association order of the reference's SSE3 build, so the results match
// the reference's FP64 CPU results bit for bit.
//
// Pull form.  The reference pushes each post-collision value into the
// neighbour's slot (src/lb/streamers/SimpleCollideAndStreamDelegate.h:28-36).
// Here each site stores its own post-collision values contiguously (coalesced
// SoA stores) and the next step gathers slot i of site x from x - c_i.  Boundary
// slots become gather rules on the site's own values:
//   bounce-back     slot i = f*_{inv i}(x)            (SimpleBounceBackDelegate.h:36-44)
//   BFL q >= 1/2    slot i = (f*_d + (2q-1) f*_i)/(2q), d = inv i
//   BFL q <  1/2    slot i = 2q f*_d + (1-2q) slot_d  (the post-step, BouzidiFirdaousLallemandDelegate.h:54-93)
//   Nash / Ladd     the ghost value is computed in the producing step and kept in
//                   a per-link ghost buffer (f*_d itself stays: the BFL rule of the
//                   opposite wall link reads it)
//   GZS             the virtual-node value is computed in the producing step
//                   (reads the neighbour's pre-collision f by re-gathering it) and
//                   stored in f*_d(x), which nothing else reads (d points into the wall).
#include <cuda_runtime.h>

#include "../../include/hemeb200.h"
#include "device.h"
#include "f64_site.cuh"
#include "hb_common.h"

namespace hb {
namespace {

constexpr int kGeneralBlocksPerSM = 4;

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// Three blocks of 256 per SM: TRT otherwise takes 92 registers and runs two
// (measured 0.228 -> 0.200 ms per launch on the 4M pipe, no spills); LBGK fits
// in 80 anyway.  The sponge-layer kernels and the output steps would spill under the
// bound and keep the compiler's allocation.
template <int K, bool GATHER, bool MACRO>
__global__ void __launch_bounds__(256, (is_sponge(K) || MACRO) ? 1 : 3) k_bulk(const StepArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  const int r = __ldg(a.meta + s);
  if (r < 0) return;
  bulk_site_f64<K, GATHER, MACRO>(a, s, r);
}

// The boundary kernel is latency-bound.  Its gather issues the eighteen loads
// of a record together with the BFL cut distances and own-site values
// (f64_site.cuh), which needs the registers to hold them: with LBGK or TRT,
// bounce-back or BFL walls and no outputs it runs four blocks of 128 per SM
// (125 registers).  4M-site pipe, time alone / whole step: five blocks (96
// registers, 88 bytes spilled) 0.0523 / 0.2233 ms, four blocks 0.0429 / 0.2171
// ms; with the BFL loads issued link by link, five blocks 0.0545 / 0.2219 ms and
// four 0.0585 / 0.2261 ms.  The sponge-layer kernels, GZS walls and output steps
// keep the compiler's allocation.
template <int K, int WALL, bool GATHER, bool MACRO>
__global__ void __launch_bounds__(128, (!is_sponge(K) && WALL != kGZS && !MACRO) ? kGeneralBlocksPerSM : 1)
    k_general(const StepArgs a, int g0) {
  const int g = g0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= a.gen.G) return;
  general_site_f64<K, WALL, GATHER, MACRO>(a, g);
}

// The records without iolet links (collision types 0 and 1: irregular fluid
// sites and wall sites, the first bins) in a kernel compiled without the iolet
// rules, and the rest in k_general after it on the same stream.  4M-site pipe:
// whole step 0.2165 -> 0.2140 ms (the two launches alone 0.0430 -> 0.0469 ms:
// the iolet records' short second launch adds its own latency).
template <int K, int WALL, bool GATHER, bool MACRO>
__global__ void __launch_bounds__(128, (!is_sponge(K) && WALL != kGZS && !MACRO) ? kGeneralBlocksPerSM : 1)
    k_general_walls(const StepArgs a) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= a.gen.G_noiolet) return;
  general_site_f64<K, WALL, GATHER, MACRO, false>(a, g);
}

template <int WALL>
__global__ void __launch_bounds__(256) k_gather(const StepArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  double f[Q];
  gather_any<WALL, true>(a, s, f);
#pragma unroll
  for (int i = 0; i < Q; i++) a.fout[(int64_t)i * a.np + s] = f[i];
}

template <int WALL>
__global__ void __launch_bounds__(256) k_gather_aos(const StepArgs a, const int* st2ref, double* aos) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  double f[Q];
  gather_any<WALL, true>(a, s, f);
  const int64_t base = (int64_t)st2ref[s] * Q;
#pragma unroll
  for (int i = 0; i < Q; i++) aos[base + i] = f[i];
}

// One block per Windkessel iolet.  The flow-rate sum runs in the reference's
// order (sites in contiguous order, one add after another, InOutLetWK3.cc:95):
// the block stages the contributions in shared memory with coalesced loads and
// thread 0 adds them in sequence, so the outlet density is bit-identical.
__global__ void k_wk3_begin(WK3Dev* wk3, const double* cpl_buf, double* dens_row) {
  constexpr int kChunk = 2048;
  __shared__ double stage[kChunk];
  WK3Dev& W = wk3[blockIdx.x];
  const int n = W.count_prev;
  double acc = 0.0;
  for (int base = 0; base < n; base += kChunk) {
    const int m = min(kChunk, n - base);
    for (int k = threadIdx.x; k < m; k += blockDim.x) stage[k] = cpl_buf[W.cpl_start + base + k];
    __syncthreads();
    if (threadIdx.x == 0)
      for (int k = 0; k < m; k++) acc = acc + stage[k];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    // InOutLetWK3::DoComms (self-message on one rank), then the centre site's
    // DoPreStreamCoupling and DoPostStreamCoupling (InOutLetWK3.cc:33-105).
    const double density = W.density_new;
    double flow = 0.0 + acc;
    if (n != 0) flow = flow * W.area / (double)n;
    dens_row[W.iolet] = density;
    double d_after = density, flow_old = W.flow_old;
    if (W.centre_couples) {
      const double pressure = density * kCs2;
      if (W.kind == kWK2) {
        // InOutLetWK2::DoPreStreamCoupling / DoPostStreamCoupling (InOutLetWK2.cc:66-95).
        const double R0 = W.rp, C0 = W.cp;
        const double pn = R0 / (1.0 + R0 * C0) * (flow + C0 * pressure);
        W.density_new = pn / kCs2;
        d_after = W.density_new;
      } else {
        const double Rc = W.rc, Rp = W.rp, Cp = W.cp;
        const double pn = (Rp * Cp * pressure + (Rc + Rp) * (2.0 * flow - W.flow_old) + Rc * Rp * Cp * (flow - W.flow_old)) / (1.0 + Rp * Cp);
        W.density_new = pn / kCs2;
        d_after = W.density_new;
        flow_old = flow;
      }
    }
    W.density = d_after;
    W.flow = flow;
    W.flow_old = flow_old;
    W.count_prev = W.cpl_count;
  }
}

// ---------------------------------------------------------------------------
// Stress caches of an output step from the tensor the step stored
// (BaseStreamer::UpdateMinsAndMaxes, src/lb/streamers/BaseStreamer.h:123-217;
// Lattice::CalculateVonMisesStress, CalculateShearRate, CalculateStressTensor,
// CalculateTractionOnAPoint and the two projections, src/lb/lattices/Lattice.h:983-1180).
// Every expression keeps the reference's association order.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void load_pi(const StepArgs& a, int s, double pi[3][3], double& tau) {
  const double* o = a.pi + s;
  pi[0][0] = o[0];
  pi[1][0] = o[a.np];
  pi[2][0] = o[2 * a.np];
  pi[1][1] = o[3 * a.np];
  pi[2][1] = o[4 * a.np];
  pi[2][2] = o[5 * a.np];
  tau = o[6 * a.np];
  pi[0][1] = pi[1][0];
  pi[0][2] = pi[2][0];
  pi[1][2] = pi[2][1];
}

// sigma = -Pi - (rho - 1) cs^2 I: Matrix3D's `pi * -1.0` then addDiagonal(-pressure).
__device__ __forceinline__ void stress_tensor(const double pi[3][3], double rho, double st[3][3]) {
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) st[r][c] = -1.0 * pi[r][c];
  const double pressure = (rho - 1) * kCs2;
#pragma unroll
  for (int r = 0; r < 3; r++) st[r][r] += -pressure;
}

// Site-wide caches for every site; the traction family is zero off the wall
// (k_stress_walls then fills the wall sites).
__global__ void __launch_bounds__(256) k_stress_sites(const StepArgs a, int field, double* out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  const int64_t np = a.np;
  if (field >= HB_STRESS_TRACTION) {
    out[s] = 0.0;
    out[np + s] = 0.0;
    out[2 * np + s] = 0.0;
    return;
  }
  double pi[3][3], tau;
  load_pi(a, s, pi, tau);
  if (field == HB_STRESS_VON_MISES) {
    const double sxx_yy = pi[0][0] - pi[1][1];
    const double syy_zz = pi[1][1] - pi[2][2];
    const double szz_xx = pi[2][2] - pi[0][0];
    const double sxy = pi[0][1], syz = pi[1][2], szx = pi[2][0];
    const double t1 = sxx_yy * sxx_yy + syy_zz * syy_zz + szz_xx * szz_xx;
    const double t2 = sxy * sxy + syz * syz + szx * szx;
    out[s] = sqrt(0.5 * (t1 + 6.0 * t2));
  } else if (field == HB_STRESS_SHEAR_RATE) {
    double sr = 0.0;
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int c = 0; c < 3; c++) sr += pi[r][c] * pi[r][c];
    sr = sqrt(sr) / (-2.0 * kCs2 * a.rho[s]);
    sr /= (tau - 0.5);
    out[s] = sr;
  } else {
    double st[3][3];
    stress_tensor(pi, a.rho[s], st);
    out[s] = st[0][0];
    out[np + s] = st[0][1];
    out[2 * np + s] = st[0][2];
    out[3 * np + s] = st[1][1];
    out[4 * np + s] = st[1][2];
    out[5 * np + s] = st[2][2];
  }
}

// Traction sigma.n at wall sites and its tangential and normal projections.
__global__ void __launch_bounds__(128) k_stress_walls(const StepArgs a, int field, double* out) {
  const GeneralDev& G = a.gen;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.G) return;
  if (__ldg(G.wall + g) == 0u) return;
  const int s = __ldg(G.site + g);
  const double nor[3] = {(double)__ldg(G.nrm + g), (double)__ldg(G.nrm + G.G + g), (double)__ldg(G.nrm + 2 * G.G + g)};
  double pi[3][3], tau, st[3][3], t[3];
  load_pi(a, s, pi, tau);
  stress_tensor(pi, a.rho[s], st);
#pragma unroll
  for (int r = 0; r < 3; r++) {
    t[r] = 0.0;
#pragma unroll
    for (int c = 0; c < 3; c++) t[r] += st[r][c] * nor[c];
  }
  double v[3] = {t[0], t[1], t[2]};
  if (field != HB_STRESS_TRACTION) {
    const double m = t[0] * nor[0] + t[1] * nor[1] + t[2] * nor[2];
#pragma unroll
    for (int k = 0; k < 3; k++) v[k] = field == HB_STRESS_NORMAL_TRACTION ? nor[k] * m : t[k] - nor[k] * m;
  }
  out[s] = v[0];
  out[a.np + s] = v[1];
  out[2 * a.np + s] = v[2];
}

struct Row19 {
  double v[Q];
};

// f[i*dir_stride + s*site_stride] = row[i]: SoA with (np, 1), AoS with (1, 19).
__global__ void k_fill(double* f, int64_t dir_stride, int64_t site_stride, int n, Row19 row) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
#pragma unroll
  for (int i = 0; i < Q; i++) f[(int64_t)i * dir_stride + (int64_t)s * site_stride] = row.v[i];
}

__global__ void k_soa_to_aos(const double* soa, int64_t np, const int* st2ref, int n, double* aos) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (int64_t)n * Q) return;
  const int s = (int)(k / Q), i = (int)(k % Q);
  aos[(int64_t)st2ref[s] * Q + i] = soa[(int64_t)i * np + s];
}

__global__ void k_aos_to_soa(const double* aos, const int* st2ref, int n, double* soa, int64_t np) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (int64_t)n * Q) return;
  const int s = (int)(k / Q), i = (int)(k % Q);
  soa[(int64_t)i * np + s] = aos[(int64_t)st2ref[s] * Q + i];
}

template <int K, int WALL, bool GATHER, bool MACRO>
void launch4(const StepArgs& a, int which, int bb, int gb, cudaStream_t st) {
  if ((which & 1) && a.n > 0) k_bulk<K, GATHER, MACRO><<<(a.n + bb - 1) / bb, bb, 0, st>>>(a);
  const int g0 = a.gen.G_noiolet;
  if ((which & (kLaunchBoundary | kLaunchWallRecords)) && g0 > 0)
    k_general_walls<K, WALL, GATHER, MACRO><<<(g0 + gb - 1) / gb, gb, 0, st>>>(a);
  if ((which & (kLaunchBoundary | kLaunchIoletRecords)) && a.gen.G > g0)
    k_general<K, WALL, GATHER, MACRO><<<(a.gen.G - g0 + gb - 1) / gb, gb, 0, st>>>(a, g0);
}

template <int K, int WALL>
void launch2(const StepArgs& a, bool gather, bool macro, int which, int bb, int gb, cudaStream_t st) {
  if (gather) {
    if (macro) launch4<K, WALL, true, true>(a, which, bb, gb, st);
    else launch4<K, WALL, true, false>(a, which, bb, gb, st);
  } else {
    if (macro) launch4<K, WALL, false, true>(a, which, bb, gb, st);
    else launch4<K, WALL, false, false>(a, which, bb, gb, st);
  }
}

template <int K>
void launch1(const StepArgs& a, int wall, bool gather, bool macro, int which, int bb, int gb, cudaStream_t st) {
  if (wall == kSBB) launch2<K, kSBB>(a, gather, macro, which, bb, gb, st);
  else if (wall == kBFL) launch2<K, kBFL>(a, gather, macro, which, bb, gb, st);
  else launch2<K, kGZS>(a, gather, macro, which, bb, gb, st);
}

}  // namespace

// ---------------------------------------------------------------------------
// Conserved sums: total density and momentum over the sites, FP64, in a fixed
// order (deterministic): pass 1 writes one partial per block into scratch,
// pass 2 adds the partials in block order.
// f[i*dir_stride + s*site_stride] is distribution i of site s.
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kSumThreads) k_moment_partial(const double* f, int64_t dir_stride, int64_t site_stride,
                                                                int64_t n, double* partial) {
  __shared__ double red[4][kSumThreads];
  const int64_t base = (int64_t)blockIdx.x * kSumSitesPerBlock;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int k = threadIdx.x; k < kSumSitesPerBlock; k += kSumThreads) {
    const int64_t s = base + k;
    if (s >= n) break;
    double fi[Q];
#pragma unroll
    for (int i = 0; i < Q; i++) fi[i] = f[(int64_t)i * dir_stride + s * site_stride];
    double r, mx, my, mz;
    moments(fi, r, mx, my, mz);
    acc[0] += r;
    acc[1] += mx;
    acc[2] += my;
    acc[3] += mz;
  }
#pragma unroll
  for (int c = 0; c < 4; c++) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int w = kSumThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
#pragma unroll
      for (int c = 0; c < 4; c++) red[c][threadIdx.x] = red[c][threadIdx.x] + red[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 4) partial[4 * (int64_t)blockIdx.x + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void k_moment_final(const double* partial, int nblocks, double* out) {
  const int c = threadIdx.x;
  if (c >= 4) return;
  double acc = 0.0;
  for (int b = 0; b < nblocks; b++) acc = acc + partial[4 * (int64_t)b + c];
  out[c] = acc;
}

int moment_sum_blocks(int64_t n) { return (int)((n + kSumSitesPerBlock - 1) / kSumSitesPerBlock); }

void launch_moment_sums(const double* f, int64_t dir_stride, int64_t site_stride, int64_t n, double* scratch,
                        double* out, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = moment_sum_blocks(n);
  if (nb > 0) k_moment_partial<<<nb, kSumThreads, 0, st>>>(f, dir_stride, site_stride, n, scratch);
  k_moment_final<<<1, 32, 0, st>>>(scratch, nb, out);
}

void launch_step_f64(const StepArgs& a, int kernel, int wall, bool gather, bool macro, int which, int bulk_block,
                     int general_block, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (kernel == kLBGK) launch1<kLBGK>(a, wall, gather, macro, which, bulk_block, general_block, st);
  else if (kernel == kTRT) launch1<kTRT>(a, wall, gather, macro, which, bulk_block, general_block, st);
  else if (kernel == kLES) launch1<kLES>(a, wall, gather, macro, which, bulk_block, general_block, st);
  else if (kernel == kLBGKSL) launch1<kLBGKSL>(a, wall, gather, macro, which, bulk_block, general_block, st);
  else launch1<kTRTSL>(a, wall, gather, macro, which, bulk_block, general_block, st);
}

void launch_gather_f64(const StepArgs& a, int wall, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  const int b = 256;
  if (a.n <= 0) return;
  if (wall == kBFL) k_gather<kBFL><<<(a.n + b - 1) / b, b, 0, st>>>(a);
  else if (wall == kGZS) k_gather<kGZS><<<(a.n + b - 1) / b, b, 0, st>>>(a);
  else k_gather<kSBB><<<(a.n + b - 1) / b, b, 0, st>>>(a);
}

void launch_stress_field(const StepArgs& a, int field, double* out, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (a.n <= 0) return;
  k_stress_sites<<<(a.n + 255) / 256, 256, 0, st>>>(a, field, out);
  if (field >= HB_STRESS_TRACTION && a.gen.G > 0) k_stress_walls<<<(a.gen.G + 127) / 128, 128, 0, st>>>(a, field, out);
}

void launch_gather_aos_f64(const StepArgs& a, int wall, const int* st2ref, double* aos, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  const int b = 256;
  if (a.n <= 0) return;
  if (wall == kBFL) k_gather_aos<kBFL><<<(a.n + b - 1) / b, b, 0, st>>>(a, st2ref, aos);
  else if (wall == kGZS) k_gather_aos<kGZS><<<(a.n + b - 1) / b, b, 0, st>>>(a, st2ref, aos);
  else k_gather_aos<kSBB><<<(a.n + b - 1) / b, b, 0, st>>>(a, st2ref, aos);
}

void launch_wk3_begin(WK3Dev* wk3, int nwk3, const double* cpl_buf, double* dens_row, void* stream) {
  if (nwk3 > 0) k_wk3_begin<<<nwk3, 256, 0, (cudaStream_t)stream>>>(wk3, cpl_buf, dens_row);
}

void launch_equilibrium_f64(double* f, int64_t np, int n, const double feq[19], void* stream) {
  Row19 r;
  for (int i = 0; i < Q; i++) r.v[i] = feq[i];
  if (n > 0) k_fill<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(f, np, 1, n, r);
}

void launch_equilibrium_aos_f64(double* f, int n, const double feq[19], void* stream) {
  Row19 r;
  for (int i = 0; i < Q; i++) r.v[i] = feq[i];
  if (n > 0) k_fill<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(f, 1, Q, n, r);
}

void launch_soa_to_aos_f64(const double* soa, int64_t np, const int* st2ref, int n, double* aos, void* stream) {
  const int64_t tot = (int64_t)n * Q;
  if (tot > 0) k_soa_to_aos<<<(unsigned)((tot + 255) / 256), 256, 0, (cudaStream_t)stream>>>(soa, np, st2ref, n, aos);
}

void launch_aos_to_soa_f64(const double* aos, const int* st2ref, int n, double* soa, int64_t np, void* stream) {
  const int64_t tot = (int64_t)n * Q;
  if (tot > 0) k_aos_to_soa<<<(unsigned)((tot + 255) / 256), 256, 0, (cudaStream_t)stream>>>(aos, st2ref, n, soa, np);
}

}  // namespace hb
