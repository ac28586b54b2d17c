// kernels_mixed.cu -- collide-and-stream with shifted low-precision storage.
//
// Storage holds g_i = f_i - w_i rho0 (rho0 = 1), the deviation from the rest
// equilibrium, in FP32 or FP16 (scaled); the collision runs in FP32 on g, so
// rounding falls only on the deviation.  In shifted variables (w_i = w_inv(i)):
//   rho = 1 + sum g,  m = sum c g,
//   geq_i = w_i (drho - 3/2 |m|^2/rho + 9/2 (c_i.m)^2/rho + 3 c_i.m),
//   g*_i = g_i + omega (g_i - geq_i)             (LBGK; TRT and LES likewise),
// and every streaming rule of the FP64 kernels (bounce-back, BFL, Nash, Ladd,
// GZS) carries over unchanged because its coefficients sum to one over pairs of
// equal weight.  FP64 stays where the reference's conservation or stability
// needs it: iolet density targets (given in FP64, subtracted from rho0 in FP64),
// the Windkessel flow sums and ODE (kernels_f64.cu), the macroscopic outputs.
#include "mixed_site.cuh"

namespace hb {
namespace {

template <class S, int K, bool GATHER, bool MACRO>
__global__ void __launch_bounds__(256) k_bulk_m(const StepArgs a, const MixArgs m) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  const int r = __ldg(a.meta + s);
  if (r < 0) return;
  bulk_site_m<S, K, GATHER, MACRO>(a, m, s, r);
}

// Two plain bulk sites per thread (s and s + 256 of a 512-site tile), both
// gathered before either collides: a thread keeps twice the loads in flight,
// which FP16 storage (2 bytes per load) needs to cover HBM latency.
template <class S, int K, bool MACRO>
__global__ void __launch_bounds__(256) k_bulk_m2(const StepArgs a, const MixArgs m) {
  const int s0 = blockIdx.x * 512 + threadIdx.x, s1 = s0 + 256;
  const int r0 = s0 < a.n ? __ldg(a.meta + s0) : -1;
  const int r1 = s1 < a.n ? __ldg(a.meta + s1) : -1;
  float g0[Q], g1[Q];
  if (r0 >= 0) gather_bulk_m<S>(a, m, s0, r0, g0);
  if (r1 >= 0) gather_bulk_m<S>(a, m, s1, r1, g1);
  if (r0 >= 0) bulk_collide_m<S, K, MACRO>(a, m, s0, g0);
  if (r1 >= 0) bulk_collide_m<S, K, MACRO>(a, m, s1, g1);
}

// Steady-state plain bulk sites of the FP16 shifted form (LBGK, TRT; no outputs),
// SPT sites per thread (s, s + 256, ...), all gathered before any collides (run
// with one).
// Each load is one address add: the run table row holds the plane offsets
// i * np + run_off[i] (Solver::upload).  The collision runs on the stored
// scale, G = kScale * g (kScale = kHalfScale for FP16, 1 for FP32), so a value
// is converted but never rescaled on its way in or out: with D = sum G and
// M = sum c G,
//   geq_i = w_i (D - 3/2 |M|^2 / (kScale + D) + 9/2 (c_i.M)^2 / (kScale + D) + 3 c_i.M),
// which is kScale times the unscaled equilibrium of kernels_mixed.cu's header.
// Opposite directions share the even part of the equilibrium.  The kernel is
// issue-bound (about 460 instructions a site), so the positivity check compares
// each value with its constant threshold (one predicated compare; NaN fails it
// as before) and the stores walk one pointer by the plane stride.  4M-site
// pipe, FP16 bulk kernel 0.0963 -> 0.0850 ms with the plane offsets, 0.0817 ms
// with the trimmed check and stores (0.45 -> 0.52 of the measured copy
// bandwidth), the whole FP16 step 33.1k -> 37.6k MLUPS.  With the instructions
// trimmed, one site per thread (40 registers, six blocks of 256 per SM) beats
// two (64 registers, four blocks): 0.0826 -> 0.0779 ms, step 39.3k MLUPS; three
// sites per thread measured 0.0903 ms, two held to 48 registers 0.0861 ms.
template <class S>
struct Lp;
template <>
struct Lp<float> {
  static constexpr float kScale = 1.0f;
  static __device__ __forceinline__ float ld(const void* base, int64_t k) { return __ldg(static_cast<const float*>(base) + k); }
  static __device__ __forceinline__ void st(void* base, int64_t k, float v) { static_cast<float*>(base)[k] = v; }
};
template <>
struct Lp<__half> {
  static constexpr float kScale = kHalfScale;
  static __device__ __forceinline__ float ld(const void* base, int64_t k) {
    return __half2float(__ldg(static_cast<const __half*>(base) + k));
  }
  static __device__ __forceinline__ void st(void* base, int64_t k, float v) { static_cast<__half*>(base)[k] = __float2half_rn(v); }
};

template <class S, int K>
__device__ __forceinline__ void collide_scaled(const StepArgs& a, const MixArgs& m, int s, const float* G) {
  float D = 0.0f, Mx = 0.0f, My = 0.0f, Mz = 0.0f;
  bool bad = false;
#pragma unroll
  for (int i = 0; i < Q; i++) {
    D += G[i];
    Mx += (float)cx(i) * G[i];
    My += (float)cy(i) * G[i];
    Mz += (float)cz(i) * G[i];
    bad |= !(G[i] > -wf(i) * Lp<S>::kScale);
  }
  if (bad) atomicOr(a.status, kStatusUnstable);
  const float inv = 1.0f / (Lp<S>::kScale + D);
  const float nh = 4.5f * inv;
  const float t1 = D - 1.5f * (Mx * Mx + My * My + Mz * Mz) * inv;
  float neq[Q];
  neq[0] = G[0] - wf(0) * t1;
#pragma unroll
  for (int i = 1; i < Q; i += 2) {  // (i, i + 1) are opposite directions
    const float mde = (float)cx(i) * Mx + (float)cy(i) * My + (float)cz(i) * Mz;
    const float even = wf(i) * (t1 + nh * mde * mde), odd = wf(i) * (3.0f * mde);
    neq[i] = G[i] - (even + odd);
    neq[i + 1] = G[i + 1] - (even - odd);
  }
  const float om = (float)a.omega;
  if (K == kTRT) {
    const float omm = (float)a.omega_minus;
    Lp<S>::st(m.fout, s, G[0] + om * neq[0]);
#pragma unroll
    for (int i = 1; i < Q; i += 2) {
      const float sym = 0.5f * om * (neq[i] + neq[i + 1]), asym = 0.5f * omm * (neq[i] - neq[i + 1]);
      Lp<S>::st(m.fout, (int64_t)i * a.np + s, G[i] + sym + asym);
      Lp<S>::st(m.fout, (int64_t)(i + 1) * a.np + s, G[i + 1] + sym - asym);
    }
  } else {
    S* o = static_cast<S*>(m.fout) + s;
#pragma unroll
    for (int i = 0; i < Q; i++) {
      Lp<S>::st(o, 0, G[i] + om * neq[i]);
      o += a.np;
    }
  }
}

template <class S, int K, int SPT>
__global__ void __launch_bounds__(256) k_bulk_lp(const StepArgs a, const MixArgs m) {
  const int s0 = blockIdx.x * (256 * SPT) + threadIdx.x;
  int r[SPT];
  float G[SPT][Q];
#pragma unroll
  for (int k = 0; k < SPT; k++) {
    const int s = s0 + 256 * k;
    r[k] = s < a.n ? __ldg(a.meta + s) : -1;
  }
#pragma unroll
  for (int k = 0; k < SPT; k++) {
    if (r[k] < 0) continue;
    const int s = s0 + 256 * k;
    const int4* o4 = reinterpret_cast<const int4*>(a.run_po) + 5 * r[k];
    int po[20];
#pragma unroll
    for (int j = 0; j < 5; j++) {
      const int4 v = __ldg(o4 + j);
      po[4 * j] = v.x;
      po[4 * j + 1] = v.y;
      po[4 * j + 2] = v.z;
      po[4 * j + 3] = v.w;
    }
#pragma unroll
    for (int i = 0; i < Q; i++) G[k][i] = Lp<S>::ld(m.fin, (int64_t)s + po[i]);
  }
#pragma unroll
  for (int k = 0; k < SPT; k++)
    if (r[k] >= 0) collide_scaled<S, K>(a, m, s0 + 256 * k, G[k]);
}

// The boundary kernel is latency-bound: outside the LES kernel, GZS walls and
// output steps it runs six blocks of 128 per SM (up to 80 registers), which
// holds the gather and the BFL loads in flight together (mixed_site.cuh).
// FP32 on the 4M pipe, time alone / whole step: eight blocks 0.0355 / 0.1231
// ms, six 0.0326 / 0.1211 ms, five 0.0336 / 0.1227 ms; with the BFL loads
// issued link by link and eight blocks, 0.0428 / 0.1252 ms.  FP16 storage (its
// loads half the width) runs eight: 0.0505 / 0.1021 ms at six, 0.0413 / 0.0963
// ms at eight.
template <class S, int K, int WALL, bool GATHER, bool MACRO>
__global__ void __launch_bounds__(128, (K != kLES && WALL != kGZS && !MACRO) ? (sizeof(S) == 2 ? 8 : 6) : 1)
    k_general_m(const StepArgs a, const MixArgs m, int g0) {
  const int gi = g0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (gi >= a.gen.G) return;
  general_site_m<S, K, WALL, GATHER, MACRO>(a, m, gi);
}

// The records without iolet links, compiled without the iolet rules (as the
// FP64 k_general_walls); k_general_m takes the rest beside it.
template <class S, int K, int WALL, bool GATHER, bool MACRO>
__global__ void __launch_bounds__(128, (K != kLES && WALL != kGZS && !MACRO) ? (sizeof(S) == 2 ? 8 : 6) : 1)
    k_general_m_walls(const StepArgs a, const MixArgs m) {
  const int gi = blockIdx.x * blockDim.x + threadIdx.x;
  if (gi >= a.gen.G_noiolet) return;
  general_site_m<S, K, WALL, GATHER, MACRO, false>(a, m, gi);
}

template <class S, int WALL, bool GATHER>
__global__ void __launch_bounds__(256) k_to_aos_m(const StepArgs a, const MixArgs m, const int* st2ref, double* aos) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  float g[Q];
  gather_any_m<S, WALL, GATHER>(a, m, s, g);
  const int64_t base = (int64_t)st2ref[s] * Q;
#pragma unroll
  for (int i = 0; i < Q; i++) aos[base + i] = weight(i) + (double)g[i];
}

template <class S>
__global__ void k_from_aos_m(const double* aos, const int* st2ref, int n, int64_t np, void* out) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (int64_t)n * Q) return;
  const int s = (int)(k / Q), i = (int)(k % Q);
  Store<S>::store(out, (int64_t)i * np + s, (float)(aos[(int64_t)st2ref[s] * Q + i] - weight(i)));
}

template <class S, int K, int WALL, bool GATHER, bool MACRO>
void launch_m4(const StepArgs& a, const MixArgs& m, int which, cudaStream_t st) {
  if ((which & 1) && a.n > 0) {
    // FP16 only: FP32 storage measured no faster with it (0.1060 against 0.1060 ms on the
    // 4M pipe), and keeping FP32 on the general kernel's arithmetic keeps a sharded
    // FP32 lattice bit-identical to the single lattice.
    if (GATHER && !MACRO && (K == kLBGK || K == kTRT) && a.run_po && sizeof(S) == 2)
      k_bulk_lp<S, (K == kTRT ? kTRT : kLBGK), 1><<<(a.n + 255) / 256, 256, 0, st>>>(a, m);
    else if (GATHER && sizeof(S) == 2) k_bulk_m2<S, K, MACRO><<<(a.n + 511) / 512, 256, 0, st>>>(a, m);
    else k_bulk_m<S, K, GATHER, MACRO><<<(a.n + 255) / 256, 256, 0, st>>>(a, m);
  }
  const int g0 = a.gen.G_noiolet;
  if ((which & (kLaunchBoundary | kLaunchWallRecords)) && g0 > 0)
    k_general_m_walls<S, K, WALL, GATHER, MACRO><<<(g0 + 127) / 128, 128, 0, st>>>(a, m);
  if ((which & (kLaunchBoundary | kLaunchIoletRecords)) && a.gen.G > g0)
    k_general_m<S, K, WALL, GATHER, MACRO><<<(a.gen.G - g0 + 127) / 128, 128, 0, st>>>(a, m, g0);
}

template <class S, int K, int WALL>
void launch_m2(const StepArgs& a, const MixArgs& m, bool gather, bool macro, int which, cudaStream_t st) {
  if (gather) {
    if (macro) launch_m4<S, K, WALL, true, true>(a, m, which, st);
    else launch_m4<S, K, WALL, true, false>(a, m, which, st);
  } else {
    if (macro) launch_m4<S, K, WALL, false, true>(a, m, which, st);
    else launch_m4<S, K, WALL, false, false>(a, m, which, st);
  }
}

template <class S, int K>
void launch_m1(const StepArgs& a, const MixArgs& m, int wall, bool gather, bool macro, int which, cudaStream_t st) {
  if (wall == kSBB) launch_m2<S, K, kSBB>(a, m, gather, macro, which, st);
  else if (wall == kBFL) launch_m2<S, K, kBFL>(a, m, gather, macro, which, st);
  else launch_m2<S, K, kGZS>(a, m, gather, macro, which, st);
}

template <class S>
void launch_m0(const StepArgs& a, const MixArgs& m, int kernel, int wall, bool gather, bool macro, int which, cudaStream_t st) {
  if (kernel == kLBGK) launch_m1<S, kLBGK>(a, m, wall, gather, macro, which, st);
  else if (kernel == kTRT) launch_m1<S, kTRT>(a, m, wall, gather, macro, which, st);
  else launch_m1<S, kLES>(a, m, wall, gather, macro, which, st);
}

template <class S, int WALL>
void launch_to_aos2(const StepArgs& a, const MixArgs& m, bool gather, const int* st2ref, double* aos, cudaStream_t st) {
  if (gather) k_to_aos_m<S, WALL, true><<<(a.n + 255) / 256, 256, 0, st>>>(a, m, st2ref, aos);
  else k_to_aos_m<S, WALL, false><<<(a.n + 255) / 256, 256, 0, st>>>(a, m, st2ref, aos);
}

template <class S>
void launch_to_aos1(const StepArgs& a, const MixArgs& m, int wall, bool gather, const int* st2ref, double* aos, cudaStream_t st) {
  if (wall == kBFL) launch_to_aos2<S, kBFL>(a, m, gather, st2ref, aos, st);
  else if (wall == kGZS) launch_to_aos2<S, kGZS>(a, m, gather, st2ref, aos, st);
  else launch_to_aos2<S, kSBB>(a, m, gather, st2ref, aos, st);
}

}  // namespace

void launch_step_mixed(const StepArgs& a, int precision, const void* fin, void* fout, const float* gin, float* gout,
                       int kernel, int wall, bool gather, bool macro, int which, void* stream) {
  const MixArgs m{fin, fout, gin, gout};
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == HB_STORE_FP16) launch_m0<__half>(a, m, kernel, wall, gather, macro, which, st);
  else launch_m0<float>(a, m, kernel, wall, gather, macro, which, st);
}

void launch_to_aos_mixed(const StepArgs& a, int precision, const void* fin, const float* gin, int wall, bool gather,
                         const int* st2ref, double* aos, void* stream) {
  const MixArgs m{fin, nullptr, gin, nullptr};
  if (a.n <= 0) return;
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == HB_STORE_FP16) launch_to_aos1<__half>(a, m, wall, gather, st2ref, aos, st);
  else launch_to_aos1<float>(a, m, wall, gather, st2ref, aos, st);
}

void launch_from_aos_mixed(const double* aos, const int* st2ref, int n, int64_t np, int precision, void* out, void* stream) {
  const int64_t tot = (int64_t)n * Q;
  if (tot <= 0) return;
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned blocks = (unsigned)((tot + 255) / 256);
  if (precision == HB_STORE_FP16) k_from_aos_m<__half><<<blocks, 256, 0, st>>>(aos, st2ref, n, np, out);
  else k_from_aos_m<float><<<blocks, 256, 0, st>>>(aos, st2ref, n, np, out);
}

}  // namespace hb
