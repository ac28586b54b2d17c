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

// The boundary kernel is latency-bound: outside the LES kernel, GZS walls and
// output steps it is held to 64 registers (eight blocks of 128 per SM; its own
// allocation is 68-72), measured 30.3k -> 30.7k MLUPS for the FP32 step on the 4M pipe.
template <class S, int K, int WALL, bool GATHER, bool MACRO>
__global__ void __launch_bounds__(128, (K != kLES && WALL != kGZS && !MACRO) ? 8 : 1)
    k_general_m(const StepArgs a, const MixArgs m) {
  const int gi = blockIdx.x * blockDim.x + threadIdx.x;
  if (gi >= a.gen.G) return;
  general_site_m<S, K, WALL, GATHER, MACRO>(a, m, gi);
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
    if (GATHER && sizeof(S) == 2) k_bulk_m2<S, K, MACRO><<<(a.n + 511) / 512, 256, 0, st>>>(a, m);
    else k_bulk_m<S, K, GATHER, MACRO><<<(a.n + 255) / 256, 256, 0, st>>>(a, m);
  }
  if ((which & 2) && a.gen.G > 0) k_general_m<S, K, WALL, GATHER, MACRO><<<(a.gen.G + 127) / 128, 128, 0, st>>>(a, m);
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
