// mixed_site.cuh -- per-site routines of the shifted low-precision forms
// (g = f - w rho0 stored in FP32 or scaled FP16, FP32 collision), shared by the
// single-lattice kernels (kernels_mixed.cu) and the batched persistent kernel
// (kernels_batch.cu).  See kernels_mixed.cu for the formulation.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "../../include/hemeb200.h"
#include "device.h"
#include "hb_common.h"

namespace hb {
namespace {

template <class S>
struct Store;

template <>
struct Store<float> {
  static __device__ __forceinline__ float load(const void* p, int64_t k) { return __ldg(static_cast<const float*>(p) + k); }
  static __device__ __forceinline__ void store(void* p, int64_t k, float v) { static_cast<float*>(p)[k] = v; }
};

// FP16 holds g * kHalfScale; the scale is a power of two, so scaling is exact.
template <>
struct Store<__half> {
  static __device__ __forceinline__ float load(const void* p, int64_t k) {
    return __half2float(__ldg(static_cast<const __half*>(p) + k)) * (1.0f / kHalfScale);
  }
  static __device__ __forceinline__ void store(void* p, int64_t k, float v) {
    static_cast<__half*>(p)[k] = __float2half_rn(v * kHalfScale);
  }
};

__device__ __forceinline__ float wf(int i) { return (float)weight(i); }

struct GeqF {
  float drho, rho, mx, my, mz, t1, nh;
  __device__ __forceinline__ GeqF(float dr, float x, float y, float z) : drho(dr), mx(x), my(y), mz(z) {
    rho = 1.0f + drho;
    const float inv = 1.0f / rho;
    nh = 4.5f * inv;
    t1 = drho - 1.5f * (mx * mx + my * my + mz * mz) * inv;
  }
  __device__ __forceinline__ float mde(int i) const { return (float)cx(i) * mx + (float)cy(i) * my + (float)cz(i) * mz; }
  // w_i (t1 + nh (c_i.m)^2) + w_i 3 (c_i.m), each operation rounded as written,
  // so that all() below gives the same bits.
  __device__ __forceinline__ float operator()(int i) const {
    const float e = mde(i);
    const float even = __fmul_rn(wf(i), __fmaf_rn(__fmul_rn(nh, e), e, t1));
    const float odd = __fmul_rn(wf(i), __fmul_rn(3.0f, e));
    return __fadd_rn(even, odd);
  }
  // Every direction's value; opposite directions (i, i + 1) share the even part.
  __device__ __forceinline__ void all(float* out) const {
    out[0] = (*this)(0);
#pragma unroll
    for (int i = 1; i < Q; i += 2) {
      const float e = mde(i);
      const float even = __fmul_rn(wf(i), __fmaf_rn(__fmul_rn(nh, e), e, t1));
      const float odd = __fmul_rn(wf(i), __fmul_rn(3.0f, e));
      out[i] = __fadd_rn(even, odd);
      out[i + 1] = __fsub_rn(even, odd);
    }
  }
};

__device__ __forceinline__ void moments_g(const float* g, float& drho, float& mx, float& my, float& mz) {
  drho = mx = my = mz = 0.0f;
#pragma unroll
  for (int i = 0; i < Q; i++) {
    drho += g[i];
    mx += (float)cx(i) * g[i];
    my += (float)cy(i) * g[i];
    mz += (float)cz(i) * g[i];
  }
}

__device__ __forceinline__ float les_tau_f(const StepArgs& a, const float* fneq, float vt) {
  const float tau0 = (float)a.tau;
  float q12 = 0.0f;
#pragma unroll
  for (int p = 0; p < 3; p++)
#pragma unroll
    for (int r = 0; r < 3; r++) {
      float qij = 0.0f;
#pragma unroll
      for (int v = 0; v < Q; v++) qij += (float)(cc(p, v) * cc(r, v)) * fneq[v];
      q12 += qij * qij;
    }
  q12 = sqrtf(q12);
  const float ks = (float)(18.0 * 1.4142135623730950488016887242097 * 0.01);
  const float tau_les = 0.5f * (tau0 + sqrtf(tau0 * tau0 + ks * q12));
  if (a.t <= a.lifetime / 2) return (vt == tau0) ? tau_les : vt;
  if (a.t < a.lifetime) return (tau_les - vt) * 2.0f / (float)a.lifetime * (float)a.t + (2.0f * vt - tau_les);
  return tau_les;
}

template <int K>
__device__ __forceinline__ float collide_one_f(const StepArgs& a, const float* g, const float* fneq, float om, int i) {
  if (K == kTRT) {
    const float op = (float)a.omega, omm = (float)a.omega_minus;
    if (i == 0) return g[0] + op * fneq[0];
    const int j = inv(i);
    const float sym = 0.5f * op * (fneq[i] + fneq[j]);
    const float asym = 0.5f * omm * (fneq[i] - fneq[j]);
    return g[i] + sym + asym;
  }
  return g[i] + fneq[i] * om;
}

__device__ __forceinline__ double wss_mag_f(float tau, const float* gp, const float* g, const float nor[3]) {
  float pi[3][3];
#pragma unroll
  for (int p = 0; p < 3; p++)
#pragma unroll
    for (int r = 0; r <= p; r++) {
      float acc = 0.0f;
#pragma unroll
      for (int l = 0; l < Q; l++) acc += (gp[l] - g[l]) * (float)(cc(p, l) * cc(r, l));
      pi[p][r] = acc * -(tau - 0.5f);
    }
  pi[0][1] = pi[1][0];
  pi[0][2] = pi[2][0];
  pi[1][2] = pi[2][1];
  float sq = 0.0f, ns = 0.0f;
#pragma unroll
  for (int p = 0; p < 3; p++) {
    const float sv = pi[p][0] * nor[0] + pi[p][1] * nor[1] + pi[p][2] * nor[2];
    sq += sv * sv;
    ns += sv * nor[p];
  }
  return (double)sqrtf(fmaxf(sq - ns * ns, 0.0f));
}

// Momentum flux tensor of an output step for the stress caches (FP32 sums of the
// shifted values: gp - g equals fp - f), stored as FP64 like store_pi.
__device__ __forceinline__ void store_pi_f(const StepArgs& a, int s, float tau, const float* gp, const float* g) {
  float pi[3][3];
#pragma unroll
  for (int p = 0; p < 3; p++)
#pragma unroll
    for (int r = 0; r <= p; r++) {
      float acc = 0.0f;
#pragma unroll
      for (int l = 0; l < Q; l++) acc += (gp[l] - g[l]) * (float)(cc(p, l) * cc(r, l));
      pi[p][r] = acc * -(tau - 0.5f);
    }
  double* o = a.pi + s;
  o[0] = (double)pi[0][0];
  o[a.np] = (double)pi[1][0];
  o[2 * a.np] = (double)pi[2][0];
  o[3 * a.np] = (double)pi[1][1];
  o[4 * a.np] = (double)pi[2][1];
  o[5 * a.np] = (double)pi[2][2];
  o[6 * a.np] = (double)tau;
}

__device__ __forceinline__ bool parabolic_f(const IoletDev& I, const double x[3], uint64_t t, float v[3]) {
  const double dx = x[0] - I.pos[0], dy = x[1] - I.pos[1], dz = x[2] - I.pos[2];
  const double z = dx * I.nrm[0] + dy * I.nrm[1] + dz * I.nrm[2];
  const double rsq = (dx * dx + dy * dy + dz * dz) - z * z;
  const double r2a2 = rsq / (I.radius * I.radius);
  double mx = I.max_speed;
  if (t < I.warmup) mx *= (double)t / (double)I.warmup;
  const double s = mx * (1. - r2a2);
  v[0] = (float)(I.nrm[0] * s);
  v[1] = (float)(I.nrm[1] * s);
  v[2] = (float)(I.nrm[2] * s);
  return !(r2a2 > 1.0);
}

// The velocity of a velocity iolet's link d of general site gi (parabolic, file
// velocity or Womersley; half-way point or neighbour as for the FP64 kernels),
// evaluated in FP64 and narrowed.
__device__ __forceinline__ bool link_velocity_f(const StepArgs& a, const IoletDev& I, int io, int gi, int d, bool half,
                                                const double pos[3], float v[3]) {
  if (I.kind == kWomersley) {
    const double* A = a.wom_amp + ((int64_t)__ldg(a.gen.wom + gi) * 18 + (d - 1)) * 4 + (half ? 0 : 2);
    const double speed = __ldg(A) * a.dens_row[kRowA + io] - __ldg(A + 1) * a.dens_row[kRowB + io];
    v[0] = (float)(I.nrm[0] * -speed);
    v[1] = (float)(I.nrm[1] * -speed);
    v[2] = (float)(I.nrm[2] * -speed);
    return true;
  }
  const double h = half ? 0.5 : 1.0;
  const double x[3] = {pos[0] + h * cx(d), pos[1] + h * cy(d), pos[2] + h * cz(d)};
  if (I.kind == kParabolic) return parabolic_f(I, x, (uint64_t)(unsigned int)a.t, v);
  const double dx = x[0] - I.pos[0], dy = x[1] - I.pos[1], dz = x[2] - I.pos[2];
  const double z = dx * I.nrm[0] + dy * I.nrm[1] + dz * I.nrm[2];
  const double r2a2 = ((dx * dx + dy * dy + dz * dz) - z * z) / (I.radius * I.radius);
  const double s = a.dens_row[kRowA + io] * (1. - r2a2);
  v[0] = (float)(I.nrm[0] * s);
  v[1] = (float)(I.nrm[1] * s);
  v[2] = (float)(I.nrm[2] * s);
  return !(r2a2 > 1.0);
}

__device__ __forceinline__ void run_offsets(const StepArgs& a, int r, int* off) {
  const int4* o4 = reinterpret_cast<const int4*>(a.run_off) + 5 * r;
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const int4 v = __ldg(o4 + k);
    off[4 * k] = v.x;
    off[4 * k + 1] = v.y;
    off[4 * k + 2] = v.z;
    off[4 * k + 3] = v.w;
  }
}

// Arguments of the shifted kernels: StepArgs for the shared tables, plus typed
// storage pointers (fin/fout/gin/gout of StepArgs are unused here).
struct MixArgs {
  const void* fin;
  void* fout;
  const float* gin;
  float* gout;
};

template <class S>
__device__ __forceinline__ float ldg_s(const MixArgs& m, int64_t k) { return Store<S>::load(m.fin, k); }

template <class S>
__device__ __forceinline__ void gather_bulk_m(const StepArgs& a, const MixArgs& m, int s, int r, float* g) {
  if (a.run_po) {
    // The run table's plane offsets i * np + run_off[i]: one add per load.
    const int4* o4 = reinterpret_cast<const int4*>(a.run_po) + 5 * r;
    int po[20];
#pragma unroll
    for (int k = 0; k < 5; k++) {
      const int4 v = __ldg(o4 + k);
      po[4 * k] = v.x;
      po[4 * k + 1] = v.y;
      po[4 * k + 2] = v.z;
      po[4 * k + 3] = v.w;
    }
    const S* base = static_cast<const S*>(m.fin) + s;
#pragma unroll
    for (int i = 0; i < Q; i++) g[i] = Store<S>::load(base, po[i]);
    return;
  }
  int off[20];
  run_offsets(a, r, off);
  g[0] = ldg_s<S>(m, s);
#pragma unroll
  for (int i = 1; i < Q; i++) g[i] = ldg_s<S>(m, (int64_t)i * a.np + (s + off[i]));
}

// Every slot's first value is one load (predicated between the ghost buffer and
// the distributions, with no branch on the link masks): the ghost of an iolet
// link, g*_d of the own site for a wall link, g*_i of the source site otherwise
// (s + run offset for a record that follows its run, else its pull table).  The
// BFL correction of wall links follows as a predicated step (as the FP64 kernel).
template <class S, int WALL, bool IO = true>
__device__ __forceinline__ void gather_general_m(const StepArgs& a, const MixArgs& m, int gi, int s, float* g) {
  const GeneralDev& G = a.gen;
  const uint32_t wm = __ldg(G.wall + gi), im = IO ? __ldg(G.iolet + gi) : 0u;
  const int run = __ldg(G.run + gi);
  int src[18];
  if (run >= 0) {
    int off[20];
    run_offsets(a, run, off);
#pragma unroll
    for (int i = 1; i < Q; i++) src[i - 1] = s + off[i];
  } else {
#pragma unroll
    for (int i = 1; i < Q; i++) src[i - 1] = __ldg(G.src + (int64_t)(i - 1) * G.G + gi);
  }
  g[0] = ldg_s<S>(m, s);
#pragma unroll
  for (int i = 1; i < Q; i++) {
    const int d = inv(i);
    const bool bw = (wm >> (d - 1)) & 1u, bi = (im >> (d - 1)) & 1u;
    const int64_t k = bw ? (int64_t)d * a.np + s : (int64_t)i * a.np + src[i - 1];
    float v;
    if (bi) v = __ldg(m.gin + (int64_t)(d - 1) * G.G + gi);
    else v = ldg_s<S>(m, k);
    g[i] = v;
  }
  if (WALL == kBFL && wm) {
    // The BFL rule of gather_general (f64_site.cuh), in FP32 on the stored
    // deviations; cut distances and own-site values loaded before any arithmetic.
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

template <class S, int WALL, bool GATHER>
__device__ __forceinline__ void gather_any_m(const StepArgs& a, const MixArgs& m, int s, float* g) {
  if (!GATHER) {
#pragma unroll
    for (int i = 0; i < Q; i++) g[i] = ldg_s<S>(m, (int64_t)i * a.np + s);
    return;
  }
  const int r = __ldg(a.meta + s);
  if (r >= 0) gather_bulk_m<S>(a, m, s, r, g);
  else gather_general_m<S, WALL>(a, m, -r - 1, s, g);
}

__device__ __forceinline__ void flag_unstable_status(const float* g, int* status) {
  bool bad = false;
#pragma unroll
  for (int i = 0; i < Q; i++) bad |= !(g[i] > -wf(i));
  if (bad) atomicOr(status, kStatusUnstable);
}

__device__ __forceinline__ void flag_unstable_m(const StepArgs& a, const float* g) { flag_unstable_status(g, a.status); }

// Collision and store of plain bulk site s from its pre-collision g.  The bulk
// kernels issue about 490 instructions a site for 152 bytes (FP32), so the
// equilibrium is evaluated by pairs of opposite directions and the stores walk
// one pointer (4M pipe, FP32 bulk kernel 0.1065 -> 0.1038 ms, 0.83 -> 0.85 of
// the measured copy bandwidth).
template <class S, int K, bool MACRO>
__device__ __forceinline__ void bulk_collide_m(const StepArgs& a, const MixArgs& m, int s, const float* g) {
  flag_unstable_m(a, g);
  float drho, mx, my, mz;
  moments_g(g, drho, mx, my, mz);
  const GeqF geq(drho, mx, my, mz);
  float fneq[Q];
  geq.all(fneq);
#pragma unroll
  for (int i = 0; i < Q; i++) fneq[i] = g[i] - fneq[i];
  float om = (float)a.omega, tau = (float)a.tau;
  if (K == kLES) {
    tau = les_tau_f(a, fneq, (float)__ldg(a.vtau + s));
    om = -1.0f / tau;
  }
  {
    S* o = static_cast<S*>(m.fout) + s;
#pragma unroll
    for (int i = 0; i < Q; i++) {
      Store<S>::store(o, 0, collide_one_f<K>(a, g, fneq, om, i));
      o += a.np;
    }
  }
  if (MACRO) {
    const float rho = 1.0f + drho;
    a.rho[s] = (double)rho;
    a.u[s] = (double)(mx / rho);
    a.u[a.np + s] = (double)(my / rho);
    a.u[2 * a.np + s] = (double)(mz / rho);
    a.wss[s] = kNoValue;
    if (a.pi) {
      float gp[Q];
#pragma unroll
      for (int i = 0; i < Q; i++) gp[i] = collide_one_f<K>(a, g, fneq, om, i);
      store_pi_f(a, s, tau, gp, g);
    }
  }
}

// One plain bulk site s of run r (k_bulk_m, and the batched kernel).
template <class S, int K, bool GATHER, bool MACRO>
__device__ __forceinline__ void bulk_site_m(const StepArgs& a, const MixArgs& m, int s, int r) {
  float g[Q];
  if (GATHER) gather_bulk_m<S>(a, m, s, r, g);
  else {
#pragma unroll
    for (int i = 0; i < Q; i++) g[i] = ldg_s<S>(m, (int64_t)i * a.np + s);
  }
  bulk_collide_m<S, K, MACRO>(a, m, s, g);
}

// One general site gi (k_general_m, and the batched kernel).
template <class S, int K, int WALL, bool GATHER, bool MACRO, bool IO = true>
__device__ __forceinline__ void general_site_m(const StepArgs& a, const MixArgs& m, int gi) {
  const GeneralDev& G = a.gen;
  const int s = __ldg(G.site + gi);
  const uint32_t wm = __ldg(G.wall + gi), im = IO ? __ldg(G.iolet + gi) : 0u;
  float g[Q];
  if (GATHER) gather_general_m<S, WALL, IO>(a, m, gi, s, g);
  else {
#pragma unroll
    for (int i = 0; i < Q; i++) g[i] = ldg_s<S>(m, (int64_t)i * a.np + s);
  }
  flag_unstable_m(a, g);
  float drho, mx, my, mz;
  moments_g(g, drho, mx, my, mz);
  const float rho = 1.0f + drho;
  const float ux = mx / rho, uy = my / rho, uz = mz / rho;
  const GeqF geq(drho, mx, my, mz);
  float fneq[Q];
#pragma unroll
  for (int i = 0; i < Q; i++) fneq[i] = g[i] - geq(i);
  float om = (float)a.omega, tau = (float)a.tau;
  if (K == kLES) {
    tau = les_tau_f(a, fneq, (float)__ldg(a.vtau + s));
    om = -1.0f / tau;
  }
  float gp[Q], out[Q];
#pragma unroll
  for (int i = 0; i < Q; i++) out[i] = gp[i] = collide_one_f<K>(a, g, fneq, om, i);
  int io = -1;
  if (im) {
    io = __ldg(G.io + gi);
    const IoletDev& I = a.iolets[io];
    const double pos[3] = {(double)__ldg(G.xyz + gi), (double)__ldg(G.xyz + G.G + gi), (double)__ldg(G.xyz + 2 * G.G + gi)};
#pragma unroll
    for (int d = 1; d < Q; d++) {
      if (!((im >> (d - 1)) & 1u)) continue;
      float v;
      if (is_velocity_iolet(I.kind)) {
        float w[3];
        if (!link_velocity_f(a, I, io, gi, d, true, pos, w)) {
          atomicOr(a.status, kStatusIoletRadius);
          w[0] = w[1] = w[2] = 0.0f;
        }
        const float corr = 2.0f * wf(d) * rho * (w[0] * cx(d) + w[1] * cy(d) + w[2] * cz(d)) * 3.0f;
        v = gp[d] - corr;
      } else {
        const double rb = a.dens_row[io];
        const float drb = (float)(rb - 1.0);
        const float rbf = (float)rb;
        const float nx = (float)I.nrm_f[0], ny = (float)I.nrm_f[1], nz = (float)I.nrm_f[2];
        const float comp = ux * nx + uy * ny + uz * nz;
        const GeqF gq(drb, nx * comp * rbf, ny * comp * rbf, nz * comp * rbf);
        v = gq(inv(d));
      }
      m.gout[(int64_t)(d - 1) * G.G + gi] = v;
    }
  }
  if (WALL == kGZS && wm) {
#pragma unroll
    for (int d = 1; d < Q; d++) {
      if (!((wm >> (d - 1)) & 1u)) continue;
      const int i = inv(d);
      const float q = __ldg(G.q + (int64_t)(d - 1) * G.G + gi);
      const float fac = 1.0f - 1.0f / q;
      float mw0 = mx * fac, mw1 = my * fac, mw2 = mz * fac;
      float fnw_i = fneq[i], fnw_d = fneq[d];
      bool sbb = false;
      if (q < 0.75f) {
        if ((im >> (i - 1)) & 1u) {
          const IoletDev& I = a.iolets[io];
          if (!is_velocity_iolet(I.kind)) {
            sbb = true;
          } else {
            const double p3[3] = {(double)__ldg(G.xyz + gi), (double)__ldg(G.xyz + G.G + gi), (double)__ldg(G.xyz + 2 * G.G + gi)};
            float nv[3];
            if (!link_velocity_f(a, I, io, gi, i, false, p3, nv)) {
              atomicOr(a.status, kStatusIoletRadius);
              nv[0] = nv[1] = nv[2] = 0.0f;
            }
            const float k2 = (1.0f - q) * rho * (q - 1.0f) / (q + 1.0f);
            mw0 = q * mw0 + k2 * nv[0];
            mw1 = q * mw1 + k2 * nv[1];
            mw2 = q * mw2 + k2 * nv[2];
          }
        } else if ((wm >> (i - 1)) & 1u) {
          sbb = true;
        } else {
          const int grun = __ldg(G.run + gi);
          const int nb = grun >= 0 ? s + __ldg(a.run_off + 20 * grun + d) : __ldg(G.src + (int64_t)(d - 1) * G.G + gi);
          float gn[Q];
          gather_any_m<S, WALL, GATHER>(a, m, nb, gn);
          float dn, mnx, mny, mnz;
          moments_g(gn, dn, mnx, mny, mnz);
          const float rn = 1.0f + dn;
          const GeqF gqn(dn, mnx, mny, mnz);
          const float k2 = (1.0f - q) * rho * (q - 1.0f) / (q + 1.0f) / rn;
          mw0 = q * mw0 + k2 * mnx;
          mw1 = q * mw1 + k2 * mny;
          mw2 = q * mw2 + k2 * mnz;
          fnw_i = q * fnw_i + (1.0f - q) * (gn[i] - gqn(i));
          fnw_d = q * fnw_d + (1.0f - q) * (gn[d] - gqn(d));
        }
      }
      if (sbb) continue;
      const GeqF gw(drho, mw0, mw1, mw2);
      const float gw_i = gw(i) + fnw_i;
      float v;
      if (K == kTRT) {
        const float sym = 0.5f * (float)a.omega * (fnw_i + fnw_d);
        const float asym = 0.5f * (float)a.omega_minus * (fnw_i - fnw_d);
        v = gw_i + sym + asym;
      } else {
        v = gw_i + fnw_i * om;
      }
      out[d] = v;
    }
  }
#pragma unroll
  for (int i = 0; i < Q; i++) Store<S>::store(m.fout, (int64_t)i * a.np + s, out[i]);
  const int cpl = im ? __ldg(G.cpl + gi) : -1;
  if (cpl >= 0) {
    const IoletDev& I = a.iolets[io];
    a.cpl_buf[cpl] = (double)ux * (-I.nrm[0]) + (double)uy * (-I.nrm[1]) + (double)uz * (-I.nrm[2]);
  }
  if (MACRO) {
    a.rho[s] = (double)rho;
    a.u[s] = (double)ux;
    a.u[a.np + s] = (double)uy;
    a.u[2 * a.np + s] = (double)uz;
    if (wm) {
      const float nor[3] = {__ldg(G.nrm + gi), __ldg(G.nrm + G.G + gi), __ldg(G.nrm + 2 * G.G + gi)};
      a.wss[s] = wss_mag_f(tau, gp, g, nor);
    } else {
      a.wss[s] = kNoValue;
    }
    if (a.pi) store_pi_f(a, s, tau, gp, g);
  }
}

// Pre-collision f (FP64, AoS, reference order) from the shifted storage.
}  // namespace
}  // namespace hb
