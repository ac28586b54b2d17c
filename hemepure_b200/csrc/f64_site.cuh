// f64_site.cuh -- per-site device routines of the FP64 collide-and-stream step
// (kernels_f64.cu).  Every translation unit that includes it is compiled with
// -fmad=false: each product and sum is rounded separately, in the association
// order of the reference's SSE3 build.
#pragma once

#include <cuda_runtime.h>

#include "device.h"
#include "hb_common.h"

namespace hb {
namespace {

// ---------------------------------------------------------------------------
// Lattice maths in the reference's SSE3 order (src/lb/lattices/Lattice.h:51-110, 374-448).
// ---------------------------------------------------------------------------

__device__ __forceinline__ void moments(const double* f, double& rho, double& mx, double& my, double& mz) {
  double dl = 0.0, dh = f[18];
  double xl = 0.0, xh = (double)cx(18) * f[18];
  double yl = 0.0, yh = (double)cy(18) * f[18];
  double zl = 0.0, zh = (double)cz(18) * f[18];
#pragma unroll
  for (int d = 0; d < 18; d += 2) {
    dl = dl + f[d];
    dh = dh + f[d + 1];
    xl = xl + (double)cx(d) * f[d];
    xh = xh + (double)cx(d + 1) * f[d + 1];
    yl = yl + (double)cy(d) * f[d];
    yh = yh + (double)cy(d + 1) * f[d + 1];
    zl = zl + (double)cz(d) * f[d];
    zh = zh + (double)cz(d + 1) * f[d + 1];
  }
  rho = dl + dh;
  mx = xl + xh;
  my = yl + yh;
  mz = zl + zh;
}

struct FeqConst {
  double rho, mx, my, mz, t1, nh;
  __device__ __forceinline__ FeqConst(double r, double x, double y, double z) : rho(r), mx(x), my(y), mz(z) {
    const double th = (3. / 2.) * (mx * mx + my * my + mz * mz);
    const double d1 = 1. / rho;
    nh = (9. / 2.) * d1;
    t1 = rho - th * d1;
  }
  __device__ __forceinline__ double operator()(int i) const {
    const double mde = (double)cx(i) * mx + (double)cy(i) * my + (double)cz(i) * mz;
    return weight(i) * ((t1 + nh * (mde * mde)) + 3. * mde);
  }
};

// Relaxation time of the LES kernel (LBGKLESSpongeLayer::CalculateTau and
// compute_tau_smagorinsky, src/lb/kernels/LBGKLESSpongeLayer.h:122-182).
__device__ __forceinline__ double les_tau(const StepArgs& a, const double* fneq, double vt) {
  const double tau0 = a.tau;
  double q12 = 0.0;
#pragma unroll
  for (int p = 0; p < 3; p++)
#pragma unroll
    for (int r = 0; r < 3; r++) {
      double qij = 0.0;
#pragma unroll
      for (int v = 0; v < Q; v++) qij += (double)(cc(p, v) * cc(r, v)) * fneq[v];
      q12 += qij * qij;
    }
  q12 = sqrt(q12);
  constexpr double kSmag = 18.0 * 1.4142135623730950488016887242097 * 1.0 * 0.1 * 0.1;
  const double tau_les = 1. / 2. * (tau0 + sqrt((tau0 * 1.0 * 1.0) * (tau0 * 1.0 * 1.0) + kSmag * q12) / (1.0 * 1.0));
  if (a.t <= a.lifetime / 2) return (vt == tau0) ? tau_les : vt;
  if (a.t < a.lifetime) return (tau_les - vt) * 2.0 / (double)a.lifetime * (double)a.t + (2.0 * vt - tau_les);
  return tau_les;
}

// Relaxation time of the LBGK and TRT sponge-layer kernels (CalculateTau,
// src/lb/kernels/LBGKSpongeLayer.h:124-140, TRTSpongeLayer.h:157-172): the site's
// sponge time for the first half of the lifetime, then a linear return to tau0.
__device__ __forceinline__ double sponge_tau(const StepArgs& a, double vt) {
  const double tau0 = a.tau;
  if (a.t <= a.lifetime / 2) return vt;
  if (a.t < a.lifetime) return (tau0 - vt) * 2.0 / (double)a.lifetime * (double)a.t + (2.0 * vt - tau0);
  return tau0;
}

// Post-collision value of direction i for kernel K (LBGK.h:64-72, TRT.h:80-109,
// and the sponge-layer kernels).  `omega_site` is the site's -1/tau for LBGK,
// LES and LBGKSL, and its antisymmetric rate for TRTSL, whose symmetric rate stays
// the global omega (TRTSpongeLayer.h:86-115).
template <int K>
__device__ __forceinline__ double collide_one(const StepArgs& a, const double* f, const double* fneq, double omega_site, int i) {
  if (K == kTRT || K == kTRTSL) {
    const double omm = K == kTRT ? a.omega_minus : omega_site;
    if (i == 0) return f[0] + (0.5 * a.omega * (fneq[0] + fneq[0])) - (0.5 * omm * (fneq[0] - fneq[0]));
    const int j = inv(i);
    const int lo = i < j ? i : j, hi = i < j ? j : i;
    const double sym = 0.5 * a.omega * (fneq[lo] + fneq[hi]);
    const double asym = 0.5 * omm * (fneq[lo] - fneq[hi]);
    return i == lo ? (f[i] + sym + asym) : (f[i] + sym - asym);
  }
  return f[i] + fneq[i] * omega_site;
}

// The site's relaxation time and the rate collide_one takes for kernel K.
template <int K>
__device__ __forceinline__ void site_rates(const StepArgs& a, const double* fneq, int s, double& tau, double& om) {
  tau = a.tau;
  om = a.omega;
  if (K == kLES) {
    tau = les_tau(a, fneq, __ldg(a.vtau + s));
    om = -1.0 / tau;
  } else if (K == kLBGKSL) {
    tau = sponge_tau(a, __ldg(a.vtau + s));
    om = -1.0 / tau;
  } else if (K == kTRTSL) {
    tau = sponge_tau(a, __ldg(a.vtau + s));
    const double tau_minus = 0.5 + a.lambda / (tau - 0.5);
    om = -1.0 / tau_minus;
  }
}

// Wall-shear-stress magnitude (Lattice::CalculateWallShearStressMagnitude,
// CalculatePiTensor; src/lb/lattices/Lattice.h:1122-1156, 1353-1383).
__device__ __forceinline__ double wss_mag(double tau, const double* fpost, const double* f, const double nor[3]) {
  double pi[3][3];
#pragma unroll
  for (int p = 0; p < 3; p++)
#pragma unroll
    for (int r = 0; r <= p; r++) {
      double acc = 0.0;
#pragma unroll
      for (int l = 0; l < Q; l++) acc += (fpost[l] - f[l]) * (double)cc(p, l) * (double)cc(r, l);
      pi[p][r] = acc * -(tau - 0.5);
    }
  pi[0][1] = pi[1][0];
  pi[0][2] = pi[2][0];
  pi[1][2] = pi[2][1];
  double sv[3] = {0.0, 0.0, 0.0}, sq = 0.0, ns = 0.0;
#pragma unroll
  for (int p = 0; p < 3; p++) {
#pragma unroll
    for (int r = 0; r < 3; r++) sv[p] += pi[p][r] * nor[r];
    sq += sv[p] * sv[p];
    ns += sv[p] * nor[p];
  }
  return sqrt(sq - ns * ns);
}

// Non-equilibrium momentum flux tensor of an output step, stored for the stress
// caches: the lower triangle in CalculatePiTensor's order and rounding
// (src/lb/lattices/Lattice.h:1353-1383) as xx, xy, xz, yy, yz, zz, then tau.
__device__ __forceinline__ void store_pi(const StepArgs& a, int s, double tau, const double* fpost, const double* f) {
  double pi[3][3];
#pragma unroll
  for (int p = 0; p < 3; p++)
#pragma unroll
    for (int r = 0; r <= p; r++) {
      double acc = 0.0;
#pragma unroll
      for (int l = 0; l < Q; l++) acc += (fpost[l] - f[l]) * (double)cc(p, l) * (double)cc(r, l);
      pi[p][r] = acc * -(tau - 0.5);
    }
  double* o = a.pi + s;
  o[0] = pi[0][0];
  o[a.np] = pi[1][0];
  o[2 * a.np] = pi[2][0];
  o[3 * a.np] = pi[1][1];
  o[4 * a.np] = pi[2][1];
  o[5 * a.np] = pi[2][2];
  o[6 * a.np] = tau;
}

// InOutLetParabolicVelocity::GetVelocity (src/lb/iolets/InOutLetParabolicVelocity.cc:30-58).
__device__ __forceinline__ bool parabolic(const IoletDev& I, const double x[3], uint64_t t, double v[3]) {
  const double dx = x[0] - I.pos[0], dy = x[1] - I.pos[1], dz = x[2] - I.pos[2];
  const double z = dx * I.nrm[0] + dy * I.nrm[1] + dz * I.nrm[2];
  const double rsq = (dx * dx + dy * dy + dz * dz) - z * z;
  const double r2a2 = rsq / (I.radius * I.radius);
  double mx = I.max_speed;
  if (t < I.warmup) mx *= (double)t / (double)I.warmup;
  const double s = mx * (1. - r2a2);
  v[0] = I.nrm[0] * s;
  v[1] = I.nrm[1] * s;
  v[2] = I.nrm[2] * s;
  return !(r2a2 > 1.0);
}

// InOutLetVelocity::GetVelocity of a velocity iolet for link d of general site g:
// at the Ladd half-way point pos + c_d / 2 (half) or at the neighbour pos + c_d
// (the GZS extrapolation).  Parabolic: the profile above.  File velocity
// (src/lb/iolets/InOutLetFileVelocity.cc:104-128): the same profile with the
// step's peak speed from the iolet row.  Womersley
// (src/lb/iolets/InOutLetWomersleyVelocity.cc:25-41): Re(A exp(i omega t)) along
// -normal, A from the link table and exp(i omega t) from the iolet row, the
// product's real part rounded as the host's complex multiply rounds it.
// Returns false for a point outside a parabolic profile's radius.
__device__ __forceinline__ bool link_velocity(const StepArgs& a, const IoletDev& I, int io, int g, int d, bool half,
                                              const double pos[3], double v[3]) {
  if (I.kind == kWomersley) {
    const double* A = a.wom_amp + ((int64_t)__ldg(a.gen.wom + g) * 18 + (d - 1)) * 4 + (half ? 0 : 2);
    const double re = __ldg(A), im = __ldg(A + 1);
    const double speed = re * a.dens_row[kRowA + io] - im * a.dens_row[kRowB + io];
    v[0] = I.nrm[0] * -speed;
    v[1] = I.nrm[1] * -speed;
    v[2] = I.nrm[2] * -speed;
    return true;
  }
  double x[3] = {pos[0], pos[1], pos[2]};
  if (half) {
    x[0] += 0.5 * cx(d);
    x[1] += 0.5 * cy(d);
    x[2] += 0.5 * cz(d);
  } else {
    x[0] += cx(d);
    x[1] += cy(d);
    x[2] += cz(d);
  }
  if (I.kind == kParabolic) return parabolic(I, x, (uint64_t)(unsigned int)a.t, v);
  const double dx = x[0] - I.pos[0], dy = x[1] - I.pos[1], dz = x[2] - I.pos[2];
  const double z = dx * I.nrm[0] + dy * I.nrm[1] + dz * I.nrm[2];
  const double rsq = (dx * dx + dy * dy + dz * dz) - z * z;
  const double r2a2 = rsq / (I.radius * I.radius);
  const double s = a.dens_row[kRowA + io] * (1. - r2a2);
  v[0] = I.nrm[0] * s;
  v[1] = I.nrm[1] * s;
  v[2] = I.nrm[2] * s;
  return !(r2a2 > 1.0);
}

__device__ __forceinline__ double ld(const double* p) { return __ldg(p); }

// Pre-collision f of a plain bulk site.
__device__ __forceinline__ void load_run_offsets(const StepArgs& a, int r, int* off);

__device__ __forceinline__ void gather_bulk(const StepArgs& a, int s, int r, double* f) {
  int off[20];
  load_run_offsets(a, r, off);
  f[0] = ld(a.fin + s);
#pragma unroll
  for (int i = 1; i < Q; i++) f[i] = ld(a.fin + (int64_t)i * a.np + (s + off[i]));
}

// Pre-collision f of general site g (rules above).
__device__ __forceinline__ void load_run_offsets(const StepArgs& a, int r, int* off) {
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

// Every slot's first value is one load whose address needs no branch: the
// ghost of an iolet link, f*_d of the own site for a wall link, f*_i of the
// source site otherwise.  The source site of slot i is s + run_off[run][i] for a
// record whose bulk slots follow its run (L1-resident offsets), else the
// record's pull table entry (which holds the record's own site for a slot that
// a boundary rule fills).  All eighteen loads are issued together, and a warp
// issues them once whatever its sites' link masks; the BFL correction of wall
// links follows as a predicated step.  (4M-site pipe, boundary kernel alone:
// branching per link 0.0599 ms, pull table for every record 0.0554 ms, run
// offsets where they apply 0.0541 ms.)
template <int WALL, bool IO = true>
__device__ __forceinline__ void gather_general(const StepArgs& a, int g, int s, double* f) {
  const GeneralDev& G = a.gen;
  const uint32_t wm = __ldg(G.wall + g), im = IO ? __ldg(G.iolet + g) : 0u;
  int src[18];
  const int run = __ldg(G.run + g);
  if (run >= 0) {
    int off[20];
    load_run_offsets(a, run, off);
#pragma unroll
    for (int i = 1; i < Q; i++) src[i - 1] = s + off[i];
  } else {
#pragma unroll
    for (int i = 1; i < Q; i++) src[i - 1] = __ldg(G.src + (int64_t)(i - 1) * G.G + g);
  }
  f[0] = ld(a.fin + s);
#pragma unroll
  for (int i = 1; i < Q; i++) {
    const int d = inv(i);
    const bool bw = (wm >> (d - 1)) & 1u, bi = (im >> (d - 1)) & 1u;
    const double* p = bi ? a.gin + (int64_t)(d - 1) * G.G + g
                         : a.fin + (bw ? (int64_t)d * a.np + s : (int64_t)i * a.np + src[i - 1]);
    f[i] = ld(p);
  }
  if (WALL == kBFL && wm) {
    // BFL on wall link d with no wall behind (slot i = inv(d)): q >= 1/2 takes
    // (f*_d + (2q-1) f*_i) / (2q); q < 1/2 keeps f*_d and takes the post-step
    // 2q f*_d + (1-2q) f[d] (slot d is never corrected itself, as link i has no
    // wall).  Every cut distance and own-site value is loaded before any
    // arithmetic, so they share one round trip with the gather (4M-site pipe,
    // boundary kernel alone 0.0545 -> 0.0429 ms together with 128 registers).
    float qv[18];
    double fo[18];
#pragma unroll
    for (int i = 1; i < Q; i++) {
      const int d = inv(i);
      const bool corr = ((wm >> (d - 1)) & 1u) && !((wm >> (i - 1)) & 1u);
      qv[i - 1] = corr ? __ldg(G.q + (int64_t)(d - 1) * G.G + g) : 1.0f;
      fo[i - 1] = corr ? ld(a.fin + (int64_t)i * a.np + s) : 0.0;
    }
#pragma unroll
    for (int i = 1; i < Q; i++) {
      const int d = inv(i);
      const bool corr = ((wm >> (d - 1)) & 1u) && !((wm >> (i - 1)) & 1u);
      if (corr) {
        const double q = (double)qv[i - 1];
        if (!(q < 0.5)) f[i] = (f[i] + (2.0 * q - 1) * fo[i - 1]) / (2.0 * q);
        else f[i] = 2.0 * q * f[i] + (1.0 - 2.0 * q) * f[d];
      }
    }
  }
}

// Pre-collision f of any site (GZS neighbours, materialisation).
template <int WALL, bool GATHER>
__device__ __forceinline__ void gather_any(const StepArgs& a, int s, double* f) {
  if (!GATHER) {
#pragma unroll
    for (int i = 0; i < Q; i++) f[i] = ld(a.fin + (int64_t)i * a.np + s);
    return;
  }
  const int r = __ldg(a.meta + s);
  if (r >= 0) gather_bulk(a, s, r, f);
  else gather_general<WALL>(a, -r - 1, s, f);
}

__device__ __forceinline__ void flag_unstable(const StepArgs& a, const double* f) {
  bool bad = false;
#pragma unroll
  for (int i = 0; i < Q; i++) bad |= !(f[i] > 0.0);
  if (bad) atomicOr(a.status, kStatusUnstable);
}

// ---------------------------------------------------------------------------
// Per-site steps
// ---------------------------------------------------------------------------

// One plain bulk site s of run r.
template <int K, bool GATHER, bool MACRO>
__device__ __forceinline__ void bulk_site_f64(const StepArgs& a, int s, int r) {
  double f[Q];
  if (GATHER) gather_bulk(a, s, r, f);
  else {
#pragma unroll
    for (int i = 0; i < Q; i++) f[i] = ld(a.fin + (int64_t)i * a.np + s);
  }
  flag_unstable(a, f);
  double rho, mx, my, mz;
  moments(f, rho, mx, my, mz);
  const FeqConst feq(rho, mx, my, mz);
  double fneq[Q];
#pragma unroll
  for (int i = 0; i < Q; i++) fneq[i] = f[i] - feq(i);
  double om, tau;
  site_rates<K>(a, fneq, s, tau, om);
#pragma unroll
  for (int i = 0; i < Q; i++) a.fout[(int64_t)i * a.np + s] = collide_one<K>(a, f, fneq, om, i);
  if (MACRO) {
    a.rho[s] = rho;
    a.u[s] = mx / rho;
    a.u[a.np + s] = my / rho;
    a.u[2 * a.np + s] = mz / rho;
    a.wss[s] = kNoValue;
    if (a.pi) {
      double fp[Q];
#pragma unroll
      for (int i = 0; i < Q; i++) fp[i] = collide_one<K>(a, f, fneq, om, i);
      store_pi(a, s, tau, fp, f);
    }
  }
}

// One general (boundary or irregular) site record g.
template <int K, int WALL, bool GATHER, bool MACRO, bool IO = true>
__device__ __forceinline__ void general_site_f64(const StepArgs& a, int g) {
  const GeneralDev& G = a.gen;
  const int s = __ldg(G.site + g);
  const uint32_t wm = __ldg(G.wall + g), im = IO ? __ldg(G.iolet + g) : 0u;
  double f[Q];
  if (GATHER) gather_general<WALL, IO>(a, g, s, f);
  else {
#pragma unroll
    for (int i = 0; i < Q; i++) f[i] = ld(a.fin + (int64_t)i * a.np + s);
  }
  flag_unstable(a, f);
  double rho, mx, my, mz;
  moments(f, rho, mx, my, mz);
  const double ux = mx / rho, uy = my / rho, uz = mz / rho;
  const FeqConst feq(rho, mx, my, mz);
  double fneq[Q];
#pragma unroll
  for (int i = 0; i < Q; i++) fneq[i] = f[i] - feq(i);
  double om, tau;
  site_rates<K>(a, fneq, s, tau, om);
  double fp[Q];
#pragma unroll
  for (int i = 0; i < Q; i++) fp[i] = collide_one<K>(a, f, fneq, om, i);
  double out[Q];
#pragma unroll
  for (int i = 0; i < Q; i++) out[i] = fp[i];

  int io = -1;
  if (im) io = __ldg(G.io + g);
  if (im) {
    const IoletDev& I = a.iolets[io];
    const int kind = I.kind;
    double pos[3] = {(double)__ldg(G.xyz + g), (double)__ldg(G.xyz + G.G + g), (double)__ldg(G.xyz + 2 * G.G + g)};
#pragma unroll
    for (int d = 1; d < Q; d++) {
      if (!((im >> (d - 1)) & 1u)) continue;
      if (is_velocity_iolet(kind)) {
        // LaddIoletDelegate::StreamLink (src/lb/streamers/LaddIoletDelegate.h:37-86).
        double w[3];
        if (!link_velocity(a, I, io, g, d, true, pos, w)) {
          atomicOr(a.status, kStatusIoletRadius);
          w[0] = w[1] = w[2] = 0.0;
        }
        w[0] *= rho;
        w[1] *= rho;
        w[2] *= rho;
        const double corr = 2. * weight(d) * (w[0] * cx(d) + w[1] * cy(d) + w[2] * cz(d)) / kCs2;
        a.gout[(int64_t)(d - 1) * G.G + g] = fp[d] - corr;
      } else {
        // NashZerothOrderPressureDelegate::StreamLink (src/lb/streamers/NashZerothOrderPressureDelegate.h:36-76).
        const double rb = a.dens_row[io];
        const double nx = I.nrm_f[0], ny = I.nrm_f[1], nz = I.nrm_f[2];
        const double comp = (mx / rho) * nx + (my / rho) * ny + (mz / rho) * nz;
        const FeqConst gq(rb, nx * comp * rb, ny * comp * rb, nz * comp * rb);
        a.gout[(int64_t)(d - 1) * G.G + g] = gq(inv(d));
      }
    }
  }
  if (WALL == kGZS && wm) {
    // GuoZhengShiDelegate::StreamLink (src/lb/streamers/GuoZhengShiDelegate.h:127-293).
#pragma unroll
    for (int d = 1; d < Q; d++) {
      if (!((wm >> (d - 1)) & 1u)) continue;
      const int i = inv(d);
      const double q = (double)__ldg(G.q + (int64_t)(d - 1) * G.G + g);
      const double fac = 1. - 1. / q;
      double mw0 = mx * fac, mw1 = my * fac, mw2 = mz * fac;
      double fnw_i = fneq[i], fnw_d = fneq[d];
      bool sbb = false;
      if (q < 0.75) {
        if ((im >> (i - 1)) & 1u) {
          const IoletDev& I = a.iolets[io];
          if (!is_velocity_iolet(I.kind)) {
            sbb = true;
          } else {
            const double p3[3] = {(double)__ldg(G.xyz + g), (double)__ldg(G.xyz + G.G + g), (double)__ldg(G.xyz + 2 * G.G + g)};
            double nv[3];
            if (!link_velocity(a, I, io, g, i, false, p3, nv)) {
              atomicOr(a.status, kStatusIoletRadius);
              nv[0] = nv[1] = nv[2] = 0.0;
            }
            mw0 = q * mw0 + (1. - q) * rho * (nv[0] * (q - 1) / (q + 1));
            mw1 = q * mw1 + (1. - q) * rho * (nv[1] * (q - 1) / (q + 1));
            mw2 = q * mw2 + (1. - q) * rho * (nv[2] * (q - 1) / (q + 1));
          }
        } else if ((wm >> (i - 1)) & 1u) {
          sbb = true;
        } else {
          const int grun = __ldg(G.run + g);
          const int nb = grun >= 0 ? s + __ldg(a.run_off + 20 * grun + d) : __ldg(G.src + (int64_t)(d - 1) * G.G + g);
          double fn[Q];
          gather_any<WALL, GATHER>(a, nb, fn);
          double rn, mnx, mny, mnz;
          moments(fn, rn, mnx, mny, mnz);
          const double vn0 = mnx / rn, vn1 = mny / rn, vn2 = mnz / rn;
          const FeqConst fqn(rn, mnx, mny, mnz);
          mw0 = q * mw0 + (1. - q) * rho * (vn0 * (q - 1) / (q + 1));
          mw1 = q * mw1 + (1. - q) * rho * (vn1 * (q - 1) / (q + 1));
          mw2 = q * mw2 + (1. - q) * rho * (vn2 * (q - 1) / (q + 1));
          fnw_i = q * fnw_i + (1. - q) * (fn[i] - fqn(i));
          fnw_d = q * fnw_d + (1. - q) * (fn[d] - fqn(d));
        }
      }
      if (sbb) continue;  // slot i reads f*_d, already in out[d]
      const FeqConst fqw(rho, mw0, mw1, mw2);
      const double fw_i = fqw(i) + fnw_i;
      double v;
      if (K == kTRT) {
        const int lo = i < d ? i : d;
        const double fn_lo = lo == i ? fnw_i : fnw_d, fn_hi = lo == i ? fnw_d : fnw_i;
        const double sym = 0.5 * a.omega * (fn_lo + fn_hi);
        const double asym = 0.5 * a.omega_minus * (fn_lo - fn_hi);
        v = i == lo ? (fw_i + sym + asym) : (fw_i + sym - asym);
      } else {
        v = fw_i + fnw_i * om;
      }
      out[d] = v;
    }
  }
#pragma unroll
  for (int i = 0; i < Q; i++) a.fout[(int64_t)i * a.np + s] = out[i];

  const int cpl = im ? __ldg(G.cpl + g) : -1;
  if (cpl >= 0) {
    const IoletDev& I = a.iolets[io];
    a.cpl_buf[cpl] = ux * (-I.nrm[0]) + uy * (-I.nrm[1]) + uz * (-I.nrm[2]);
  }
  if (MACRO) {
    a.rho[s] = rho;
    a.u[s] = ux;
    a.u[a.np + s] = uy;
    a.u[2 * a.np + s] = uz;
    if (wm) {
      const double nor[3] = {(double)__ldg(G.nrm + g), (double)__ldg(G.nrm + G.G + g), (double)__ldg(G.nrm + 2 * G.G + g)};
      a.wss[s] = wss_mag(tau, fp, f, nor);
    } else {
      a.wss[s] = kNoValue;
    }
    if (a.pi) store_pi(a, s, tau, fp, f);
  }
}

}  // namespace
}  // namespace hb
