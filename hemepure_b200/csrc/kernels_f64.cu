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

// Post-collision value of direction i for kernel K (LBGK.h:64-72, TRT.h:80-109).
template <int K>
__device__ __forceinline__ double collide_one(const StepArgs& a, const double* f, const double* fneq, double omega_site, int i) {
  if (K == kTRT) {
    if (i == 0) return f[0] + (0.5 * a.omega * (fneq[0] + fneq[0])) - (0.5 * a.omega_minus * (fneq[0] - fneq[0]));
    const int j = inv(i);
    const int lo = i < j ? i : j, hi = i < j ? j : i;
    const double sym = 0.5 * a.omega * (fneq[lo] + fneq[hi]);
    const double asym = 0.5 * a.omega_minus * (fneq[lo] - fneq[hi]);
    return i == lo ? (f[i] + sym + asym) : (f[i] + sym - asym);
  }
  return f[i] + fneq[i] * omega_site;
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

template <int WALL>
__device__ __forceinline__ void gather_general(const StepArgs& a, int g, int s, double* f) {
  const GeneralDev& G = a.gen;
  const uint32_t wm = __ldg(G.wall + g), im = __ldg(G.iolet + g);
  const int run = __ldg(G.run + g);
  int off[20];
  if (run >= 0) load_run_offsets(a, run, off);
  f[0] = ld(a.fin + s);
#pragma unroll
  for (int i = 1; i < Q; i++) {
    const int d = inv(i);
    const bool bw = (wm >> (d - 1)) & 1u, bi = (im >> (d - 1)) & 1u;
    if (bi) {
      f[i] = ld(a.gin + (int64_t)(d - 1) * G.G + g);
    } else if (bw) {
      if (WALL == kBFL) {
        const double q = (double)__ldg(G.q + (int64_t)(d - 1) * G.G + g);
        const bool wi = (wm >> (i - 1)) & 1u;
        const double fd = ld(a.fin + (int64_t)d * a.np + s);
        if (wi || q < 0.5) f[i] = fd;
        else f[i] = (fd + (2.0 * q - 1) * ld(a.fin + (int64_t)i * a.np + s)) / (2.0 * q);
      } else {
        f[i] = ld(a.fin + (int64_t)d * a.np + s);
      }
    } else {
      const int src = run >= 0 ? s + off[i] : __ldg(G.src + (int64_t)(i - 1) * G.G + g);
      f[i] = ld(a.fin + (int64_t)i * a.np + src);
    }
  }
  if (WALL == kBFL && wm) {
#pragma unroll
    for (int d = 1; d < Q; d++) {
      const int i = inv(d);
      if (((wm >> (d - 1)) & 1u) && !((wm >> (i - 1)) & 1u)) {
        const double q = (double)__ldg(G.q + (int64_t)(d - 1) * G.G + g);
        if (q < 0.5) f[i] = 2.0 * q * f[i] + (1.0 - 2.0 * q) * f[d];
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
// Kernels
// ---------------------------------------------------------------------------

template <int K, bool GATHER, bool MACRO>
__global__ void __launch_bounds__(256) k_bulk(const StepArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  const int r = __ldg(a.meta + s);
  if (r < 0) return;
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
  double om = a.omega, tau = a.tau;
  if (K == kLES) {
    tau = les_tau(a, fneq, __ldg(a.vtau + s));
    om = -1.0 / tau;
  }
#pragma unroll
  for (int i = 0; i < Q; i++) a.fout[(int64_t)i * a.np + s] = collide_one<K>(a, f, fneq, om, i);
  if (MACRO) {
    a.rho[s] = rho;
    a.u[s] = mx / rho;
    a.u[a.np + s] = my / rho;
    a.u[2 * a.np + s] = mz / rho;
    a.wss[s] = kNoValue;
  }
}

template <int K, int WALL, bool GATHER, bool MACRO>
__global__ void __launch_bounds__(128) k_general(const StepArgs a) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const GeneralDev& G = a.gen;
  if (g >= G.G) return;
  const int s = __ldg(G.site + g);
  const uint32_t wm = __ldg(G.wall + g), im = __ldg(G.iolet + g);
  double f[Q];
  if (GATHER) gather_general<WALL>(a, g, s, f);
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
  double om = a.omega, tau = a.tau;
  if (K == kLES) {
    tau = les_tau(a, fneq, __ldg(a.vtau + s));
    om = -1.0 / tau;
  }
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
      if (kind == kParabolic) {
        // LaddIoletDelegate::StreamLink (src/lb/streamers/LaddIoletDelegate.h:37-86).
        double hw[3] = {pos[0], pos[1], pos[2]};
        hw[0] += 0.5 * cx(d);
        hw[1] += 0.5 * cy(d);
        hw[2] += 0.5 * cz(d);
        double w[3];
        if (!parabolic(I, hw, (uint64_t)(unsigned int)a.t, w)) {
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
          if (I.kind != kParabolic) {
            sbb = true;
          } else {
            double np3[3] = {(double)__ldg(G.xyz + g) + cx(i), (double)__ldg(G.xyz + G.G + g) + cy(i),
                             (double)__ldg(G.xyz + 2 * G.G + g) + cz(i)};
            double nv[3];
            if (!parabolic(I, np3, (uint64_t)(unsigned int)a.t, nv)) {
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
  }
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
      const double Rc = W.rc, Rp = W.rp, Cp = W.cp;
      const double pn = (Rp * Cp * pressure + (Rc + Rp) * (2.0 * flow - W.flow_old) + Rc * Rp * Cp * (flow - W.flow_old)) / (1.0 + Rp * Cp);
      W.density_new = pn / kCs2;
      d_after = W.density_new;
      flow_old = flow;
    }
    W.density = d_after;
    W.flow = flow;
    W.flow_old = flow_old;
    W.count_prev = W.cpl_count;
  }
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
  if ((which & 2) && a.gen.G > 0) k_general<K, WALL, GATHER, MACRO><<<(a.gen.G + gb - 1) / gb, gb, 0, st>>>(a);
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
  else launch1<kLES>(a, wall, gather, macro, which, bulk_block, general_block, st);
}

void launch_gather_f64(const StepArgs& a, int wall, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  const int b = 256;
  if (a.n <= 0) return;
  if (wall == kBFL) k_gather<kBFL><<<(a.n + b - 1) / b, b, 0, st>>>(a);
  else if (wall == kGZS) k_gather<kGZS><<<(a.n + b - 1) / b, b, 0, st>>>(a);
  else k_gather<kSBB><<<(a.n + b - 1) / b, b, 0, st>>>(a);
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
