// solver.cpp -- device state and the time-step loop of one lattice.
//
// One step (src/lb/lb.hpp:191-346 and src/SimulationMaster.cc:346-383):
//   RequestComms   Windkessel DoComms on the device (k_wk3_begin), cosine
//                  densities from the host table (InOutLetCosine::GetDensity with
//                  the 0-indexed step, BoundaryValues.cc:211-214)
//   PreReceive     k_bulk over plain bulk sites, k_general over the rest
//   PostReceive    nothing: the BFL post-step is applied when the next step
//                  gathers (kernels_f64.cu)
//   EndIteration   swap the two buffers, time step + 1
#include "solver.h"
#include "shard.h"
#include "extraction.h"

#include <algorithm>
#include <cstdio>
#include <cmath>
#include <cstring>

namespace hb {

DeviceBuffer::~DeviceBuffer() {
  if (p) cudaFree(p);
}

void DeviceBuffer::alloc(size_t b) {
  if (p) {
    cudaFree(p);
    p = nullptr;
  }
  bytes = b;
  if (b == 0) return;
  cudaError_t e = cudaMalloc(&p, b);
  if (e != cudaSuccess) {
    p = nullptr;
    throw Error{e == cudaErrorMemoryAllocation ? HB_ERR_OOM : HB_ERR_CUDA,
                std::string("cudaMalloc(") + std::to_string(b) + "): " + cudaGetErrorString(e)};
  }
}

void Solver::check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error{HB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

namespace {

// Lattice::CalculateFeq at zero momentum (the equilibrium initial condition,
// src/lb/InitialCondition.hpp:29-40).
void feq_host(double rho, double mx, double my, double mz, double* feq) {
  const double th = (3. / 2.) * (mx * mx + my * my + mz * mz);
  const double d1 = 1. / rho;
  const double nh = (9. / 2.) * d1;
  for (int i = 0; i < Q; i++) {
    const double mde = (double)cx(i) * mx + (double)cy(i) * my + (double)cz(i) * mz;
    const double t1 = rho - th * d1;
    feq[i] = weight(i) * ((t1 + nh * (mde * mde)) + 3. * mde);
  }
}

template <class T>
void upload_vec(DeviceBuffer& b, const std::vector<T>& v, int64_t& total) {
  b.alloc(v.size() * sizeof(T));
  if (!v.empty()) {
    cudaError_t e = cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) throw Error{HB_ERR_CUDA, std::string("cudaMemcpy: ") + cudaGetErrorString(e)};
  }
  total += (int64_t)b.bytes;
}

}  // namespace

void validate_case(const hb_params& p, const hb_options& o) {
  if (o.kernel < 0 || o.kernel > kTRTSL || o.wall < 0 || o.wall > 2) throw Error{HB_ERR_ARG, "unknown kernel or wall type"};
  if (o.precision < HB_STORE_FP64 || o.precision > HB_STORE_FP16) throw Error{HB_ERR_ARG, "unknown storage precision"};
  if (is_sponge(o.kernel) && o.wall == kGZS)
    throw Error{HB_ERR_UNSUPPORTED, "GZS walls with a sponge-layer kernel: the virtual-node collision has no relaxation time"};
  if ((o.kernel == kLBGKSL || o.kernel == kTRTSL) && o.precision != HB_STORE_FP64)
    throw Error{HB_ERR_UNSUPPORTED, "the LBGKSL and TRTSL kernels run with FP64 storage"};
  if (!(p.tau > 0.5)) throw Error{HB_ERR_ARG, "tau must exceed 1/2"};
  for (int k = 0; k < p.n_inlets + p.n_outlets; k++) {
    const hb_iolet& io = k < p.n_inlets ? p.inlets[k] : p.outlets[k - p.n_inlets];
    if (io.kind < 0 || io.kind > kWomersley) throw Error{HB_ERR_ARG, "unknown iolet kind"};
    if ((io.kind == kFile || io.kind == kFileVelocity) && (!io.table || io.table_steps == 0))
      throw Error{HB_ERR_ARG, "a file iolet needs its table"};
    if (io.kind == kWomersley && !(io.period > 0.0 && io.radius > 0.0))
      throw Error{HB_ERR_ARG, "a Womersley iolet needs a positive period and radius"};
  }
}

Solver::Solver(LatticeTables tables, const hb_params& params, const hb_options& opt, Layout* layout)
    : t_(std::move(tables)), p_(params), opt_(opt) {
  validate_case(p_, opt_);
  // The file iolets' tables are the caller's only for the call: keep copies.
  for (int idx = 0; idx < 32; idx++) {
    const int cnt = idx < 16 ? p_.n_inlets : p_.n_outlets;
    if (idx % 16 >= cnt) continue;
    hb_iolet& io = idx < 16 ? p_.inlets[idx] : p_.outlets[idx - 16];
    if (io.kind != kFile && io.kind != kFileVelocity) continue;
    tables_[idx].assign(io.table, io.table + io.table_steps);
    io.table = tables_[idx].data();
  }
  if ((opt_.wall == kBFL || opt_.wall == kGZS) && t_.q.empty()) throw Error{HB_ERR_ARG, "BFL and GZS walls need wall distances"};
  check(cudaSetDevice(opt_.device), "cudaSetDevice");
  if (layout) L_ = std::move(*layout);
  else L_ = build_layout(t_, p_, opt_.wall);
  t_step_ = p_.initial_step ? p_.initial_step : 1;
  omega_ = -1.0 / p_.tau;
  {
    const double lambda = p_.relaxation_parameter;
    const double tau_minus = 0.5 + lambda / (p_.tau - 0.5);
    omega_minus_ = -1.0 / tau_minus;
  }
  check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  // The latency-bound boundary kernel runs on the side stream at the highest
  // priority, so its blocks are dispatched ahead of the bulk kernel's queued ones
  // (4M-site pipe: FP32 step 29.3k -> 30.3k MLUPS; FP64 unchanged).
  int prio_lo = 0, prio_hi = 0;
  check(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi), "cudaDeviceGetStreamPriorityRange");
  check(cudaStreamCreateWithPriority(&side_, cudaStreamNonBlocking, prio_hi), "cudaStreamCreate");
  check(cudaStreamCreateWithPriority(&side2_, cudaStreamNonBlocking, prio_hi), "cudaStreamCreate");
  check(cudaEventCreate(&ev0_), "cudaEventCreate");
  check(cudaEventCreate(&ev1_), "cudaEventCreate");
  check(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "cudaEventCreate");
  check(cudaEventCreateWithFlags(&join_, cudaEventDisableTiming), "cudaEventCreate");
  check(cudaEventCreateWithFlags(&join2_, cudaEventDisableTiming), "cudaEventCreate");
  upload();
}

Solver::~Solver() {
  if (stream_) cudaStreamSynchronize(stream_);
  if (xev_) cudaEventDestroy(xev_);
  if (side_) cudaStreamSynchronize(side_);
  if (side2_) cudaStreamSynchronize(side2_);
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  if (fork_) cudaEventDestroy(fork_);
  if (join_) cudaEventDestroy(join_);
  if (join2_) cudaEventDestroy(join2_);
  if (side_) cudaStreamDestroy(side_);
  if (side2_) cudaStreamDestroy(side2_);
  if (stream_) cudaStreamDestroy(stream_);
  if (status_host_) cudaFreeHost(status_host_);
  if (host_rows_) cudaFreeHost(host_rows_);
  if (rows_ev_) cudaEventDestroy(rows_ev_);
}

void Solver::upload() {
  const int n = L_.n;
  const int64_t np = L_.np;
  int64_t tot = 0;
  for (int b = 0; b < 2; b++) {
    f_[b].alloc((size_t)Q * np * elem_bytes());
    tot += (int64_t)f_[b].bytes;
    check(cudaMemset(f_[b].p, 0, f_[b].bytes), "cudaMemset");
  }
  for (int b = 0; b < 2; b++) {
    ghost_[b].alloc((size_t)18 * std::max(1, L_.G) * (mixed() ? sizeof(float) : sizeof(double)));
    tot += (int64_t)ghost_[b].bytes;
    check(cudaMemset(ghost_[b].p, 0, ghost_[b].bytes), "cudaMemset");
  }
  upload_vec(meta_, L_.meta, tot);
  upload_vec(run_off_, L_.run_off, tot);
  if (opt_.precision != HB_STORE_FP64 && (int64_t)Q * np < ((int64_t)1 << 31)) {
    // Plane offsets for the shifted forms' bulk gather: one address add per load.
    std::vector<int> po(L_.run_off.size(), 0);
    for (size_t r = 0; r < po.size() / 20; r++)
      for (int i = 0; i < Q; i++) po[r * 20 + i] = (int)((int64_t)i * np + L_.run_off[r * 20 + i]);
    upload_vec(run_po_, po, tot);
  }
  upload_vec(st2ref_, L_.st2ref, tot);
  upload_vec(g_site_, L_.g_site, tot);
  upload_vec(g_run_, L_.g_run, tot);
  upload_vec(g_wall_, L_.g_wall, tot);
  upload_vec(g_iolet_, L_.g_iolet, tot);
  upload_vec(g_src_, L_.g_src, tot);
  upload_vec(g_q_, L_.g_q, tot);
  upload_vec(g_nrm_, L_.g_nrm, tot);
  upload_vec(g_io_, L_.g_io, tot);
  upload_vec(g_cpl_, L_.g_cpl, tot);
  upload_vec(g_xyz_, L_.g_xyz, tot);
  // Womersley links: the time-independent factor of the profile at the two points
  // a link's velocity is taken at (the Ladd half-way point, and the neighbour the
  // GZS wall rule extrapolates from), computed once on the host.
  {
    std::vector<int> wom(L_.G, -1);
    std::vector<double> amp;
    for (int g = 0; g < L_.G; g++) {
      const uint32_t im = L_.g_iolet[g];
      if (!im) continue;
      const int idx = L_.g_io[g];
      const hb_iolet& c = idx < 16 ? p_.inlets[idx] : p_.outlets[idx - 16];
      if (c.kind != kWomersley) continue;
      wom[g] = (int)(amp.size() / (18 * 4));
      amp.resize(amp.size() + 18 * 4, 0.0);
      double* row = amp.data() + amp.size() - 18 * 4;
      const double x0 = L_.g_xyz[g], y0 = L_.g_xyz[(size_t)L_.G + g], z0 = L_.g_xyz[2 * (size_t)L_.G + g];
      for (int d = 1; d < Q; d++) {
        if (!((im >> (d - 1)) & 1u)) continue;
        double hw[3] = {x0, y0, z0};
        hw[0] += 0.5 * cx(d);
        hw[1] += 0.5 * cy(d);
        hw[2] += 0.5 * cz(d);
        const double nb[3] = {x0 + cx(d), y0 + cy(d), z0 + cz(d)};
        const std::complex<double> ah = womersley_amplitude(c, hw), an = womersley_amplitude(c, nb);
        row[(d - 1) * 4 + 0] = ah.real();
        row[(d - 1) * 4 + 1] = ah.imag();
        row[(d - 1) * 4 + 2] = an.real();
        row[(d - 1) * 4 + 3] = an.imag();
      }
    }
    if (!amp.empty()) {
      upload_vec(g_wom_, wom, tot);
      upload_vec(wom_amp_, amp, tot);
    }
  }

  // LES sponge relaxation time per site (LBGKLESSpongeLayer::InitState,
  // src/lb/kernels/LBGKLESSpongeLayer.h:87-116), in storage order.  The
  // reference subtracts the outlet position from the site's integer coordinates
  // with Vector3D<site_t>::operator-, which converts the position to integers
  // first by truncation (src/util/Vector3D.h:238-243,396), so the squared
  // distance is an integer.
  if (is_sponge(opt_.kernel)) {
    std::vector<double> vt(n);
    const double width = p_.sponge_width, widthsq = width * width;
    for (int s = 0; s < n; s++) {
      const int x = L_.st2ref[s];
      double vr = 1.0;
      for (int k = 0; k < p_.n_outlets; k++) {
        const int64_t dx = (int64_t)t_.coords[3 * x] - (int64_t)p_.outlets[k].position[0];
        const int64_t dy = (int64_t)t_.coords[3 * x + 1] - (int64_t)p_.outlets[k].position[1];
        const int64_t dz = (int64_t)t_.coords[3 * x + 2] - (int64_t)p_.outlets[k].position[2];
        const double distsq = (double)(dx * dx + dy * dy + dz * dz);
        const double dist = std::sqrt(distsq);
        if (distsq <= widthsq) vr *= 1.0 + (p_.viscosity_ratio - 1.0) * (dist / width - 1.0) * (dist / width - 1.0);
      }
      vt[s] = vr * (p_.tau - 0.5) + 0.5;
    }
    upload_vec(vtau_, vt, tot);
  }

  // Iolet table.
  std::vector<IoletDev> io(32);
  std::memset(io.data(), 0, io.size() * sizeof(IoletDev));
  for (int idx = 0; idx < 32; idx++) {
    const int cnt = idx < 16 ? p_.n_inlets : p_.n_outlets;
    if (idx % 16 >= cnt) continue;
    const hb_iolet& c = idx < 16 ? p_.inlets[idx] : p_.outlets[idx - 16];
    IoletDev& d = io[idx];
    d.kind = c.kind;
    d.dir0 = L_.dir0[idx];
    d.wk3 = -1;
    for (int k = 0; k < 3; k++) {
      d.pos[k] = c.position[k];
      d.nrm[k] = c.normal[k];
      d.nrm_f[k] = (double)(float)c.normal[k];
    }
    d.radius = c.radius;
    d.max_speed = c.max_speed;
    d.warmup = c.warmup;
  }
  std::vector<WK3Dev> wk(L_.couplings.size());
  for (size_t k = 0; k < L_.couplings.size(); k++) {
    const auto& c = L_.couplings[k];
    const hb_iolet& cfg = c.iolet < 16 ? p_.inlets[c.iolet] : p_.outlets[c.iolet - 16];
    WK3Dev& w = wk[k];
    std::memset(&w, 0, sizeof(w));
    w.density = w.density_new = 1.0;
    w.flow = w.flow_old = 0.0;
    w.kind = cfg.kind;
    w.rc = cfg.rc;
    w.rp = cfg.rp;
    w.cp = cfg.cp;
    w.area = cfg.area;
    w.cpl_start = c.start;
    w.cpl_count = c.count;
    w.count_prev = 0;
    w.centre_couples = c.centre_couples ? 1 : 0;
    w.iolet = c.iolet;
    io[c.iolet].wk3 = (int)k;
  }
  nwk3_ = (int)wk.size();
  upload_vec(iolets_, io, tot);
  upload_vec(wk3_, wk, tot);
  std::vector<double> zeros(std::max(1, L_.cpl_total), 0.0);
  upload_vec(cpl_buf_, zeros, tot);
  dens_rows_ = 1024;
  dens_.alloc((size_t)dens_rows_ * kRowStride * sizeof(double));
  tot += (int64_t)dens_.bytes;
  check(cudaHostAlloc((void**)&host_rows_, (size_t)dens_rows_ * kRowStride * sizeof(double), cudaHostAllocDefault),
        "cudaHostAlloc");
  for (size_t k = 0; k < (size_t)dens_rows_ * kRowStride; k++) host_rows_[k] = 1.0;
  check(cudaEventCreateWithFlags(&rows_ev_, cudaEventDisableTiming), "cudaEventCreate");
  status_.alloc(sizeof(int));
  // The status word comes back after every hb_step call: a pinned host word makes
  // that read a direct copy instead of a staged one.
  check(cudaHostAlloc((void**)&status_host_, sizeof(int), cudaHostAllocDefault), "cudaHostAlloc");
  *status_host_ = 0;
  check(cudaMemset(status_.p, 0, sizeof(int)), "cudaMemset");
  dev_bytes_ = tot;

  // Equilibrium initial condition in direct form.
  double feq[Q];
  feq_host(p_.initial_density, 0.0, 0.0, 0.0, feq);
  if (!mixed()) {
    launch_equilibrium_f64(f_[0].as<double>(), np, n, feq, stream_);
  } else {
    // The equilibrium filled in FP64 AoS on the device, then shifted and narrowed.
    DeviceBuffer aos;
    aos.alloc((size_t)n * Q * sizeof(double));
    launch_equilibrium_aos_f64(aos.as<double>(), n, feq, stream_);
    launch_from_aos_mixed(aos.as<double>(), st2ref_.as<int>(), n, np, opt_.precision, f_[0].p, stream_);
    check(cudaStreamSynchronize(stream_), "initialisation");
  }
  check(cudaGetLastError(), "equilibrium fill");
  cur_ = 0;
  direct_ = true;
  check(cudaStreamSynchronize(stream_), "initialisation");
}

void Solver::ensure_macro() {
  if (rho_.p) return;
  rho_.alloc((size_t)L_.np * sizeof(double));
  u_.alloc((size_t)3 * L_.np * sizeof(double));
  wss_.alloc((size_t)L_.np * sizeof(double));
  dev_bytes_ += (int64_t)(rho_.bytes + u_.bytes + wss_.bytes);
}

StepArgs Solver::args() const {
  StepArgs a;
  std::memset(&a, 0, sizeof(a));
  a.fin = f_[cur_].as<double>();
  a.fout = f_[1 - cur_].as<double>();
  a.gin = ghost_[cur_].as<double>();
  a.gout = ghost_[1 - cur_].as<double>();
  a.np = L_.np;
  a.n = L_.n;
  a.meta = meta_.as<int>();
  a.run_off = run_off_.as<int>();
  a.run_po = run_po_.p ? run_po_.as<int>() : nullptr;
  a.gen.G = L_.G;
  a.gen.G_noiolet = L_.kind_start[2];
  a.gen.site = g_site_.as<int>();
  a.gen.run = g_run_.as<int>();
  a.gen.wall = g_wall_.as<uint32_t>();
  a.gen.iolet = g_iolet_.as<uint32_t>();
  a.gen.src = g_src_.as<int>();
  a.gen.q = g_q_.as<float>();
  a.gen.nrm = g_nrm_.as<float>();
  a.gen.io = g_io_.as<int>();
  a.gen.cpl = g_cpl_.as<int>();
  a.gen.xyz = g_xyz_.as<int>();
  a.gen.wom = g_wom_.as<int>();
  a.wom_amp = wom_amp_.as<double>();
  a.tau = p_.tau;
  a.omega = omega_;
  a.omega_minus = omega_minus_;
  a.lambda = p_.relaxation_parameter;
  a.vtau = vtau_.as<double>();
  a.t = t_step_;
  a.lifetime = p_.sponge_lifetime;
  a.iolets = iolets_.as<IoletDev>();
  a.dens_row = dens_.as<double>() + (size_t)row_ * kRowStride;
  a.cpl_buf = cpl_buf_.as<double>();
  a.rho = rho_.as<double>();
  a.u = u_.as<double>();
  a.wss = wss_.as<double>();
  a.status = status_.as<int>();
  return a;
}

// Host-side iolet rows for `count` steps from t_first (1-based): the cosine and
// file iolets' GetDensity(t - 1), the file-velocity iolets' peak speed at t and
// the Womersley iolets' exp(i omega t).  Windkessel entries are written on the device.
void Solver::fill_density_rows(uint64_t t_first, int count) {
  if (rows_pending_) check(cudaEventSynchronize(rows_ev_), "iolet row upload");
  rows_pending_ = false;
  double mind = 1.7976931348623157e308;
  for (int k = 0; k < p_.n_inlets + p_.n_outlets; k++) {
    const hb_iolet& c = k < p_.n_inlets ? p_.inlets[k] : p_.outlets[k - p_.n_inlets];
    // InOutLet::GetDensityMin: cosine mean - amplitude, file its table's minimum, others 1.
    const double dmin = c.kind == kCosine ? c.density_mean - c.density_amp : c.kind == kFile ? c.density_min : 1.0;
    if (dmin < mind) mind = dmin;
  }
  for (int r = 0; r < count; r++) {
    const uint64_t t0 = t_first + (uint64_t)r - 1;
    for (int idx = 0; idx < 32; idx++) {
      const int cnt = idx < 16 ? p_.n_inlets : p_.n_outlets;
      double v = 1.0;
      if (idx % 16 < cnt) {
        const hb_iolet& c = idx < 16 ? p_.inlets[idx] : p_.outlets[idx - 16];
        if (c.kind == kCosine) {
          const double w = 2.0 * kPi / c.period;
          const double target = c.density_mean + c.density_amp * std::cos(w * (double)t0 + c.phase);
          if (t0 >= c.warmup) v = target;
          else {
            const double fac = ((double)t0) / ((double)c.warmup);
            v = fac * target + (1. - fac) * mind;
          }
        }
      }
      double va = 0.0, vb = 0.0;
      if (idx % 16 < cnt) {
        const hb_iolet& c = idx < 16 ? p_.inlets[idx] : p_.outlets[idx - 16];
        if (c.kind == kFile) v = c.table[t0 < c.table_steps ? t0 : c.table_steps - 1];
        if (dens_override_ && (c.kind == kCosine || c.kind == kFile)) v = dens_override_v_[idx];
        // Velocity iolets see BoundaryValues::GetTimeStep, the 1-based step as unsigned int.
        const uint64_t t1 = (uint64_t)(unsigned int)(t0 + 1);
        if (c.kind == kFileVelocity) va = c.table[t1 < c.table_steps ? t1 : c.table_steps - 1];
        if (c.kind == kWomersley) {
          const std::complex<double> e = womersley_phase(c, t1);
          va = e.real();
          vb = e.imag();
        }
      }
      double* row = host_rows_ + (size_t)r * kRowStride;
      row[idx] = v;
      row[kRowA + idx] = va;
      row[kRowB + idx] = vb;
    }
  }
  check(cudaMemcpyAsync(dens_.p, host_rows_, (size_t)count * kRowStride * sizeof(double), cudaMemcpyHostToDevice,
                        stream_),
        "iolet row upload");
  check(cudaEventRecord(rows_ev_, stream_), "event");
  rows_pending_ = true;
}

// The rows depend on the step alone (the Windkessel kernel rewrites its own
// entries of a row at that row's step), so the rows a call needs are uploaded
// together when it starts: up to 1024 rows for an hb_step call of many steps,
// one row (768 bytes) for a call that advances one step.
int Solver::density_row(uint64_t t, int64_t steps_ahead) {
  if (!rows_valid_ || t < rows_first_ || t >= rows_first_ + (uint64_t)rows_count_) {
    const int count = (int)std::max<int64_t>(1, std::min<int64_t>(steps_ahead, dens_rows_));
    fill_density_rows(t, count);
    rows_first_ = t;
    rows_count_ = count;
    rows_valid_ = true;
  }
  return (int)(t - rows_first_);
}

void Solver::set_iolet_densities(const double* inlets, int n_inlets, const double* outlets, int n_outlets) {
  rows_valid_ = false;
  if (!inlets && !outlets) {
    dens_override_ = false;
    return;
  }
  if (!inlets || !outlets || n_inlets != p_.n_inlets || n_outlets != p_.n_outlets)
    throw Error{HB_ERR_ARG, "iolet density override needs one value per inlet and per outlet of the case"};
  for (int k = 0; k < n_inlets; k++) dens_override_v_[k] = inlets[k];
  for (int k = 0; k < n_outlets; k++) dens_override_v_[16 + k] = outlets[k];
  dens_override_ = true;
}

void Solver::request_comms() {
  if (!phase_open_) row_ = density_row(t_step_, 1);
  launch_wk3_begin(wk3_.as<WK3Dev>(), nwk3_, cpl_buf_.as<double>(), dens_.as<double>() + (size_t)row_ * kRowStride, stream_);
  phase_open_ = true;
}

void Solver::pre_receive(bool macro, int which, bool stress) {
  if (!phase_open_) request_comms();
  if (macro) ensure_macro();
  stress = stress && macro;
  if (stress && !pi_.p) {
    pi_.alloc((size_t)7 * L_.np * sizeof(double));
    dev_bytes_ += (int64_t)pi_.bytes;
  }
  StepArgs a = args();
  a.pi = stress ? pi_.as<double>() : nullptr;
  // Boundary records with iolet links run in their own kernel on a second side
  // stream, beside those without (independent records, disjoint slots).  4M
  // pipe, whole step: FP64 0.2140 -> 0.2136 ms, FP32 0.1208 -> 0.1190 ms, FP16
  // 0.0963 -> 0.0903 ms.  Their few blocks are launched first, so they are not
  // queued behind the wall records' four waves (boundary work alone: FP64
  // 0.0430 -> 0.0390 ms, FP16 0.0383 -> 0.0317 ms).
  const bool split = L_.kind_start[2] > 0 && L_.kind_start[2] < L_.G;
  if ((which & kLaunchBoundary) && L_.G > 0) {
    // The boundary kernels are latency-bound and the bulk kernel bandwidth-bound:
    // run them side by side, all after the Windkessel update.
    check(cudaEventRecord(fork_, stream_), "fork");
    if (split) {
      check(cudaStreamWaitEvent(side2_, fork_, 0), "fork");
      launch(a, macro, kLaunchIoletRecords, side2_);
      check(cudaEventRecord(join2_, side2_), "join");
    }
    check(cudaStreamWaitEvent(side_, fork_, 0), "fork");
    launch(a, macro, split ? kLaunchWallRecords : kLaunchBoundary, side_);
    check(cudaEventRecord(join_, side_), "join");
    if (which & kLaunchBulk) launch(a, macro, kLaunchBulk, stream_);
    check(cudaStreamWaitEvent(stream_, join_, 0), "join");
    if (split) check(cudaStreamWaitEvent(stream_, join2_, 0), "join");
  } else {
    launch(a, macro, which, stream_);
  }
  check(cudaGetLastError(), "step kernel launch");
  phase_macro_ = macro;
  phase_stress_ = stress;
}

void Solver::launch(const StepArgs& a, bool macro, int which, cudaStream_t st) {
  if (!mixed()) {
    launch_step_f64(a, opt_.kernel, opt_.wall, !direct_, macro, which, 256, 128, st);
  } else {
    launch_step_mixed(a, opt_.precision, f_[cur_].p, f_[1 - cur_].p, ghost_[cur_].as<float>(), ghost_[1 - cur_].as<float>(),
                      opt_.kernel, opt_.wall, !direct_, macro, which, st);
  }
}

// Pre-collision f in FP64 AoS reference order: the current state (use_prev false)
// or the state that entered the last completed step (use_prev true).
void Solver::to_aos(bool use_prev, double* dev_aos) {
  StepArgs a = args();
  const int b = use_prev ? 1 - cur_ : cur_;
  const bool gather = use_prev ? !prev_direct_ : !direct_;
  launch_to_aos_mixed(a, opt_.precision, f_[b].p, ghost_[b].as<float>(), opt_.wall, gather, st2ref_.as<int>(),
                      dev_aos, stream_);
  check(cudaGetLastError(), "to_aos launch");
}

void Solver::end_iteration() {
  prev_direct_ = direct_;
  prev_valid_ = true;
  cur_ = 1 - cur_;
  direct_ = false;
  t_step_++;
  phase_open_ = false;
  macro_valid_ = phase_macro_;
  phase_macro_ = false;
  stress_valid_ = phase_stress_;
  phase_stress_ = false;
}

int Solver::read_status() {
  check(cudaMemcpyAsync(status_host_, status_.p, sizeof(int), cudaMemcpyDeviceToHost, stream_), "status read");
  check(cudaStreamSynchronize(stream_), "step");
  const int st = *status_host_;
  if (st) {
    status_sticky_ |= st;
    check(cudaMemsetAsync(status_.p, 0, sizeof(int), stream_), "status reset");
  }
  return st;
}

int Solver::step(int64_t nsteps, uint32_t flags) {
  if (nsteps < 0) throw Error{HB_ERR_ARG, "negative step count"};
  if (shard_ && nsteps > 1)
    throw Error{HB_ERR_ARG, "a shard advances one step per call: its halo is exchanged between steps"};
  int64_t launches = 0;
  // The boundary records without and with iolet links are two kernels.
  const int boundary_launches =
      L_.G == 0 ? 0 : (L_.kind_start[2] > 0 ? 1 : 0) + (L_.G > L_.kind_start[2] ? 1 : 0);
  const int per_step = (nwk3_ ? 1 : 0) + (L_.n > 0 ? 1 : 0) + boundary_launches;
  check(cudaEventRecord(ev0_, stream_), "event");
  for (int64_t j = 0; j < nsteps; j++) {
    row_ = density_row(t_step_, nsteps - j);
    phase_open_ = true;
    launch_wk3_begin(wk3_.as<WK3Dev>(), nwk3_, cpl_buf_.as<double>(), dens_.as<double>() + (size_t)row_ * kRowStride, stream_);
    const bool macro = (flags & HB_STEP_MACRO) && (j == nsteps - 1);
    pre_receive(macro, 3, (flags & HB_STEP_STRESS) != 0);
    end_iteration();
    launches += per_step;
  }
  check(cudaEventRecord(ev1_, stream_), "event");
  const int st = read_status();
  float ms = 0;
  check(cudaEventElapsedTime(&ms, ev0_, ev1_), "event timing");
  last_ms_ = ms;
  last_launches_ = launches;
  if (st & kStatusIoletRadius) return HB_ERR_IOLET_RADIUS;
  if (st & kStatusUnstable) return HB_UNSTABLE;
  return HB_OK;
}

int Solver::profile(int64_t nsteps, double ms[3]) {
  ms[0] = ms[1] = ms[2] = 0.0;
  cudaEvent_t e[3];
  for (auto& x : e) check(cudaEventCreate(&x), "cudaEventCreate");
  int rc = HB_OK;
  // Pass 0: the launches hb_step issues; pass 1: the bulk and boundary kernels
  // one after the other.
  for (int pass = 0; pass < 2; pass++) {
    for (int64_t j = 0; j < nsteps; j++) {
      {
        row_ = density_row(t_step_, nsteps - j);
        phase_open_ = true;
        launch_wk3_begin(wk3_.as<WK3Dev>(), nwk3_, cpl_buf_.as<double>(), dens_.as<double>() + (size_t)row_ * kRowStride, stream_);
        check(cudaEventRecord(e[0], stream_), "event");
        if (pass == 0) {
          pre_receive(false, 3);
          check(cudaEventRecord(e[1], stream_), "event");
        } else {
          pre_receive(false, 1);
          check(cudaEventRecord(e[1], stream_), "event");
          pre_receive(false, 2);
        }
        check(cudaEventRecord(e[2], stream_), "event");
        end_iteration();
        check(cudaEventSynchronize(e[2]), "event sync");
        float a = 0, b = 0;
        check(cudaEventElapsedTime(&a, e[0], e[1]), "event");
        check(cudaEventElapsedTime(&b, e[1], e[2]), "event");
        if (pass == 0) {
          ms[0] += a;
        } else {
          ms[1] += a;
          ms[2] += b;
        }
      }
    }
  }
  for (auto& x : e) cudaEventDestroy(x);
  const int st = read_status();
  if (st & kStatusIoletRadius) rc = HB_ERR_IOLET_RADIUS;
  else if (st & kStatusUnstable) rc = HB_UNSTABLE;
  return rc;
}

// Turn post-collision f* into the pre-collision f the reference holds in f_old.
void Solver::materialise() {
  if (direct_) return;
  StepArgs a = args();
  launch_gather_f64(a, opt_.wall, stream_);
  check(cudaGetLastError(), "gather launch");
  cur_ = 1 - cur_;
  direct_ = true;
  prev_valid_ = false;
}

bool Solver::previous_aos_device(double* aos) {
  if (!prev_valid_) return false;
  if (mixed()) {
    to_aos(true, aos);
    return true;
  }
  StepArgs a = args();
  a.fin = f_[1 - cur_].as<double>();
  a.gin = ghost_[1 - cur_].as<double>();
  if (prev_direct_) {
    launch_soa_to_aos_f64(a.fin, L_.np, st2ref_.as<int>(), L_.n, aos, stream_);
  } else {
    launch_gather_aos_f64(a, opt_.wall, st2ref_.as<int>(), aos, stream_);
  }
  check(cudaGetLastError(), "previous-state gather");
  return true;
}

bool Solver::get_previous_fs(double* f) {
  DeviceBuffer tmp;
  tmp.alloc((size_t)L_.n * Q * sizeof(double));
  if (!previous_aos_device(tmp.as<double>())) return false;
  check(cudaMemcpyAsync(f, tmp.p, (size_t)L_.n * Q * sizeof(double), cudaMemcpyDeviceToHost, stream_), "f download");
  check(cudaStreamSynchronize(stream_), "get_previous_fs");
  return true;
}

Solver::Selection Solver::select(const hb_selector& sel, bool macro, const bool stress[6], bool distributions) {
  const int n = L_.n;
  const int64_t np = L_.np;
  if (macro && (!macro_valid_ || !rho_.p))
    throw Error{HB_ERR_ARG, "the last step did not fill the macroscopic caches (pass HB_STEP_MACRO)"};
  for (int k = 0; k < 6; k++)
    if (stress[k] && (!stress_valid_ || !pi_.p))
      throw Error{HB_ERR_ARG, "the last step did not fill the stress caches (pass HB_STEP_MACRO | HB_STEP_STRESS)"};
  if (!sel_coords_.p) {
    std::vector<int32_t> c((size_t)3 * n);
    std::vector<uint8_t> w(n), st(n);
    for (int i = 0; i < n; i++) {
      for (int d = 0; d < 3; d++) c[(size_t)3 * i + d] = (int32_t)t_.coords[(size_t)3 * i + d];
      w[i] = t_.wall[i] != 0;
      st[i] = (uint8_t)t_.stype[i];
    }
    std::vector<int> r2s(L_.ref2st.begin(), L_.ref2st.begin() + n);
    int64_t tot = 0;
    upload_vec(sel_coords_, c, tot);
    upload_vec(sel_wall_, w, tot);
    upload_vec(sel_stype_, st, tot);
    upload_vec(ref2st_, r2s, tot);
    dev_bytes_ += tot;
  }
  SelectArgs a{};
  selector_state(sel, &a);  // the reference selectors' float state (extraction.cpp)
  a.n = n;
  a.coords = sel_coords_.as<int32_t>();
  a.wall = sel_wall_.as<uint8_t>();
  a.stype = sel_stype_.as<uint8_t>();
  a.voxel = dx_;
  for (int d = 0; d < 3; d++) a.origin[d] = origin_[d];
  DeviceBuffer mask, counts, total, idx;
  mask.alloc((size_t)std::max(1, n));
  counts.alloc((size_t)std::max(1, select_blocks(n)) * sizeof(int));
  total.alloc(sizeof(int));
  idx.alloc((size_t)std::max(1, n) * sizeof(int));
  launch_select(a, mask.as<uint8_t>(), counts.as<int>(), total.as<int>(), idx.as<int>(), stream_);
  check(cudaGetLastError(), "selector launch");
  int m = 0;
  check(cudaMemcpyAsync(&m, total.p, sizeof(int), cudaMemcpyDeviceToHost, stream_), "selection count");
  check(cudaStreamSynchronize(stream_), "selection");
  Selection out;
  out.idx.resize(m);
  if (m > 0)
    check(cudaMemcpyAsync(out.idx.data(), idx.p, (size_t)m * sizeof(int), cudaMemcpyDeviceToHost, stream_), "selection");
  DeviceBuffer buf;
  auto fetch = [&](const double* src, int64_t stride, int width, std::vector<double>& dst) {
    dst.resize((size_t)m * width);
    if (m == 0) return;
    if (buf.bytes < (size_t)m * width * sizeof(double)) buf.alloc((size_t)m * 19 * sizeof(double));
    launch_gather_selected(src, stride, width, idx.as<int>(), ref2st_.as<int>(), m, buf.as<double>(), stream_);
    check(cudaGetLastError(), "selected gather");
    check(cudaMemcpyAsync(dst.data(), buf.p, dst.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_), "selected download");
    check(cudaStreamSynchronize(stream_), "selected download");
  };
  if (macro) {
    fetch(rho_.as<double>(), np, 1, out.rho);
    fetch(u_.as<double>(), np, 3, out.u);
    fetch(wss_.as<double>(), np, 1, out.wss);
  }
  for (int k = 0; k < 6; k++) {
    if (!stress[k]) continue;
    if (!stress_out_.p) {
      stress_out_.alloc((size_t)6 * np * sizeof(double));
      dev_bytes_ += (int64_t)stress_out_.bytes;
    }
    StepArgs sa = args();
    sa.pi = pi_.as<double>();
    launch_stress_field(sa, k, stress_out_.as<double>(), stream_);
    check(cudaGetLastError(), "stress field launch");
    fetch(stress_out_.as<double>(), np, stress_len(k), out.stress[k]);
  }
  if (distributions) {
    DeviceBuffer aos;
    aos.alloc((size_t)std::max(1, n) * Q * sizeof(double));
    if (!previous_aos_device(aos.as<double>()))
      throw Error{HB_ERR_ARG, "the distributions of the last step are no longer held"};
    out.fd.resize((size_t)m * Q);
    if (m > 0) {
      buf.alloc((size_t)m * Q * sizeof(double));
      launch_gather_rows(aos.as<double>(), Q, idx.as<int>(), m, buf.as<double>(), stream_);
      check(cudaGetLastError(), "selected rows");
      check(cudaMemcpyAsync(out.fd.data(), buf.p, out.fd.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_),
            "selected download");
    }
  }
  check(cudaStreamSynchronize(stream_), "selection");
  return out;
}

void Solver::set_units(double dt, double dx, const double origin[3]) {
  dt_ = dt;
  dx_ = dx;
  for (int k = 0; k < 3; k++) origin_[k] = origin[k];
}

void Solver::get_fs(double* f) {
  if (mixed()) {
    DeviceBuffer tmp;
    tmp.alloc((size_t)L_.n * Q * sizeof(double));
    to_aos(false, tmp.as<double>());
    check(cudaMemcpyAsync(f, tmp.p, (size_t)L_.n * Q * sizeof(double), cudaMemcpyDeviceToHost, stream_), "f download");
    check(cudaStreamSynchronize(stream_), "get_fs");
    return;
  }
  materialise();
  double* aos = f_[1 - cur_].as<double>();  // the spare buffer holds n*19 doubles
  launch_soa_to_aos_f64(f_[cur_].as<double>(), L_.np, st2ref_.as<int>(), L_.n, aos, stream_);
  check(cudaGetLastError(), "soa_to_aos launch");
  check(cudaMemcpyAsync(f, aos, (size_t)L_.n * Q * sizeof(double), cudaMemcpyDeviceToHost, stream_), "f download");
  check(cudaStreamSynchronize(stream_), "get_fs");
}

void Solver::set_fs(const double* f) {
  if (mixed()) {
    DeviceBuffer tmp;
    tmp.alloc((size_t)L_.n * Q * sizeof(double));
    check(cudaMemcpyAsync(tmp.p, f, (size_t)L_.n * Q * sizeof(double), cudaMemcpyHostToDevice, stream_), "f upload");
    launch_from_aos_mixed(tmp.as<double>(), st2ref_.as<int>(), L_.n, L_.np, opt_.precision, f_[cur_].p, stream_);
    check(cudaGetLastError(), "from_aos launch");
    direct_ = true;
    prev_valid_ = false;
    check(cudaStreamSynchronize(stream_), "set_fs");
    return;
  }
  double* aos = f_[1 - cur_].as<double>();
  check(cudaMemcpyAsync(aos, f, (size_t)L_.n * Q * sizeof(double), cudaMemcpyHostToDevice, stream_), "f upload");
  launch_aos_to_soa_f64(aos, st2ref_.as<int>(), L_.n, f_[cur_].as<double>(), L_.np, stream_);
  check(cudaGetLastError(), "aos_to_soa launch");
  direct_ = true;
  prev_valid_ = false;
  check(cudaStreamSynchronize(stream_), "set_fs");
}

void Solver::get_macro(double* rho, double* u, double* wss) {
  if (!macro_valid_ || !rho_.p) throw Error{HB_ERR_ARG, "no step has filled the macroscopic caches (pass HB_STEP_MACRO)"};
  const int n = L_.n;
  const int64_t np = L_.np;
  std::vector<double> r(np), uu(3 * np), w(np);
  check(cudaMemcpyAsync(r.data(), rho_.p, np * sizeof(double), cudaMemcpyDeviceToHost, stream_), "macro download");
  check(cudaMemcpyAsync(uu.data(), u_.p, 3 * np * sizeof(double), cudaMemcpyDeviceToHost, stream_), "macro download");
  check(cudaMemcpyAsync(w.data(), wss_.p, np * sizeof(double), cudaMemcpyDeviceToHost, stream_), "macro download");
  check(cudaStreamSynchronize(stream_), "get_macro");
  for (int s = 0; s < n; s++) {
    const int x = L_.st2ref[s];
    if (rho) rho[x] = r[s];
    if (u) {
      u[3 * x] = uu[s];
      u[3 * x + 1] = uu[np + s];
      u[3 * x + 2] = uu[2 * np + s];
    }
    if (wss) wss[x] = w[s];
  }
}

int Solver::stress_len(int field) {
  switch (field) {
    case HB_STRESS_VON_MISES:
    case HB_STRESS_SHEAR_RATE:
      return 1;
    case HB_STRESS_TENSOR:
      return 6;
    case HB_STRESS_TRACTION:
    case HB_STRESS_TANGENTIAL_TRACTION:
    case HB_STRESS_NORMAL_TRACTION:
      return 3;
    default:
      throw Error{HB_ERR_ARG, "unknown stress field " + std::to_string(field)};
  }
}

void Solver::get_stress(int field, double* out) {
  const int k = stress_len(field);
  if (!stress_valid_ || !pi_.p)
    throw Error{HB_ERR_ARG, "no step has filled the stress caches (pass HB_STEP_MACRO | HB_STEP_STRESS)"};
  const int n = L_.n;
  const int64_t np = L_.np;
  if (!stress_out_.p) {
    stress_out_.alloc((size_t)6 * np * sizeof(double));
    dev_bytes_ += (int64_t)stress_out_.bytes;
  }
  StepArgs a = args();
  a.pi = pi_.as<double>();
  launch_stress_field(a, field, stress_out_.as<double>(), stream_);
  check(cudaGetLastError(), "stress field launch");
  std::vector<double> v((size_t)k * np);
  check(cudaMemcpyAsync(v.data(), stress_out_.p, v.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_),
        "stress download");
  check(cudaStreamSynchronize(stream_), "get_stress");
  for (int s = 0; s < n; s++) {
    const int64_t x = L_.st2ref[s];
    for (int c = 0; c < k; c++) out[x * k + c] = v[(size_t)c * np + s];
  }
}

void Solver::moment_sums(double out[4]) {
  const int nb = moment_sum_blocks(L_.n);
  if (sum_scratch_.bytes < (size_t)std::max(1, nb) * 4 * sizeof(double)) {
    sum_scratch_.alloc((size_t)std::max(1, nb) * 4 * sizeof(double));
    sum_out_.alloc(4 * sizeof(double));
  }
  DeviceBuffer tmp;
  const double* f;
  int64_t dir_stride, site_stride;
  if (mixed()) {
    tmp.alloc((size_t)L_.n * Q * sizeof(double));
    to_aos(false, tmp.as<double>());
    f = tmp.as<double>();
    dir_stride = 1;
    site_stride = Q;
  } else {
    materialise();
    f = f_[cur_].as<double>();
    dir_stride = L_.np;
    site_stride = 1;
  }
  launch_moment_sums(f, dir_stride, site_stride, L_.n, sum_scratch_.as<double>(), sum_out_.as<double>(), stream_);
  check(cudaGetLastError(), "moment sums launch");
  check(cudaMemcpyAsync(out, sum_out_.p, 4 * sizeof(double), cudaMemcpyDeviceToHost, stream_), "sums download");
  check(cudaStreamSynchronize(stream_), "moment_sums");
}

// File layout of write_state (host byte order, little-endian on these hosts):
// char[8] "HBSTATE1"; int64 n, uint64 time step, int32 Windkessel iolets W,
// int32 coupling slots C; int64 coords[n*3] (reference order, to check the
// lattice on restore); double f[n*19] (AoS, reference order: the pre-collision
// distributions of the next step); W records of double density, density_new,
// flow, flow_old and int64 sites summed at the previous step; double cpl[C].
void Solver::write_state(const std::string& path) {
  if (mixed()) throw Error{HB_ERR_UNSUPPORTED, "the FP64 state file holds FP64 storage only"};
  const int64_t n = L_.n;
  std::vector<double> f((size_t)n * Q);
  get_fs(f.data());
  std::vector<WK3Dev> wk(nwk3_);
  if (nwk3_)
    check(cudaMemcpyAsync(wk.data(), wk3_.p, wk.size() * sizeof(WK3Dev), cudaMemcpyDeviceToHost, stream_), "state");
  const int32_t ncpl = L_.cpl_total;
  std::vector<double> cpl(std::max(1, ncpl));
  check(cudaMemcpyAsync(cpl.data(), cpl_buf_.p, cpl.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_), "state");
  check(cudaStreamSynchronize(stream_), "state");
  FILE* fh = std::fopen(path.c_str(), "wb");
  if (!fh) throw Error{HB_ERR_IO, "cannot write " + path};
  bool ok = std::fwrite("HBSTATE1", 1, 8, fh) == 8;
  const uint64_t t = t_step_;
  const int32_t w = nwk3_;
  ok = ok && std::fwrite(&n, 8, 1, fh) == 1 && std::fwrite(&t, 8, 1, fh) == 1 && std::fwrite(&w, 4, 1, fh) == 1 &&
       std::fwrite(&ncpl, 4, 1, fh) == 1;
  ok = ok && std::fwrite(t_.coords.data(), 8, (size_t)3 * n, fh) == (size_t)3 * n;
  ok = ok && std::fwrite(f.data(), 8, f.size(), fh) == f.size();
  for (const WK3Dev& x : wk) {
    const double v[4] = {x.density, x.density_new, x.flow, x.flow_old};
    const int64_t c = x.count_prev;
    ok = ok && std::fwrite(v, 8, 4, fh) == 4 && std::fwrite(&c, 8, 1, fh) == 1;
  }
  ok = ok && std::fwrite(cpl.data(), 8, (size_t)ncpl, fh) == (size_t)ncpl;
  ok = (std::fclose(fh) == 0) && ok;
  if (!ok) throw Error{HB_ERR_IO, "cannot write " + path};
}

void Solver::read_state(const std::string& path) {
  if (mixed()) throw Error{HB_ERR_UNSUPPORTED, "the FP64 state file holds FP64 storage only"};
  FILE* fh = std::fopen(path.c_str(), "rb");
  if (!fh) throw Error{HB_ERR_IO, "cannot open " + path};
  struct Closer {
    FILE* f;
    ~Closer() { std::fclose(f); }
  } closer{fh};
  char magic[8];
  int64_t n = 0;
  uint64_t t = 0;
  int32_t w = 0, ncpl = 0;
  if (std::fread(magic, 1, 8, fh) != 8 || std::memcmp(magic, "HBSTATE1", 8) != 0 || std::fread(&n, 8, 1, fh) != 1 ||
      std::fread(&t, 8, 1, fh) != 1 || std::fread(&w, 4, 1, fh) != 1 || std::fread(&ncpl, 4, 1, fh) != 1)
    throw Error{HB_ERR_FORMAT, path + ": not a state file"};
  if (n != L_.n || w != nwk3_ || ncpl != L_.cpl_total)
    throw Error{HB_ERR_FORMAT, path + ": the state file belongs to another lattice or case"};
  std::vector<int64_t> coords((size_t)3 * n);
  std::vector<double> f((size_t)n * Q);
  if (std::fread(coords.data(), 8, coords.size(), fh) != coords.size() || std::fread(f.data(), 8, f.size(), fh) != f.size())
    throw Error{HB_ERR_FORMAT, path + ": truncated state file"};
  if (std::memcmp(coords.data(), t_.coords.data(), coords.size() * 8) != 0)
    throw Error{HB_ERR_FORMAT, path + ": the state file's sites are not this lattice's, in this order"};
  std::vector<WK3Dev> wk(nwk3_);
  if (nwk3_)
    check(cudaMemcpyAsync(wk.data(), wk3_.p, wk.size() * sizeof(WK3Dev), cudaMemcpyDeviceToHost, stream_), "state");
  check(cudaStreamSynchronize(stream_), "state");
  for (WK3Dev& x : wk) {
    double v[4];
    int64_t c = 0;
    if (std::fread(v, 8, 4, fh) != 4 || std::fread(&c, 8, 1, fh) != 1) throw Error{HB_ERR_FORMAT, path + ": truncated state file"};
    x.density = v[0];
    x.density_new = v[1];
    x.flow = v[2];
    x.flow_old = v[3];
    x.count_prev = (int)c;
  }
  std::vector<double> cpl(std::max(1, ncpl), 0.0);
  if (std::fread(cpl.data(), 8, (size_t)ncpl, fh) != (size_t)ncpl) throw Error{HB_ERR_FORMAT, path + ": truncated state file"};
  set_fs(f.data());
  if (nwk3_)
    check(cudaMemcpyAsync(wk3_.p, wk.data(), wk.size() * sizeof(WK3Dev), cudaMemcpyHostToDevice, stream_), "state");
  check(cudaMemcpyAsync(cpl_buf_.p, cpl.data(), cpl.size() * sizeof(double), cudaMemcpyHostToDevice, stream_), "state");
  check(cudaStreamSynchronize(stream_), "state");
  t_step_ = t;
  rows_valid_ = false;
  macro_valid_ = stress_valid_ = false;
}

void Solver::get_wk3(int group, int index, double st[4]) {
  const int idx = group * 16 + index;
  for (size_t k = 0; k < L_.couplings.size(); k++) {
    if (L_.couplings[k].iolet != idx) continue;
    WK3Dev w;
    check(cudaMemcpyAsync(&w, wk3_.as<WK3Dev>() + k, sizeof(WK3Dev), cudaMemcpyDeviceToHost, stream_), "wk3 download");
    check(cudaStreamSynchronize(stream_), "get_wk3");
    st[0] = w.density;
    st[1] = w.density_new;
    st[2] = w.flow;
    st[3] = w.flow_old;
    return;
  }
  throw Error{HB_ERR_ARG, "iolet is not a Windkessel iolet"};
}

}  // namespace hb

namespace hb {

void Solver::attach_shard(int axis, int64_t lo, int64_t hi) {
  const HaloLists h = halo_lists(t_, L_, axis, lo, hi);
  int64_t tot = 0;
  for (int side = 0; side < 2; side++) {
    send_n_[side] = (int64_t)h.send[side].size();
    recv_n_[side] = (int64_t)h.recv[side].size();
    upload_vec(send_idx_[side], h.send[side].empty() ? std::vector<int64_t>{0} : h.send[side], tot);
    upload_vec(recv_idx_[side], h.recv[side].empty() ? std::vector<int64_t>{0} : h.recv[side], tot);
  }
  dev_bytes_ += tot;
  check(cudaEventCreateWithFlags(&xev_, cudaEventDisableTiming), "cudaEventCreate");
  shard_ = true;
}

void Solver::shard_sizes(int64_t counts[4]) const {
  counts[0] = send_n_[0];
  counts[1] = send_n_[1];
  counts[2] = recv_n_[0];
  counts[3] = recv_n_[1];
}

void Solver::shard_pack(void* to_lower, void* to_upper, cudaStream_t caller) {
  if (!shard_) throw Error{HB_ERR_ARG, "not a shard"};
  if ((send_n_[0] && !to_lower) || (send_n_[1] && !to_upper)) throw Error{HB_ERR_ARG, "missing send buffer"};
  // The buffer holding the last step's post-collision values (direct mode: the
  // values set by hb_set_fs, which the neighbours' first step does not read).
  const void* f = f_[cur_].p;
  void* out[2] = {to_lower, to_upper};
  for (int side = 0; side < 2; side++)
    if (send_n_[side]) launch_halo_pack(f, send_idx_[side].as<int64_t>(), send_n_[side], out[side], (int)elem_bytes(), stream_);
  check(cudaGetLastError(), "halo pack");
  check(cudaEventRecord(xev_, stream_), "event");
  if (caller && caller != stream_) check(cudaStreamWaitEvent(caller, xev_, 0), "stream wait");
}

void Solver::shard_unpack(const void* from_lower, const void* from_upper, cudaStream_t caller) {
  if (!shard_) throw Error{HB_ERR_ARG, "not a shard"};
  if ((recv_n_[0] && !from_lower) || (recv_n_[1] && !from_upper)) throw Error{HB_ERR_ARG, "missing receive buffer"};
  if (caller && caller != stream_) {
    check(cudaEventRecord(xev_, caller), "event");
    check(cudaStreamWaitEvent(stream_, xev_, 0), "stream wait");
  }
  const void* in[2] = {from_lower, from_upper};
  for (int side = 0; side < 2; side++)
    if (recv_n_[side]) launch_halo_unpack(in[side], recv_idx_[side].as<int64_t>(), recv_n_[side], f_[cur_].p, (int)elem_bytes(), stream_);
  check(cudaGetLastError(), "halo unpack");
}

}  // namespace hb
