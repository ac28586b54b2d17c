// batch.cpp -- host side of the batched form: arenas, admission, retirement,
// CUDA-graph blocks of steps.
//
// Every member owns ranges in four arenas (sites, runs, boundary records,
// lattice slots), taken first-fit at admission and given back at removal, so
// members join and leave without moving anyone else's state.  The per-lattice
// record on the device carries the time step, so a captured graph of k steps
// replays as long as the membership does not change.
#include "batch.h"

#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstring>

#include "batch_dev.h"

namespace hb {

void RangeAlloc::reset(int64_t capacity) {
  cap_ = capacity;
  free_.clear();
  used_.clear();
  if (capacity > 0) free_[0] = capacity;
}

int64_t RangeAlloc::take(int64_t n) {
  if (n <= 0) n = 1;
  for (auto it = free_.begin(); it != free_.end(); ++it) {
    if (it->second < n) continue;
    const int64_t start = it->first, len = it->second;
    free_.erase(it);
    if (len > n) free_[start + n] = len - n;
    used_[start] = n;
    return start;
  }
  return -1;
}

void RangeAlloc::give(int64_t start, int64_t n) {
  auto u = used_.find(start);
  if (u == used_.end()) return;
  n = u->second;
  used_.erase(u);
  auto next = free_.lower_bound(start);
  if (next != free_.end() && next->first == start + n) {
    n += next->second;
    free_.erase(next);
  }
  auto prev = free_.lower_bound(start);
  if (prev != free_.begin()) {
    --prev;
    if (prev->first + prev->second == start) {
      prev->second += n;
      return;
    }
  }
  free_[start] = n;
}

int64_t RangeAlloc::high_water() const {
  if (used_.empty()) return 0;
  auto last = std::prev(used_.end());
  return last->first + last->second;
}

void Batch::check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error{HB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

int64_t Batch::bytes_for(int64_t site_capacity, int64_t general_capacity, int max_lattices, int precision) {
  const int64_t np = ((site_capacity + 63) / 64) * 64;
  const int64_t elem = precision == HB_STORE_FP16 ? 2 : 4;
  const int64_t runs = std::max<int64_t>(1024, site_capacity / 4);
  const int64_t g = std::max<int64_t>(64, general_capacity);
  return 2 * 19 * np * elem + 2 * 18 * g * 4 + 4 * g * 4 + 2 * g * 5 + np * 4 + runs * 20 * 4 + g * (4 * 8 + 18 * 8 + 3 * 8) +
         np * 5 * 8 + (int64_t)max_lattices * (sizeof(BatchLatDev) + 32 * (sizeof(BatchCosDev) + sizeof(IoletDev) + 8) + 4);
}

Batch::Batch(int64_t site_capacity, int64_t general_capacity, int max_lattices, int precision, int device)
    : device_(device), precision_(precision) {
  if (precision != HB_STORE_FP32 && precision != HB_STORE_FP16)
    throw Error{HB_ERR_UNSUPPORTED, "the batched form stores shifted FP32 or FP16 distributions"};
  if (site_capacity <= 0 || site_capacity > ((int64_t)1 << 31) - 64 || max_lattices <= 0 || max_lattices > kMaxBatchLattices)
    throw Error{HB_ERR_ARG, "batch capacity out of range"};
  cap_sites_ = site_capacity;
  np_ = ((site_capacity + 63) / 64) * 64;
  cap_gen_ = std::max<int64_t>(64, general_capacity);
  max_lat_ = max_lattices;
  run_cap_ = std::max<int64_t>(1024, site_capacity / 4);
  sites_.reset(np_);
  gens_.reset(cap_gen_);
  iols_.reset(2 * cap_gen_);
  runs_.reset(run_cap_);
  for (int s = max_lat_ - 1; s >= 0; s--) free_slots_.push_back(s);
  check(cudaSetDevice(device_), "cudaSetDevice");
  cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device_);
  check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  // The latency-bound boundary kernel runs on the side stream at the highest
  // priority, so its blocks are dispatched ahead of the bulk kernel's queued ones
  // (4M-site pipe: FP32 step 29.3k -> 30.3k MLUPS; FP64 unchanged).
  int prio_lo = 0, prio_hi = 0;
  check(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi), "cudaDeviceGetStreamPriorityRange");
  check(cudaStreamCreateWithPriority(&side_, cudaStreamNonBlocking, prio_hi), "cudaStreamCreate");
  check(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "cudaEventCreate");
  check(cudaEventCreateWithFlags(&join_, cudaEventDisableTiming), "cudaEventCreate");
  check(cudaEventCreate(&ev0_), "cudaEventCreate");
  check(cudaEventCreate(&ev1_), "cudaEventCreate");
  const size_t elem = precision == HB_STORE_FP16 ? 2 : 4;
  auto alloc = [&](DeviceBuffer& b, size_t bytes, int fill) {
    b.alloc(bytes);
    dev_bytes_ += (int64_t)bytes;
    if (fill >= 0) check(cudaMemset(b.p, fill, bytes), "cudaMemset");
  };
  for (int k = 0; k < 2; k++) {
    alloc(f_[k], (size_t)Q * np_ * elem, 0);
    alloc(ghost_[k], (size_t)18 * cap_gen_ * sizeof(float), 0);
  }
  alloc(meta_, (size_t)np_ * sizeof(int), 0xFF);
  alloc(run_off_, (size_t)run_cap_ * 20 * sizeof(int), 0);
  alloc(g_site_, (size_t)cap_gen_ * sizeof(int), 0);
  alloc(g_run_, (size_t)cap_gen_ * sizeof(int), 0xFF);
  alloc(g_wall_, (size_t)cap_gen_ * sizeof(uint32_t), 0);
  alloc(g_iolet_, (size_t)cap_gen_ * sizeof(uint32_t), 0);
  alloc(g_src_, (size_t)18 * cap_gen_ * sizeof(int), 0);
  alloc(g_q_, (size_t)18 * cap_gen_ * sizeof(float), 0);
  alloc(g_nrm_, (size_t)3 * cap_gen_ * sizeof(float), 0);
  alloc(g_io_, (size_t)cap_gen_ * sizeof(int), 0xFF);
  alloc(g_cpl_, (size_t)cap_gen_ * sizeof(int), 0xFF);
  alloc(g_xyz_, (size_t)3 * cap_gen_ * sizeof(int), 0);
  alloc(g_lat_, (size_t)cap_gen_ * sizeof(int), 0xFF);
  alloc(lat_, (size_t)max_lat_ * sizeof(BatchLatDev), 0);
  alloc(cos_, (size_t)max_lat_ * 32 * sizeof(BatchCosDev), 0);
  alloc(iolets_, (size_t)max_lat_ * 32 * sizeof(IoletDev), 0);
  alloc(dens_, (size_t)max_lat_ * 32 * sizeof(double), 0);
  alloc(lat_status_, (size_t)max_lat_ * sizeof(int), 0);
  alloc(macro_list_, (size_t)max_lat_ * sizeof(int), 0);
  alloc(macro_count_, sizeof(int), 0);
  alloc(io_moments_, (size_t)4 * cap_gen_ * sizeof(float), 0);
  alloc(iol_list_, (size_t)2 * cap_gen_ * sizeof(int), 0xFF);
  alloc(iol_link_, (size_t)2 * cap_gen_, 0);
  alloc(rho_, (size_t)np_ * sizeof(double), 0);
  alloc(u_, (size_t)3 * np_ * sizeof(double), 0);
  alloc(wss_, (size_t)np_ * sizeof(double), 0);
  check(cudaDeviceSynchronize(), "batch initialisation");
}

Batch::~Batch() {
  if (stream_) cudaStreamSynchronize(stream_);
  if (graph_) cudaGraphExecDestroy(graph_);
  for (cudaEvent_t e : {ev0_, ev1_, fork_, join_})
    if (e) cudaEventDestroy(e);
  if (side_) cudaStreamDestroy(side_);
  if (stream_) cudaStreamDestroy(stream_);
}

void Batch::set_tuning(int spt, int bulk_block) {
  if ((spt != 1 && spt != 2) || (bulk_block != 128 && bulk_block != 256))
    throw Error{HB_ERR_ARG, "sites per thread must be 1 or 2 and the block 128 or 256 threads"};
  spt_ = spt;
  bulk_block_ = bulk_block;
  dirty_ = true;
}

void Batch::set_step_form(int form) {
  if (form != HB_BATCH_STEP_PERSISTENT && form != HB_BATCH_STEP_SPLIT) throw Error{HB_ERR_ARG, "unknown step form"};
  form_ = form;
  dirty_ = true;
}

int64_t Batch::active_sites() const {
  int64_t n = 0;
  for (auto& kv : members_)
    if (!kv.second->finished) n += kv.second->L.n;
  return n;
}

int64_t Batch::member_sites(int slot) const {
  auto it = members_.find(slot);
  if (it == members_.end()) throw Error{HB_ERR_ARG, "no such batch member"};
  return it->second->L.n;
}

namespace {

template <class T>
void put(DeviceBuffer& b, int64_t offset, const T* src, int64_t count, cudaStream_t st) {
  if (count <= 0) return;
  cudaError_t e = cudaMemcpyAsync(b.as<T>() + offset, src, (size_t)count * sizeof(T), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) throw Error{HB_ERR_CUDA, std::string("batch upload: ") + cudaGetErrorString(e)};
}

// rows x count block of a [rows][pitch] device array, from a [rows][count] host array.
template <class T>
void put_rows(DeviceBuffer& b, int64_t pitch, int64_t offset, const T* src, int64_t count, int rows, cudaStream_t st) {
  if (count <= 0) return;
  cudaError_t e = cudaMemcpy2DAsync(b.as<T>() + offset, (size_t)pitch * sizeof(T), src, (size_t)count * sizeof(T),
                                    (size_t)count * sizeof(T), (size_t)rows, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) throw Error{HB_ERR_CUDA, std::string("batch upload: ") + cudaGetErrorString(e)};
}

}  // namespace

void Batch::write_member_tables(const BatchMember& m) {
  const Layout& L = m.L;
  const int n = L.n, G = L.G;
  std::vector<int> meta(m.site_len, -1);
  for (int s = 0; s < n; s++) meta[s] = L.meta[s] >= 0 ? L.meta[s] + (int)m.run_base : L.meta[s] - (int)m.gen_base;
  put(meta_, m.site_base, meta.data(), (int64_t)meta.size(), stream_);
  // Run rows: the offsets of the layout, and the member's slot in the spare last entry.
  std::vector<int> rows(L.run_off);
  for (int r = 0; r < L.runs; r++) rows[(size_t)r * 20 + 19] = m.slot;
  put(run_off_, m.run_base * 20, rows.data(), (int64_t)rows.size(), stream_);
  if (G > 0) {
    std::vector<int> site(G), run(G), src((size_t)18 * G), lat(G, m.slot), cpl(G, -1);
    for (int g = 0; g < G; g++) {
      site[g] = L.g_site[g] + (int)m.site_base;
      run[g] = L.g_run[g] >= 0 ? L.g_run[g] + (int)m.run_base : -1;
    }
    for (size_t k = 0; k < src.size(); k++) src[k] = L.g_src[k] + (int)m.site_base;
    put(g_site_, m.gen_base, site.data(), G, stream_);
    put(g_run_, m.gen_base, run.data(), G, stream_);
    put(g_wall_, m.gen_base, L.g_wall.data(), G, stream_);
    put(g_iolet_, m.gen_base, L.g_iolet.data(), G, stream_);
    put(g_io_, m.gen_base, L.g_io.data(), G, stream_);
    put(g_cpl_, m.gen_base, cpl.data(), G, stream_);
    put(g_lat_, m.gen_base, lat.data(), G, stream_);
    put_rows(g_src_, cap_gen_, m.gen_base, src.data(), G, 18, stream_);
    put_rows(g_q_, cap_gen_, m.gen_base, L.g_q.data(), G, 18, stream_);
    put_rows(g_nrm_, cap_gen_, m.gen_base, L.g_nrm.data(), G, 3, stream_);
    put_rows(g_xyz_, cap_gen_, m.gen_base, L.g_xyz.data(), G, 3, stream_);
    std::vector<int> iol;
    std::vector<uint8_t> link;
    for (int g = 0; g < G; g++)
      for (int d = 1; d < Q; d++)
        if ((L.g_iolet[g] >> (d - 1)) & 1u) {
          iol.push_back(g + (int)m.gen_base);
          link.push_back((uint8_t)d);
        }
    put(iol_list_, m.iol_base, iol.data(), (int64_t)iol.size(), stream_);
    put(iol_link_, m.iol_base, link.data(), (int64_t)link.size(), stream_);
  }
}

void Batch::clear_member_tables(const BatchMember& m) {
  check(cudaMemsetAsync(meta_.as<int>() + m.site_base, 0xFF, (size_t)m.site_len * sizeof(int), stream_), "clear");
  check(cudaMemsetAsync(g_lat_.as<int>() + m.gen_base, 0xFF, (size_t)std::max(1, m.L.G) * sizeof(int), stream_), "clear");
  check(cudaMemsetAsync(iol_list_.as<int>() + m.iol_base, 0xFF, (size_t)std::max<int64_t>(1, m.iol_len) * sizeof(int), stream_),
        "clear");
  BatchLatDev z;
  std::memset(&z, 0, sizeof(z));
  check(cudaMemcpyAsync(lat_.as<BatchLatDev>() + m.slot, &z, sizeof(z), cudaMemcpyHostToDevice, stream_), "clear");
  check(cudaStreamSynchronize(stream_), "clear");
}

void validate_batch_case(const hb_params& p, int kernel, int wall) {
  if (kernel != kLBGK && kernel != kTRT) throw Error{HB_ERR_UNSUPPORTED, "the batched form runs LBGK or TRT"};
  if (wall != kSBB && wall != kBFL) throw Error{HB_ERR_UNSUPPORTED, "the batched form runs bounce-back or BFL walls"};
  for (int k = 0; k < p.n_inlets + p.n_outlets; k++) {
    const hb_iolet& io = k < p.n_inlets ? p.inlets[k] : p.outlets[k - p.n_inlets];
    if (io.kind != kCosine && io.kind != kParabolic)
      throw Error{HB_ERR_UNSUPPORTED, "the batched form runs cosine pressure and parabolic velocity iolets"};
  }
  if (!(p.tau > 0.5)) throw Error{HB_ERR_ARG, "tau must exceed 1/2"};
}

std::unique_ptr<PreparedLattice> prepare_lattice(LatticeTables t, const hb_params& p, int kernel, int wall, uint64_t steps,
                                                 Layout* layout) {
  validate_batch_case(p, kernel, wall);
  if (wall == kBFL && t.q.empty()) throw Error{HB_ERR_ARG, "BFL walls need wall distances"};
  auto prep = std::make_unique<PreparedLattice>();
  if (layout) prep->L = std::move(*layout);
  else prep->L = build_layout(t, p, wall);
  prep->t = std::move(t);
  prep->p = p;
  prep->kernel = kernel;
  prep->wall = wall;
  prep->steps = steps;
  return prep;
}

int Batch::add(LatticeTables t, const hb_params& p, int kernel, int wall, uint64_t steps) {
  auto prep = prepare_lattice(std::move(t), p, kernel, wall, steps);
  return add(*prep);
}

int Batch::add(PreparedLattice& prep) {
  if (prep.taken) throw Error{HB_ERR_ARG, "the prepared lattice was already admitted"};
  if (free_slots_.empty()) throw Error{HB_ERR_OOM, "no free lattice slot in the batch"};
  const int n = prep.L.n;
  const int64_t site_len = ((n + 63) / 64) * 64;
  const int64_t site_base = sites_.take(site_len);
  const int64_t run_base = site_base < 0 ? -1 : runs_.take(prep.L.runs);
  const int64_t gen_base = run_base < 0 ? -1 : gens_.take(std::max(1, prep.L.G));
  int64_t iol_len = 0;
  for (int g = 0; g < prep.L.G; g++) iol_len += __builtin_popcount(prep.L.g_iolet[g]);
  const int64_t iol_base = gen_base < 0 ? -1 : iols_.take(std::max<int64_t>(1, iol_len));
  if (site_base < 0 || run_base < 0 || gen_base < 0 || iol_base < 0) {
    if (site_base >= 0) sites_.give(site_base, site_len);
    if (run_base >= 0) runs_.give(run_base, prep.L.runs);
    if (gen_base >= 0) gens_.give(gen_base, std::max(1, prep.L.G));
    throw Error{HB_ERR_OOM, "the lattice does not fit in the batch's free capacity"};
  }
  auto m = std::make_unique<BatchMember>();
  m->L = std::move(prep.L);
  prep.taken = true;
  m->site_len = site_len;
  m->site_base = site_base;
  m->run_base = run_base;
  m->gen_base = gen_base;
  m->iol_base = iol_base;
  m->iol_len = iol_len;
  const hb_params& p = prep.p;
  const int kernel = prep.kernel, wall = prep.wall;
  const uint64_t steps = prep.steps;
  m->slot = free_slots_.back();
  free_slots_.pop_back();
  m->t = std::move(prep.t);
  m->p = p;
  m->kernel = kernel;
  m->wall = wall;
  m->steps = steps;
  m->t_first = p.initial_step ? p.initial_step : 1;
  m->buffer_at_admission = cur_;
  write_member_tables(*m);

  // Per-lattice records: relaxation times and time, iolets, cosine parameters.
  BatchLatDev d;
  std::memset(&d, 0, sizeof(d));
  d.tau = p.tau;
  d.omega = -1.0 / p.tau;
  d.omega_minus = -1.0 / (0.5 + p.relaxation_parameter / (p.tau - 0.5));
  d.t = m->t_first;
  d.t_first = m->t_first;
  d.t_end = m->t_first + steps;
  d.site_base = m->site_base;
  d.n_sites = m->L.n;
  d.kernel = kernel;
  d.wall = wall;
  d.io_base = 32 * m->slot;
  std::vector<IoletDev> io(32);
  std::vector<BatchCosDev> cs(32);
  std::memset(io.data(), 0, io.size() * sizeof(IoletDev));
  std::memset(cs.data(), 0, cs.size() * sizeof(BatchCosDev));
  double mind = 1.7976931348623157e308;
  for (int k = 0; k < p.n_inlets + p.n_outlets; k++) {
    const hb_iolet& c = k < p.n_inlets ? p.inlets[k] : p.outlets[k - p.n_inlets];
    mind = std::min(mind, c.kind == kCosine ? c.density_mean - c.density_amp : 1.0);
  }
  for (int idx = 0; idx < 32; idx++) {
    const int cnt = idx < 16 ? p.n_inlets : p.n_outlets;
    cs[idx].kind = -1;
    if (idx % 16 >= cnt) continue;
    const hb_iolet& c = idx < 16 ? p.inlets[idx] : p.outlets[idx - 16];
    IoletDev& v = io[idx];
    v.kind = c.kind;
    v.dir0 = m->L.dir0[idx];
    v.wk3 = -1;
    for (int k = 0; k < 3; k++) {
      v.pos[k] = c.position[k];
      v.nrm[k] = c.normal[k];
      v.nrm_f[k] = (double)(float)c.normal[k];
    }
    v.radius = c.radius;
    v.max_speed = c.max_speed;
    v.warmup = c.warmup;
    cs[idx] = BatchCosDev{c.density_mean, c.density_amp, c.phase, c.period, mind, c.warmup, c.kind, 0};
  }
  check(cudaMemcpyAsync(lat_.as<BatchLatDev>() + m->slot, &d, sizeof(d), cudaMemcpyHostToDevice, stream_), "lattice record");
  check(cudaMemcpyAsync(iolets_.as<IoletDev>() + 32 * m->slot, io.data(), 32 * sizeof(IoletDev), cudaMemcpyHostToDevice, stream_),
        "iolet records");
  check(cudaMemcpyAsync(cos_.as<BatchCosDev>() + 32 * m->slot, cs.data(), 32 * sizeof(BatchCosDev), cudaMemcpyHostToDevice, stream_),
        "cosine records");
  check(cudaMemsetAsync(lat_status_.as<int>() + m->slot, 0, sizeof(int), stream_), "status");
  // Equilibrium initial condition in shifted form.  The uniform state at rest is
  // its own post-collision state, so it is written as the distributions the next
  // step gathers from, and as the iolet ghosts that step reads.
  float geq[Q], ghost[18];
  {
    const double rho = p.initial_density;
    for (int i = 0; i < Q; i++) geq[i] = (float)(weight(i) * rho - weight(i));
    for (int d = 1; d < Q; d++) ghost[d - 1] = geq[inv(d)];
  }
  launch_fill_shift(f_[cur_].p, np_, m->site_base, m->L.n, geq, precision_, stream_);
  launch_fill_ghost(ghost_[cur_].as<float>(), cap_gen_, m->gen_base, m->L.G, ghost, stream_);
  check(cudaGetLastError(), "initial fill");
  check(cudaStreamSynchronize(stream_), "admission");
  const int slot = m->slot;
  members_[slot] = std::move(m);
  dirty_ = true;
  return slot;
}

void Batch::remove(int slot) {
  auto it = members_.find(slot);
  if (it == members_.end()) throw Error{HB_ERR_ARG, "no such batch member"};
  const BatchMember& m = *it->second;
  clear_member_tables(m);
  sites_.give(m.site_base, m.site_len);
  runs_.give(m.run_base, m.L.runs);
  gens_.give(m.gen_base, std::max(1, m.L.G));
  iols_.give(m.iol_base, std::max<int64_t>(1, m.iol_len));
  free_slots_.push_back(slot);
  members_.erase(it);
  dirty_ = true;
}

void Batch::capture(int k) {
  if (graph_) {
    cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }
  int per_sm = 0;
  if (batch_occupancy(precision_, spt_, bulk_block_, &per_sm) != 0) throw Error{HB_ERR_CUDA, "occupancy query failed"};
  const int64_t sites_hw = sites_.high_water(), gens_hw = gens_.high_water();
  const int span = bulk_block_ * spt_;
  const int bulk_tiles = (int)((sites_hw + span - 1) / span);
  const int gen_block = form_ == HB_BATCH_STEP_SPLIT ? kBatchGenBlock : bulk_block_;
  const int gen_tiles = (int)((gens_hw + gen_block - 1) / gen_block);
  const int grid = std::max(1, std::min(bulk_tiles + gen_tiles, sm_count_ * std::max(1, per_sm)));
  const int macro_grid = 2 * sm_count_;
  const int64_t iols_hw = iols_.high_water();
  const int ghost_grid = std::max(1, std::min((int)((iols_hw + 127) / 128), 8 * sm_count_));
  int n_lat = 0;
  for (auto& kv : members_) n_lat = std::max(n_lat, kv.first + 1);

  StepArgs base;
  std::memset(&base, 0, sizeof(base));
  base.np = np_;
  base.n = (int)sites_hw;
  base.meta = meta_.as<int>();
  base.run_off = run_off_.as<int>();
  base.run_po = nullptr;
  base.gen.G = (int)cap_gen_;
  base.gen.site = g_site_.as<int>();
  base.gen.run = g_run_.as<int>();
  base.gen.wall = g_wall_.as<uint32_t>();
  base.gen.iolet = g_iolet_.as<uint32_t>();
  base.gen.src = g_src_.as<int>();
  base.gen.q = g_q_.as<float>();
  base.gen.nrm = g_nrm_.as<float>();
  base.gen.io = g_io_.as<int>();
  base.gen.cpl = g_cpl_.as<int>();
  base.gen.xyz = g_xyz_.as<int>();
  base.iolets = iolets_.as<IoletDev>();
  base.rho = rho_.as<double>();
  base.u = u_.as<double>();
  base.wss = wss_.as<double>();

  check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "graph capture");
  for (int j = 0; j < k; j++) {
    const int par = (cur_ + j) & 1;
    BatchArgs b;
    std::memset(&b, 0, sizeof(b));
    b.base = base;
    b.fin = f_[par].p;
    b.fout = f_[1 - par].p;
    b.gin = ghost_[par].as<float>();
    b.gout = ghost_[1 - par].as<float>();
    b.lat = lat_.as<BatchLatDev>();
    b.g_lat = g_lat_.as<int>();
    b.dens = dens_.as<double>();
    b.lat_status = lat_status_.as<int>();
    b.macro_list = macro_list_.as<int>();
    b.macro_count = macro_count_.as<int>();
    b.io_moments = io_moments_.as<float>();
    b.iol_list = iol_list_.as<int>();
    b.iol_link = iol_link_.as<uint8_t>();
    b.iol_count = (int)iols_hw;
    b.n_lat = n_lat;
    b.bulk_tiles = bulk_tiles;
    b.gen_tiles = gen_tiles;
    launch_batch_begin(lat_.p, cos_.p, dens_.as<double>(), macro_list_.as<int>(), macro_count_.as<int>(), n_lat, stream_);
    if (form_ == HB_BATCH_STEP_SPLIT) {
      // boundary tiles on the side stream beside the bulk tiles (a fork and a
      // join inside the captured graph)
      check(cudaEventRecord(fork_, stream_), "fork");
      check(cudaStreamWaitEvent(side_, fork_, 0), "fork");
      launch_batch_gen(b, precision_, side_);
      check(cudaEventRecord(join_, side_), "join");
      launch_batch_bulk(b, precision_, spt_, bulk_block_, stream_);
      check(cudaStreamWaitEvent(stream_, join_, 0), "join");
    } else {
      launch_batch_step(b, precision_, spt_, bulk_block_, grid, stream_);
    }
    launch_batch_ghosts(b, precision_, ghost_grid, stream_);
    launch_batch_macro(b, precision_, macro_grid, stream_);
  }
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(stream_, &g);
  if (e != cudaSuccess) throw Error{HB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e)};
  e = cudaGraphInstantiate(&graph_, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) throw Error{HB_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e)};
  graph_k_ = k;
  dirty_ = false;
}

std::vector<int> Batch::run(int k) {
  std::vector<int> done;
  if (k <= 0 || members_.empty()) return done;
  // The graph alternates the buffers starting from the parity it was captured
  // for; an odd block leaves the other parity current, so it is captured again.
  // A block of k steps replays a graph of `sub` steps k / sub times: membership
  // changes (every admission and retirement) re-capture and re-instantiate the
  // graph, and a 50-step graph costs a quarter of a 200-step one to build.
  const int sub = (k > 50 && k % 50 == 0) ? 50 : k;
  if (dirty_ || graph_k_ != sub) capture(sub);
  check(cudaEventRecord(ev0_, stream_), "event");
  for (int r = 0; r < k / sub; r++) check(cudaGraphLaunch(graph_, stream_), "graph launch");
  check(cudaEventRecord(ev1_, stream_), "event");
  check(cudaStreamSynchronize(stream_), "batch block");
  float ms = 0;
  cudaEventElapsedTime(&ms, ev0_, ev1_);
  last_ms_ = ms;
  cur_ = (cur_ + k) & 1;
  if (k % 2) dirty_ = true;
  std::vector<BatchLatDev> lat(max_lat_);
  std::vector<int> status(max_lat_);
  check(cudaMemcpy(lat.data(), lat_.p, (size_t)max_lat_ * sizeof(BatchLatDev), cudaMemcpyDeviceToHost), "lattice records");
  check(cudaMemcpy(status.data(), lat_status_.p, (size_t)max_lat_ * sizeof(int), cudaMemcpyDeviceToHost), "status");
  for (auto& kv : members_) {
    BatchMember& m = *kv.second;
    if (m.finished) continue;
    const BatchLatDev& d = lat[m.slot];
    const uint64_t reached = d.t + (uint64_t)d.ran_prev;
    if (reached >= d.t_end) {
      m.finished = true;
      done.push_back(m.slot);
    } else if (status[m.slot]) {
      // Unstable (or a parabolic point outside its iolet): stop stepping it and
      // hand it back now; its macroscopic fields are not filled.
      m.finished = true;
      done.push_back(m.slot);
      const uint64_t t_end = reached;
      check(cudaMemcpy(reinterpret_cast<char*>(lat_.as<BatchLatDev>() + m.slot) + offsetof(BatchLatDev, t_end), &t_end,
                       sizeof(t_end), cudaMemcpyHostToDevice),
            "stop member");
    }
  }
  return done;
}

int Batch::status(int slot) {
  int st = 0;
  check(cudaMemcpy(&st, lat_status_.as<int>() + slot, sizeof(int), cudaMemcpyDeviceToHost), "status");
  return st;
}

uint64_t Batch::time_step(int slot) {
  BatchLatDev d;
  check(cudaMemcpy(&d, lat_.as<BatchLatDev>() + slot, sizeof(d), cudaMemcpyDeviceToHost), "lattice record");
  return d.t + (uint64_t)d.ran_prev;
}

void Batch::get_macro(int slot, double* rho, double* u, double* wss) {
  auto it = members_.find(slot);
  if (it == members_.end()) throw Error{HB_ERR_ARG, "no such batch member"};
  const BatchMember& m = *it->second;
  if (!m.finished) throw Error{HB_ERR_ARG, "the member has not finished; its fields are filled on its last step"};
  const int n = m.L.n;
  std::vector<double> r(n), uu(3 * (size_t)n), w(n);
  check(cudaMemcpy(r.data(), rho_.as<double>() + m.site_base, n * sizeof(double), cudaMemcpyDeviceToHost), "macro");
  for (int c = 0; c < 3; c++)
    check(cudaMemcpy(uu.data() + (size_t)c * n, u_.as<double>() + c * np_ + m.site_base, n * sizeof(double), cudaMemcpyDeviceToHost),
          "macro");
  check(cudaMemcpy(w.data(), wss_.as<double>() + m.site_base, n * sizeof(double), cudaMemcpyDeviceToHost), "macro");
  for (int s = 0; s < n; s++) {
    const int x = m.L.st2ref[s];
    if (rho) rho[x] = r[s];
    if (u) {
      u[3 * (size_t)x] = uu[s];
      u[3 * (size_t)x + 1] = uu[(size_t)n + s];
      u[3 * (size_t)x + 2] = uu[2 * (size_t)n + s];
    }
    if (wss) wss[x] = w[s];
  }
}

}  // namespace hb
