// capi.cpp -- the extern "C" boundary (include/hemeb200.h).  No C++ exception
// crosses it: every entry point catches and returns an HB_* status.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <string>

#include "../../include/hemeb200.h"
#include "batch.h"
#include "config.h"
#include "extraction.h"
#include "solver.h"
#include "shard.h"

struct hb_handle {
  std::unique_ptr<hb::Solver> solver;
  std::string error;
  // Wall-clock ms of hb_create_from_xml's phases: case file, geometry decode
  // (and, with the device reader, the layout and the tables' copy back), the
  // solver's construction (layout when not built already, uploads, initial state).
  double setup_ms[4] = {0, 0, 0, 0};
};

struct hb_geometry {
  hb::LatticeTables tables;
  hb::GmyTiming timing;
};

struct hb_batch {
  std::unique_ptr<hb::Batch> batch;
};

namespace {

thread_local std::string g_create_error;

template <class F>
int guard(hb_handle* h, F&& fn) {
  try {
    return fn();
  } catch (const hb::Error& e) {
    if (h) h->error = e.msg;
    else g_create_error = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    if (h) h->error = "host memory exhausted";
    else g_create_error = "host memory exhausted";
    return HB_ERR_OOM;
  } catch (const std::exception& e) {
    if (h) h->error = e.what();
    else g_create_error = e.what();
    return HB_ERR_ARG;
  }
}

int finish_create(hb::LatticeTables t, const hb_params& p, const hb_options& o, hb_handle** out,
                  hb::Layout* layout = nullptr) {
  auto h = std::make_unique<hb_handle>();
  h->solver = std::make_unique<hb::Solver>(std::move(t), p, o, layout);
  *out = h.release();
  return HB_OK;
}

}  // namespace

namespace hb {
// Message for hb_last_error(NULL, ...) from entry points that take no handle.
void set_last_error(const std::string& msg) { g_create_error = msg; }
}  // namespace hb

extern "C" {

void hb_default_options(hb_options* opt) {
  if (!opt) return;
  opt->kernel = HB_KERNEL_LBGK;
  opt->wall = HB_WALL_SBB;
  opt->precision = HB_STORE_FP64;
  opt->device = 0;
  opt->geometry_reader = HB_GEOMETRY_DEVICE;
}

int hb_create_from_xml(const char* xml_path, const hb_options* opt, hb_handle** out) {
  if (!xml_path || !out) return HB_ERR_ARG;
  *out = nullptr;
  return guard(nullptr, [&] {
    hb_options o;
    hb_default_options(&o);
    if (opt) o = *opt;
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    hb::CaseConfig c = hb::read_case(xml_path, o.kernel);
    const auto t1 = clk::now();
    // The device reader also lays the lattice out on the device.
    hb::Layout L;
    const bool dev = o.geometry_reader == HB_GEOMETRY_DEVICE;
    if (dev) hb::validate_case(c.params, o);
    hb::LatticeTables t = dev ? hb::read_gmy_device(c.gmy_path, o.device, nullptr, &c.params, o.wall, &L)
                              : hb::read_gmy(c.gmy_path);
    const auto t2 = clk::now();
    int rc = finish_create(std::move(t), c.params, o, out, dev ? &L : nullptr);
    if (rc == HB_OK) {
      (*out)->solver->set_units(c.dt, c.dx, c.origin);
      const auto t3 = clk::now();
      auto ms = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
      (*out)->setup_ms[0] = ms(t0, t1);
      (*out)->setup_ms[1] = ms(t1, t2);
      (*out)->setup_ms[2] = ms(t2, t3);
      (*out)->setup_ms[3] = ms(t0, t3);
    }
    if (rc == HB_OK && !c.checkpoint_file.empty()) {
      std::string cp = c.checkpoint_file;
      if (!cp.empty() && cp[0] != '/') {
        std::string xp(xml_path);
        size_t sl = xp.rfind('/');
        if (sl != std::string::npos) cp = xp.substr(0, sl + 1) + cp;
      }
      try {
        hb::read_checkpoint(*(*out)->solver, cp, c.has_time ? c.params.initial_step : 0);
      } catch (...) {
        delete *out;
        *out = nullptr;
        throw;
      }
    }
    return rc;
  });
}

int hb_write_state(hb_handle* h, const char* path) {
  if (!h || !path) return HB_ERR_ARG;
  return guard(h, [&] {
    h->solver->write_state(path);
    return HB_OK;
  });
}

int hb_read_state(hb_handle* h, const char* path) {
  if (!h || !path) return HB_ERR_ARG;
  return guard(h, [&] {
    h->solver->read_state(path);
    return HB_OK;
  });
}

int hb_shard_plan(const char* xml_path, int kernel, int n_shards, int* axis, int64_t* bounds) {
  if (!xml_path || !axis || !bounds || n_shards < 1) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    hb::CaseConfig c = hb::read_case(xml_path, kernel);
    hb::LatticeTables t = hb::read_gmy(c.gmy_path);
    const std::vector<int64_t> b = hb::plan_slabs(t, n_shards, axis);
    std::copy(b.begin(), b.end(), bounds);
    return HB_OK;
  });
}

int hb_create_shard_from_xml(const char* xml_path, const hb_options* opt, const hb_shard* shard, hb_handle** out) {
  if (!xml_path || !shard || !out) return HB_ERR_ARG;
  *out = nullptr;
  return guard(nullptr, [&] {
    hb_options o;
    hb_default_options(&o);
    if (opt) o = *opt;
    hb::CaseConfig c = hb::read_case(xml_path, o.kernel);
    if (!c.checkpoint_file.empty())
      throw hb::Error{HB_ERR_UNSUPPORTED, "a shard starts from the equilibrium: set its distributions with hb_set_fs"};
    hb::LatticeTables full = o.geometry_reader == HB_GEOMETRY_DEVICE ? hb::read_gmy_device(c.gmy_path, o.device)
                                                                      : hb::read_gmy(c.gmy_path);
    hb::LatticeTables t = hb::cut_shard(full, c.params, shard->axis, shard->lo, shard->hi);
    full = hb::LatticeTables();
    int rc = finish_create(std::move(t), c.params, o, out);
    if (rc != HB_OK) return rc;
    try {
      (*out)->solver->attach_shard(shard->axis, shard->lo, shard->hi);
    } catch (...) {
      delete *out;
      *out = nullptr;
      throw;
    }
    (*out)->solver->set_units(c.dt, c.dx, c.origin);
    return HB_OK;
  });
}

int hb_shard_halo_sizes(const hb_handle* h, int64_t counts[4], int* elem_bytes) {
  if (!h || !counts) return HB_ERR_ARG;
  if (!h->solver->sharded()) return HB_ERR_ARG;
  h->solver->shard_sizes(counts);
  if (elem_bytes) *elem_bytes = h->solver->elem_size();
  return HB_OK;
}

int hb_shard_pack(hb_handle* h, void* to_lower, void* to_upper, void* stream) {
  if (!h) return HB_ERR_ARG;
  return guard(h, [&] {
    h->solver->shard_pack(to_lower, to_upper, static_cast<cudaStream_t>(stream));
    return HB_OK;
  });
}

int hb_shard_unpack(hb_handle* h, const void* from_lower, const void* from_upper, void* stream) {
  if (!h) return HB_ERR_ARG;
  return guard(h, [&] {
    h->solver->shard_unpack(from_lower, from_upper, static_cast<cudaStream_t>(stream));
    return HB_OK;
  });
}

int hb_shard_site_ids(const hb_handle* h, int64_t* ids) {
  if (!h || !ids) return HB_ERR_ARG;
  const hb::LatticeTables& t = h->solver->tables();
  const int64_t n = t.owned();
  for (int64_t k = 0; k < n; k++) ids[k] = t.gid.empty() ? k : t.gid[k];
  return HB_OK;
}

int hb_shard_describe(const char* xml_path, int kernel, int wall, const hb_shard* shard, int64_t counts[6],
                      int64_t* owned, int64_t* halo, int64_t* send_lower, int64_t* send_upper, int64_t* recv_lower,
                      int64_t* recv_upper) {
  if (!xml_path || !shard || !counts) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    hb::CaseConfig c = hb::read_case(xml_path, kernel);
    hb::LatticeTables full = hb::read_gmy(c.gmy_path);
    hb::LatticeTables t = hb::cut_shard(full, c.params, shard->axis, shard->lo, shard->hi);
    const hb::Layout L = hb::build_layout(t, c.params, wall);
    const hb::HaloLists hl = hb::halo_lists(t, L, shard->axis, shard->lo, shard->hi);
    const int64_t no = t.owned();
    counts[0] = no;
    counts[1] = t.n - no;
    counts[2] = (int64_t)hl.send[0].size();
    counts[3] = (int64_t)hl.send[1].size();
    counts[4] = (int64_t)hl.recv[0].size();
    counts[5] = (int64_t)hl.recv[1].size();
    if (owned) std::copy(t.gid.begin(), t.gid.begin() + no, owned);
    if (halo) std::copy(t.gid.begin() + no, t.gid.end(), halo);
    int64_t* lists[4] = {send_lower, send_upper, recv_lower, recv_upper};
    const std::vector<int64_t>* src[4] = {&hl.send_pairs[0], &hl.send_pairs[1], &hl.recv_pairs[0], &hl.recv_pairs[1]};
    for (int k = 0; k < 4; k++)
      if (lists[k]) std::copy(src[k]->begin(), src[k]->end(), lists[k]);
    return HB_OK;
  });
}

int hb_create(const hb_lattice_desc* lat, const hb_params* params, const hb_options* opt, hb_handle** out) {
  if (!lat || !params || !out || lat->n_sites <= 0 || !lat->coords || !lat->wall_mask || !lat->iolet_mask ||
      !lat->site_type || !lat->iolet_id)
    return HB_ERR_ARG;
  *out = nullptr;
  return guard(nullptr, [&] {
    hb_options o;
    hb_default_options(&o);
    if (opt) o = *opt;
    hb::LatticeTables t;
    const int64_t n = lat->n_sites;
    t.n = n;
    for (int d = 0; d < 3; d++) t.dims[d] = lat->dims[d];
    t.coords.assign(lat->coords, lat->coords + 3 * n);
    t.wall.assign(lat->wall_mask, lat->wall_mask + n);
    t.iolet.assign(lat->iolet_mask, lat->iolet_mask + n);
    t.stype.assign(lat->site_type, lat->site_type + n);
    t.iolet_id.assign(lat->iolet_id, lat->iolet_id + n);
    if (lat->wall_distance) t.q.assign(lat->wall_distance, lat->wall_distance + 18 * n);
    if (lat->wall_normal) t.normal.assign(lat->wall_normal, lat->wall_normal + 3 * n);
    else t.normal.assign(3 * n, 0.0f);
    for (int64_t i = 0; i < n; i++) t.type_counts[t.collision_type(i)]++;
    if (lat->neighbours) t.nbr.assign(lat->neighbours, lat->neighbours + 19 * n);
    return finish_create(std::move(t), *params, o, out);
  });
}

int hb_destroy(hb_handle* h) {
  if (!h) return HB_ERR_ARG;
  delete h;
  return HB_OK;
}

int hb_last_error(const hb_handle* h, char* msg, size_t len) {
  if (!msg || len == 0) return HB_ERR_ARG;
  const std::string& e = h ? h->error : g_create_error;
  std::strncpy(msg, e.c_str(), len - 1);
  msg[len - 1] = '\0';
  return HB_OK;
}

int hb_request_comms(hb_handle* h) {
  if (!h) return HB_ERR_ARG;
  return guard(h, [&] {
    h->solver->request_comms();
    return HB_OK;
  });
}

int hb_pre_send(hb_handle* h) { return h ? HB_OK : HB_ERR_ARG; }

int hb_pre_receive(hb_handle* h, uint32_t flags) {
  if (!h) return HB_ERR_ARG;
  return guard(h, [&] {
    h->solver->pre_receive((flags & HB_STEP_MACRO) != 0, 3, (flags & HB_STEP_STRESS) != 0);
    return HB_OK;
  });
}

int hb_post_receive(hb_handle* h) { return h ? HB_OK : HB_ERR_ARG; }

int hb_end_iteration(hb_handle* h) {
  if (!h) return HB_ERR_ARG;
  return guard(h, [&] {
    h->solver->end_iteration();
    const int st = h->solver->read_status();
    if (st & hb::kStatusIoletRadius) return HB_ERR_IOLET_RADIUS;
    if (st & hb::kStatusUnstable) return HB_UNSTABLE;
    return HB_OK;
  });
}

int hb_step(hb_handle* h, int64_t n_steps, uint32_t flags) {
  if (!h) return HB_ERR_ARG;
  return guard(h, [&] { return h->solver->step(n_steps, flags); });
}

int hb_site_count(const hb_handle* h, int64_t* n) {
  if (!h || !n) return HB_ERR_ARG;
  *n = h->solver->tables().owned();  // a shard's own sites, without its halo
  return HB_OK;
}

int hb_time_step(const hb_handle* h, uint64_t* t) {
  if (!h || !t) return HB_ERR_ARG;
  *t = h->solver->time_step();
  return HB_OK;
}

int hb_set_time_step(hb_handle* h, uint64_t t) {
  if (!h || t == 0) return HB_ERR_ARG;
  h->solver->set_time_step(t);
  return HB_OK;
}

int hb_get_params(const hb_handle* h, hb_params* p) {
  if (!h || !p) return HB_ERR_ARG;
  *p = h->solver->params();
  return HB_OK;
}

int hb_get_fs(hb_handle* h, double* f) {
  if (!h || !f) return HB_ERR_ARG;
  return guard(h, [&] {
    h->solver->get_fs(f);
    return HB_OK;
  });
}

int hb_set_fs(hb_handle* h, const double* f) {
  if (!h || !f) return HB_ERR_ARG;
  return guard(h, [&] {
    h->solver->set_fs(f);
    return HB_OK;
  });
}

int hb_get_macro(hb_handle* h, double* density, double* velocity, double* wss) {
  if (!h) return HB_ERR_ARG;
  return guard(h, [&] {
    h->solver->get_macro(density, velocity, wss);
    return HB_OK;
  });
}

int hb_get_stress(hb_handle* h, int field, double* out) {
  if (!h || !out) return HB_ERR_ARG;
  return guard(h, [&] {
    h->solver->get_stress(field, out);
    return HB_OK;
  });
}

int hb_set_iolet_densities(hb_handle* h, const double* inlet_density, int n_inlets, const double* outlet_density,
                           int n_outlets) {
  if (!h) return HB_ERR_ARG;
  return guard(h, [&] {
    h->solver->set_iolet_densities(inlet_density, n_inlets, outlet_density, n_outlets);
    return HB_OK;
  });
}

int hb_moment_sums(hb_handle* h, double sums[4]) {
  if (!h || !sums) return HB_ERR_ARG;
  return guard(h, [&] {
    h->solver->moment_sums(sums);
    return HB_OK;
  });
}

int hb_get_wk3(hb_handle* h, int group, int index, double state[4]) {
  if (!h || !state || group < 0 || group > 1 || index < 0 || index > 15) return HB_ERR_ARG;
  return guard(h, [&] {
    h->solver->get_wk3(group, index, state);
    return HB_OK;
  });
}

int hb_get_tables(const hb_handle* h, int64_t* neighbours, uint32_t* wall_mask, uint32_t* iolet_mask, int32_t* site_type,
                  int32_t* iolet_id, int64_t* coords, int64_t* type_counts) {
  if (!h) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    const hb::LatticeTables& t = h->solver->tables();
    const size_t n = (size_t)t.owned();
    if (neighbours) {
      if ((int64_t)n == t.n) {
        hb::neighbour_table(t, neighbours);
      } else {  // a shard: its own sites' rows, indices in the shard's numbering (halo sites after the owned ones)
        std::vector<int64_t> all((size_t)t.n * hb::Q);
        hb::neighbour_table(t, all.data());
        std::memcpy(neighbours, all.data(), n * hb::Q * sizeof(int64_t));
      }
    }
    if (wall_mask) std::memcpy(wall_mask, t.wall.data(), n * sizeof(uint32_t));
    if (iolet_mask) std::memcpy(iolet_mask, t.iolet.data(), n * sizeof(uint32_t));
    if (site_type) std::memcpy(site_type, t.stype.data(), n * sizeof(int32_t));
    if (iolet_id) std::memcpy(iolet_id, t.iolet_id.data(), n * sizeof(int32_t));
    if (coords) std::memcpy(coords, t.coords.data(), n * 3 * sizeof(int64_t));
    if (type_counts) std::memcpy(type_counts, t.type_counts, 6 * sizeof(int64_t));
    return HB_OK;
  });
}

int hb_write_xtr(hb_handle* h, const char* path, const char* fields, const char* offset_path) {
  if (!h || !path || !fields) return HB_ERR_ARG;
  return guard(h, [&] {
    hb::write_xtr(*h->solver, path, fields, offset_path ? offset_path : "");
    return HB_OK;
  });
}

int hb_write_xtr_selected(hb_handle* h, const char* path, const char* fields, const char* offset_path,
                          const hb_selector* sel) {
  if (!h || !path || !fields || !sel) return HB_ERR_ARG;
  return guard(h, [&] {
    hb::write_xtr(*h->solver, path, fields, offset_path ? offset_path : "", sel);
    return HB_OK;
  });
}

int hb_read_checkpoint(hb_handle* h, const char* path, uint64_t step) {
  if (!h || !path) return HB_ERR_ARG;
  return guard(h, [&] {
    hb::read_checkpoint(*h->solver, path, step);
    return HB_OK;
  });
}

namespace {

hb::LatticeTables tables_from_desc(const hb_lattice_desc* lat) {
  hb::LatticeTables t;
  const int64_t n = lat->n_sites;
  t.n = n;
  for (int d = 0; d < 3; d++) t.dims[d] = lat->dims[d];
  t.coords.assign(lat->coords, lat->coords + 3 * n);
  t.wall.assign(lat->wall_mask, lat->wall_mask + n);
  t.iolet.assign(lat->iolet_mask, lat->iolet_mask + n);
  t.stype.assign(lat->site_type, lat->site_type + n);
  t.iolet_id.assign(lat->iolet_id, lat->iolet_id + n);
  if (lat->wall_distance) t.q.assign(lat->wall_distance, lat->wall_distance + 18 * n);
  if (lat->wall_normal) t.normal.assign(lat->wall_normal, lat->wall_normal + 3 * n);
  else t.normal.assign(3 * n, 0.0f);
  for (int64_t i = 0; i < n; i++) t.type_counts[t.collision_type(i)]++;
  if (lat->neighbours) t.nbr.assign(lat->neighbours, lat->neighbours + 19 * n);
  return t;
}

}  // namespace

int hb_batch_bytes(int64_t site_capacity, int64_t general_capacity, int max_lattices, int precision, int64_t* bytes) {
  if (!bytes) return HB_ERR_ARG;
  *bytes = hb::Batch::bytes_for(site_capacity, general_capacity, max_lattices, precision);
  return HB_OK;
}

int hb_batch_create(int64_t site_capacity, int64_t general_capacity, int max_lattices, int precision, int device,
                    hb_batch** out) {
  if (!out) return HB_ERR_ARG;
  *out = nullptr;
  return guard(nullptr, [&] {
    auto b = std::make_unique<hb_batch>();
    b->batch = std::make_unique<hb::Batch>(site_capacity, general_capacity, max_lattices, precision, device);
    *out = b.release();
    return HB_OK;
  });
}

int hb_batch_destroy(hb_batch* b) {
  if (!b) return HB_ERR_ARG;
  delete b;
  return HB_OK;
}

int hb_batch_add_xml(hb_batch* b, const char* xml_path, int kernel, int wall, uint64_t steps, int* slot) {
  if (!b || !xml_path || !slot) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    hb::CaseConfig c = hb::read_case(xml_path, kernel);
    *slot = b->batch->add(hb::read_gmy(c.gmy_path), c.params, kernel, wall, steps);
    return HB_OK;
  });
}

int hb_batch_add(hb_batch* b, const hb_lattice_desc* lat, const hb_params* params, int kernel, int wall, uint64_t steps,
                 int* slot) {
  if (!b || !lat || !params || !slot || lat->n_sites <= 0 || !lat->coords || !lat->wall_mask || !lat->iolet_mask ||
      !lat->site_type || !lat->iolet_id)
    return HB_ERR_ARG;
  return guard(nullptr, [&] {
    *slot = b->batch->add(tables_from_desc(lat), *params, kernel, wall, steps);
    return HB_OK;
  });
}

struct hb_batch_prep {
  std::unique_ptr<hb::PreparedLattice> prep;
};

int hb_batch_prepare_xml(const char* xml_path, int kernel, int wall, uint64_t steps, hb_batch_prep** out) {
  if (!xml_path || !out) return HB_ERR_ARG;
  *out = nullptr;
  return guard(nullptr, [&] {
    hb::CaseConfig c = hb::read_case(xml_path, kernel);
    auto h = std::make_unique<hb_batch_prep>();
    h->prep = hb::prepare_lattice(hb::read_gmy(c.gmy_path), c.params, kernel, wall, steps);
    *out = h.release();
    return HB_OK;
  });
}

int hb_batch_prepare_xml_device(const char* xml_path, int kernel, int wall, uint64_t steps, int device,
                                hb_batch_prep** out) {
  if (!xml_path || !out) return HB_ERR_ARG;
  *out = nullptr;
  return guard(nullptr, [&] {
    hb::CaseConfig c = hb::read_case(xml_path, kernel);
    hb::validate_batch_case(c.params, kernel, wall);
    hb::Layout L;
    hb::LatticeTables t = hb::read_gmy_device(c.gmy_path, device, nullptr, &c.params, wall, &L);
    auto h = std::make_unique<hb_batch_prep>();
    h->prep = hb::prepare_lattice(std::move(t), c.params, kernel, wall, steps, &L);
    *out = h.release();
    return HB_OK;
  });
}

int hb_batch_prep_sites(const hb_batch_prep* prep, int64_t* sites) {
  if (!prep || !sites || !prep->prep) return HB_ERR_ARG;
  *sites = prep->prep->L.n;
  return HB_OK;
}

int hb_batch_add_prepared(hb_batch* b, hb_batch_prep* prep, int* slot) {
  if (!b || !prep || !slot || !prep->prep) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    *slot = b->batch->add(*prep->prep);
    return HB_OK;
  });
}

int hb_batch_prep_free(hb_batch_prep* prep) {
  delete prep;
  return HB_OK;
}

int hb_batch_remove(hb_batch* b, int slot) {
  if (!b) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    b->batch->remove(slot);
    return HB_OK;
  });
}

int hb_batch_run(hb_batch* b, int k, int* finished, int max_finished, int* n_finished) {
  if (!b || k < 0) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    std::vector<int> done = b->batch->run(k);
    int m = 0;
    for (int s : done)
      if (finished && m < max_finished) finished[m++] = s;
    if (n_finished) *n_finished = finished ? m : (int)done.size();
    return HB_OK;
  });
}

int hb_batch_get_macro(hb_batch* b, int slot, double* density, double* velocity, double* wss) {
  if (!b) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    b->batch->get_macro(slot, density, velocity, wss);
    return HB_OK;
  });
}

int hb_batch_member_info(hb_batch* b, int slot, int64_t* sites, uint64_t* time_step, int* status) {
  if (!b) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    if (sites) *sites = b->batch->member_sites(slot);
    if (time_step) *time_step = b->batch->time_step(slot);
    if (status) *status = b->batch->status(slot);
    return HB_OK;
  });
}

int hb_batch_set_tuning(hb_batch* b, int sites_per_thread, int block) {
  if (!b) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    b->batch->set_tuning(sites_per_thread, block);
    return HB_OK;
  });
}

int hb_batch_set_step_form(hb_batch* b, int form) {
  if (!b) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    b->batch->set_step_form(form);
    return HB_OK;
  });
}

int hb_batch_stats(const hb_batch* b, double* last_block_ms, int64_t* active_sites, int64_t* device_bytes) {
  if (!b) return HB_ERR_ARG;
  if (last_block_ms) *last_block_ms = b->batch->last_ms();
  if (active_sites) *active_sites = b->batch->active_sites();
  if (device_bytes) *device_bytes = b->batch->device_bytes();
  return HB_OK;
}

int hb_read_case(const char* xml_path, int kernel, hb_params* params, char* gmy_path, size_t gmy_path_len) {
  if (!xml_path || !params) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    hb::CaseConfig c = hb::read_case(xml_path, kernel);
    *params = c.params;
    // The file iolets' tables live in `c`: the caller gets them from hb_read_case_iolet_table.
    for (int k = 0; k < 16; k++) params->inlets[k].table = params->outlets[k].table = nullptr;
    if (gmy_path && gmy_path_len) {
      std::strncpy(gmy_path, c.gmy_path.c_str(), gmy_path_len - 1);
      gmy_path[gmy_path_len - 1] = '\0';
    }
    return HB_OK;
  });
}

int hb_read_case_iolet_table(const char* xml_path, int kernel, int outlet, int index, double* out, uint64_t count) {
  if (!xml_path || !out || index < 0 || index >= 16 || (outlet != 0 && outlet != 1)) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    hb::CaseConfig c = hb::read_case(xml_path, kernel);
    const std::vector<double>& t = c.tables[16 * outlet + index];
    if (t.empty()) throw hb::Error{HB_ERR_ARG, "that iolet is not a file iolet"};
    for (uint64_t k = 0; k < count; k++) out[k] = t[k < t.size() ? k : t.size() - 1];
    return HB_OK;
  });
}

int hb_iolet_velocity(const hb_iolet* iolet, const double x[3], uint64_t t, double v[3]) {
  if (!iolet || !x || !v) return HB_ERR_ARG;
  return guard(nullptr, [&] { return hb::iolet_velocity(*iolet, x, t, v); });
}

int hb_geometry_open(const char* gmy_path, hb_geometry** out) {
  if (!gmy_path || !out) return HB_ERR_ARG;
  *out = nullptr;
  return guard(nullptr, [&] {
    auto g = std::make_unique<hb_geometry>();
    const auto t0 = std::chrono::steady_clock::now();
    g->tables = hb::read_gmy(gmy_path);
    g->timing.read_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    *out = g.release();
    return HB_OK;
  });
}

int hb_geometry_open_device(const char* gmy_path, int device, hb_geometry** out) {
  if (!gmy_path || !out) return HB_ERR_ARG;
  *out = nullptr;
  return guard(nullptr, [&] {
    auto g = std::make_unique<hb_geometry>();
    g->tables = hb::read_gmy_device(gmy_path, device, &g->timing);
    *out = g.release();
    return HB_OK;
  });
}

int hb_geometry_read_timing(const hb_geometry* g, double ms[5]) {
  if (!g || !ms) return HB_ERR_ARG;
  ms[0] = g->timing.read_ms;
  ms[1] = g->timing.inflate_ms;
  ms[2] = g->timing.h2d_ms;
  ms[3] = g->timing.device_ms;
  ms[4] = g->timing.d2h_ms;
  return HB_OK;
}

int hb_geometry_site_count(const hb_geometry* g, int64_t* n, int64_t dims[3]) {
  if (!g || !n) return HB_ERR_ARG;
  *n = g->tables.n;
  if (dims)
    for (int d = 0; d < 3; d++) dims[d] = g->tables.dims[d];
  return HB_OK;
}

int hb_geometry_select(const hb_geometry* g, const hb_selector* sel, double voxel_size, const double origin[3],
                       uint8_t* mask) {
  if (!g || !sel || !origin || !mask || !(voxel_size > 0)) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    const std::vector<uint8_t> m = hb::select_sites(g->tables, *sel, voxel_size, origin);
    std::memcpy(mask, m.data(), m.size());
    return HB_OK;
  });
}

int hb_geometry_tables(const hb_geometry* g, int64_t* neighbours, uint32_t* wall_mask, uint32_t* iolet_mask,
                       int32_t* site_type, int32_t* iolet_id, int64_t* coords, int64_t* type_counts,
                       double* wall_distance, double* wall_normal) {
  if (!g) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    const hb::LatticeTables& t = g->tables;
    const size_t n = (size_t)t.n;
    if (neighbours) hb::neighbour_table(t, neighbours);
    if (wall_mask) std::memcpy(wall_mask, t.wall.data(), n * sizeof(uint32_t));
    if (iolet_mask) std::memcpy(iolet_mask, t.iolet.data(), n * sizeof(uint32_t));
    if (site_type) std::memcpy(site_type, t.stype.data(), n * sizeof(int32_t));
    if (iolet_id) std::memcpy(iolet_id, t.iolet_id.data(), n * sizeof(int32_t));
    if (coords) std::memcpy(coords, t.coords.data(), n * 3 * sizeof(int64_t));
    if (type_counts) std::memcpy(type_counts, t.type_counts, 6 * sizeof(int64_t));
    if (wall_distance) {
      if (t.q.empty()) return HB_ERR_ARG;
      for (size_t k = 0; k < 18 * n; k++) wall_distance[k] = (double)t.q[k];
    }
    if (wall_normal)
      for (size_t k = 0; k < 3 * n; k++) wall_normal[k] = (double)t.normal[k];
    return HB_OK;
  });
}

int hb_geometry_layout(const hb_geometry* g, const hb_params* params, int wall, int64_t stats[4]) {
  if (!g || !params || !stats) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    hb::Layout L = hb::build_layout(g->tables, *params, wall);
    stats[0] = L.axis;
    stats[1] = L.runs;
    stats[2] = L.bulk_sites;
    stats[3] = L.G;
    return HB_OK;
  });
}

int hb_geometry_layout_digest(const hb_geometry* g, const hb_params* params, int wall, int device, uint64_t digest[32]) {
  if (!g || !params || !digest) return HB_ERR_ARG;
  return guard(nullptr, [&] {
    const hb::Layout L = device < 0 ? hb::build_layout(g->tables, *params, wall)
                                    : hb::build_layout_on_device(g->tables, *params, wall, device);
    hb::layout_digest(L, digest);
    return HB_OK;
  });
}

int hb_geometry_close(hb_geometry* g) {
  if (!g) return HB_ERR_ARG;
  delete g;
  return HB_OK;
}

int hb_setup_timing(const hb_handle* h, double ms[4]) {
  if (!h || !ms) return HB_ERR_ARG;
  for (int k = 0; k < 4; k++) ms[k] = h->setup_ms[k];
  return HB_OK;
}

int hb_last_step_timing(const hb_handle* h, double* ms, int64_t* launches) {
  if (!h) return HB_ERR_ARG;
  if (ms) *ms = h->solver->last_ms();
  if (launches) *launches = h->solver->last_launches();
  return HB_OK;
}

int hb_profile_steps(hb_handle* h, int64_t n_steps, double ms[3]) {
  if (!h || !ms || n_steps < 0) return HB_ERR_ARG;
  return guard(h, [&] { return h->solver->profile(n_steps, ms); });
}

int hb_device_bytes(const hb_handle* h, int64_t* bytes) {
  if (!h || !bytes) return HB_ERR_ARG;
  *bytes = h->solver->device_bytes();
  return HB_OK;
}

}  // extern "C"
