// layout.cpp -- storage order, run table and gather rules for the pull form.
//
// Storage order: sites sorted along the axis that gives the fewest runs (maximal
// contiguous segments of fluid sites along that axis), rows ordered by the other
// two coordinates.  A plain bulk site s pulls slot i from s + run_off[run][i];
// consecutive threads read consecutive addresses.
//
// Gather rules are derived from the reference's push semantics, one writer per
// slot of f_new (src/lb/streamers/StreamerTypeFactory.h:47-300):
//   * a site of collision type 2..5 sends iolet links to its iolet delegate,
//     which writes its own slot inv(d);
//   * a site of type 1, 4 or 5 sends wall links to the wall delegate, which
//     writes its own slot inv(d);
//   * every other link pushes into neighbourIndices[site*19 + d].
// Each slot of every site must have exactly one writer; otherwise the lattice is
// rejected (the reference's result would depend on its loop order or on stale data).
#include "layout.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <thread>

namespace hb {

int closest_direction(const double n[3]) {
  double best = 1.7976931348623157e308;
  int bi = 0;
  for (int k = 0; k < Q; k++) {
    double c[3] = {(double)cx(k), (double)cy(k), (double)cz(k)};
    const double m2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
    if (m2 != 0.0) {
      const double m = std::sqrt(m2);
      c[0] /= m;
      c[1] /= m;
      c[2] /= m;
    }
    const double ex = c[0] - n[0], ey = c[1] - n[1], ez = c[2] - n[2];
    const double dist = ex * ex + ey * ey + ez * ez;
    if (dist < best) {
      best = dist;
      bi = k;
    }
  }
  return bi;
}

namespace {

// Runs f(begin, end) over [0, n) split across up to 16 host threads (one when n
// is small).  f must not throw; passes report errors through an atomic code.
template <class F>
void parallel_for(int64_t n, F f) {
  const int64_t chunk_min = 1 << 16;
  int T = (int)std::min<int64_t>(std::max(1u, std::min(16u, std::thread::hardware_concurrency())),
                                 std::max<int64_t>(1, n / chunk_min));
  if (T <= 1) {
    f((int64_t)0, n);
    return;
  }
  std::vector<std::thread> pool;
  for (int k = 1; k < T; k++) pool.emplace_back([&, k] { f(n * k / T, n * (k + 1) / T); });
  f((int64_t)0, n / T);
  for (auto& th : pool) th.join();
}

// First error of a parallel pass (0 = none): HB_ERR_* code and message.
struct PassError {
  std::atomic<int> code{0};
  const char* msg = nullptr;
  void set(int c, const char* m) {
    int z = 0;
    if (code.compare_exchange_strong(z, c)) msg = m;
  }
  void raise() const {
    if (code.load()) throw Error{code.load(), msg};
  }
};

}  // namespace

Layout build_layout(const LatticeTables& t, const hb_params& p, int wall) {
  Layout L;
  // Sites [n, nt) of a shard's tables are halo sites: stored after the owned
  // sites, never updated, their pushes into owned sites recorded as pulls.
  const int64_t nt64 = t.n;
  const int64_t n64 = t.owned();
  if (n64 <= 0) throw Error{HB_ERR_ARG, "lattice has no fluid sites"};
  if (nt64 > (int64_t)1 << 30) throw Error{HB_ERR_UNSUPPORTED, "more than 2^30 sites in one lattice"};
  const int n = (int)n64, nt = (int)nt64;
  L.n = n;
  L.n_halo = nt - n;
  L.np = ((nt64 + 63) / 64) * 64;
  const int64_t D[3] = {t.dims[0], t.dims[1], t.dims[2]};
  PassError err;

  // Dense grid of reference indices.
  std::vector<int32_t> grid(D[0] * D[1] * D[2], -1);
  auto gidx = [&](int64_t x, int64_t y, int64_t z) { return (x * D[1] + y) * D[2] + z; };
  parallel_for(nt, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; i++) {
      const int64_t* c = &t.coords[3 * i];
      if (c[0] < 0 || c[1] < 0 || c[2] < 0 || c[0] >= D[0] || c[1] >= D[1] || c[2] >= D[2]) {
        err.set(HB_ERR_BAD_INDEX, "site coordinates outside the lattice");
        return;
      }
      int32_t expected = -1;
      if (!__atomic_compare_exchange_n(&grid[gidx(c[0], c[1], c[2])], &expected, (int32_t)i, false, __ATOMIC_RELAXED,
                                       __ATOMIC_RELAXED)) {
        err.set(HB_ERR_BAD_INDEX, "two sites share coordinates");
        return;
      }
    }
  });
  err.raise();
  // neighbourIndices[x*19 + d]: the tables' own when they carry one, else from the grid
  // (LatticeData::InitialiseNeighbourLookup).
  // (For a shard the rubbish slot is nt * Q.)
  auto neighbour = [&](int x, int d) -> int64_t {
    if (!t.nbr.empty()) return t.nbr[(size_t)x * Q + d];
    const int64_t px = t.coords[3 * x] + cx(d), py = t.coords[3 * x + 1] + cy(d), pz = t.coords[3 * x + 2] + cz(d);
    if (px < 0 || py < 0 || pz < 0 || px >= D[0] || py >= D[1] || pz >= D[2]) return nt64 * Q;
    const int32_t g = grid[gidx(px, py, pz)];
    return g >= 0 ? (int64_t)g * Q + d : nt64 * Q;
  };
  // An owned site at these coordinates (runs join owned sites only).
  auto owned_at = [&](const int64_t* c) {
    const int32_t g = grid[gidx(c[0], c[1], c[2])];
    return g >= 0 && g < n;
  };

  // Run axis: fewest sites whose predecessor along the axis is not fluid.
  int64_t best_runs = -1;
  for (int a = 0; a < 3; a++) {
    std::atomic<int64_t> runs{0};
    parallel_for(n, [&](int64_t b, int64_t e) {
      int64_t r = 0;
      for (int64_t i = b; i < e; i++) {
        int64_t c[3] = {t.coords[3 * i], t.coords[3 * i + 1], t.coords[3 * i + 2]};
        c[a] -= 1;
        if (c[a] < 0 || !owned_at(c)) r++;
      }
      runs += r;
    });
    if (best_runs < 0 || runs.load() < best_runs) {
      best_runs = runs.load();
      L.axis = a;
    }
  }
  const int a0 = L.axis, a1 = (a0 + 1) % 3, a2 = (a0 + 2) % 3;

  // Storage order: rows along a0, ordered by (c[a2], c[a1]): the grid read in
  // that order.  A site starts a run when its predecessor along a0 is not fluid.
  L.st2ref.resize(n);
  L.ref2st.resize(nt);
  for (int x = n; x < nt; x++) L.ref2st[x] = x;  // halo sites keep their order after the owned ones
  std::vector<int> run_of(n);
  {
    const int64_t R = D[a2] * D[a1];  // rows
    std::vector<int64_t> row_count(R + 1, 0);
    auto cell = [&](int64_t row, int64_t k) {
      int64_t c[3];
      c[a2] = row / D[a1];
      c[a1] = row % D[a1];
      c[a0] = k;
      const int32_t g = grid[gidx(c[0], c[1], c[2])];
      return g < n ? g : -1;
    };
    parallel_for(R, [&](int64_t b, int64_t e) {
      for (int64_t row = b; row < e; row++) {
        int64_t m = 0;
        for (int64_t k = 0; k < D[a0]; k++) m += cell(row, k) >= 0;
        row_count[row + 1] = m;
      }
    });
    for (int64_t row = 0; row < R; row++) row_count[row + 1] += row_count[row];
    parallel_for(R, [&](int64_t b, int64_t e) {
      for (int64_t row = b; row < e; row++) {
        int64_t sidx = row_count[row];
        for (int64_t k = 0; k < D[a0]; k++) {
          const int32_t x = cell(row, k);
          if (x < 0) continue;
          L.st2ref[sidx] = x;
          L.ref2st[x] = (int)sidx;
          run_of[sidx] = (k == 0 || cell(row, k - 1) < 0) ? 1 : 0;  // run start flag, numbered below
          sidx++;
        }
      }
    });
  }
  int runs = 0;
  std::vector<int> run_start;
  for (int s = 0; s < n; s++) {
    if (run_of[s]) {
      runs++;
      run_start.push_back(s);
    }
    run_of[s] = runs - 1;
  }
  run_start.push_back(n);
  L.runs = runs;

  // Slot writers from the push semantics.  src[s*19+i]: storage index of the
  // bulk source, -2 own boundary rule, -1 no writer yet.
  const size_t nslots = (size_t)n * Q;
  std::unique_ptr<int[]> src(new int[nslots]);           // filled in parallel: the first touch
  std::unique_ptr<uint8_t[]> writers(new uint8_t[nslots]);  // of these pages dominates otherwise
  parallel_for((int64_t)nslots, [&](int64_t b, int64_t e) {
    std::fill(src.get() + b, src.get() + e, -1);
    std::fill(writers.get() + b, writers.get() + e, (uint8_t)0);
  });
  parallel_for(nt, [&](int64_t b, int64_t e) {
    for (int64_t xx = b; xx < e; xx++) {
      const int x = (int)xx;
      const int ct = t.collision_type(x);
      const int sx = L.ref2st[x];
      const bool halo = x >= n;
      for (int d = 0; d < Q; d++) {
        const bool io = d > 0 && ct >= 2 && ((t.iolet[x] >> (d - 1)) & 1u);
        const bool wl = d > 0 && (ct == 1 || ct >= 4) && ((t.wall[x] >> (d - 1)) & 1u);
        if (io || wl) {
          if (halo) continue;  // a halo site's own delegates are the other shard's
          const size_t slot = (size_t)sx * Q + inv(d);
          __atomic_fetch_add(&writers[slot], (uint8_t)1, __ATOMIC_RELAXED);
          src[slot] = -2;
        } else {
          const int64_t target = neighbour(x, d);
          if (target == nt64 * Q) continue;  // the rubbish slot
          if (target < 0 || target > nt64 * Q || target % Q != d) {
            err.set(HB_ERR_BAD_INDEX, "neighbour index out of range or in the wrong direction");
            return;
          }
          const int y = (int)(target / Q);
          if (y >= n) continue;  // into a halo site: the other shard's slot
          const size_t slot = (size_t)L.ref2st[y] * Q + d;
          __atomic_fetch_add(&writers[slot], (uint8_t)1, __ATOMIC_RELAXED);
          src[slot] = sx;
        }
      }
    }
  });
  err.raise();
  parallel_for((int64_t)nslots, [&](int64_t b, int64_t e) {
    for (int64_t k = b; k < e; k++)
      if (writers[k] != 1) {
        err.set(HB_ERR_UNSUPPORTED, writers[k] == 0 ? "a distribution slot is never written in a step (inconsistent cut links)"
                                                    : "a distribution slot is written twice in a step (inconsistent cut links)");
        return;
      }
  });
  err.raise();

  // Run offsets, per direction: from the first site of the run whose slot is a
  // bulk pull.  A site follows its run when every bulk slot matches them.
  L.run_off.assign((size_t)runs * 20, 0);
  L.meta.assign(n, 0);
  std::vector<char> plain(n, 0), regular(n, 0);
  parallel_for(runs, [&](int64_t b, int64_t e) {
    for (int64_t r = b; r < e; r++) {
      int* off = &L.run_off[(size_t)r * 20];
      uint32_t set = 0;
      for (int s = run_start[r]; s < run_start[r + 1]; s++)
        for (int i = 1; i < Q; i++) {
          const int v = src[(size_t)s * Q + i];
          if (v >= 0 && v < n && !((set >> i) & 1u)) {
            off[i] = v - s;
            set |= 1u << i;
          }
        }
    }
  });
  parallel_for(n, [&](int64_t b, int64_t e) {
    for (int64_t ss = b; ss < e; ss++) {
      const int s = (int)ss;
      const int* off = &L.run_off[(size_t)run_of[s] * 20];
      bool ok = src[(size_t)s * Q] == s, all_bulk = true;
      for (int i = 1; i < Q; i++) {
        const int v = src[(size_t)s * Q + i];
        if (v < 0) all_bulk = false;
        else if (v >= n || v - s != off[i]) ok = false;  // pulls from a halo site follow no run
      }
      regular[s] = ok;
      plain[s] = ok && all_bulk && t.collision_type(L.st2ref[s]) == 0;
    }
  });

  // General sites, binned by collision type.
  std::vector<int> gl;
  {
    int64_t bin[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int s = 0; s < n; s++)
      if (!plain[s]) bin[t.collision_type(L.st2ref[s]) + 1]++;
    for (int k = 1; k < 7; k++) bin[k] += bin[k - 1];
    gl.resize(bin[6]);
    for (int s = 0; s < n; s++)
      if (!plain[s]) gl[bin[t.collision_type(L.st2ref[s])]++] = s;
  }
  const int G = (int)gl.size();
  L.G = G;
  L.bulk_sites = n - G;
  for (int s = 0; s < n; s++) L.meta[s] = plain[s] ? run_of[s] : 0;
  L.g_site.resize(G);
  L.g_run.resize(G);
  L.g_src.resize((size_t)18 * G);
  L.g_io.assign(G, -1);
  L.g_cpl.assign(G, -1);
  L.g_xyz.resize((size_t)3 * G);
  L.g_kind.resize(G);
  L.g_wall.resize(G);
  L.g_iolet.resize(G);
  L.g_q.assign((size_t)18 * G, 0.0f);
  L.g_nrm.assign((size_t)3 * G, 0.0f);

  for (int g = 0; g < G; g++) {
    const int s = gl[g];
    const int x = L.st2ref[s];
    L.meta[s] = -(g + 1);
    L.g_site[g] = s;
    L.g_run[g] = regular[s] ? run_of[s] : -1;
    const int ct = t.collision_type(x);
    L.g_kind[g] = ct;
    // Only the links the site's streamer sends to a delegate carry a rule.
    L.g_wall[g] = (ct == 1 || ct >= 4) ? t.wall[x] : 0u;
    L.g_iolet[g] = ct >= 2 ? t.iolet[x] : 0u;
    for (int i = 1; i < Q; i++) {
      const int v = src[(size_t)s * Q + i];
      L.g_src[(size_t)(i - 1) * G + g] = v >= 0 ? v : s;
    }
    for (int c = 0; c < 3; c++) L.g_xyz[(size_t)c * G + g] = (int)t.coords[3 * x + c];
    if (!t.q.empty())
      for (int d = 0; d < 18; d++) L.g_q[(size_t)d * G + g] = (float)t.q[(size_t)18 * x + d];
    if (!t.normal.empty())
      for (int c = 0; c < 3; c++) L.g_nrm[(size_t)c * G + g] = (float)t.normal[(size_t)3 * x + c];
    if (L.g_iolet[g]) {
      const int id = t.iolet_id[x];
      const int grp = t.stype[x] == 1 ? 0 : 1;
      const int cnt = grp == 0 ? p.n_inlets : p.n_outlets;
      if (id < 0 || id >= cnt) throw Error{HB_ERR_BAD_INDEX, "site refers to an iolet that the case does not define"};
      L.g_io[g] = grp * 16 + id;
    }
  }
  finish_layout(L, t, p, wall);
  return L;
}

void finish_layout(Layout& L, const LatticeTables& t, const hb_params& p, int wall) {
  const int n = L.n, G = L.G;
  L.g_cpl.assign(G, -1);
  L.regular_general = 0;
  for (int k = 0; k < 7; k++) L.kind_start[k] = 0;
  for (int g = 0; g < G; g++) {
    if (L.g_run[g] >= 0) L.regular_general++;
    L.kind_start[L.g_kind[g] + 1]++;
  }
  for (int k = 1; k < 7; k++) L.kind_start[k] += L.kind_start[k - 1];

  // The direction closest to each iolet normal.
  for (int k = 0; k < 32; k++) L.dir0[k] = 0;
  for (int k = 0; k < p.n_inlets; k++) L.dir0[k] = closest_direction(p.inlets[k].normal);
  for (int k = 0; k < p.n_outlets; k++) L.dir0[16 + k] = closest_direction(p.outlets[k].normal);
  auto iolet_cfg = [&](int idx) -> const hb_iolet& { return idx < 16 ? p.inlets[idx] : p.outlets[idx - 16]; };

  std::vector<std::vector<std::pair<int, int>>> cpl_sites(32);  // (ref index, g)
  for (int g = 0; g < G; g++) {
    const int x = L.st2ref[L.g_site[g]];
    if (L.g_iolet[g]) {
      const int idx = L.g_io[g];
      const int kind = iolet_cfg(idx).kind;
      if (kind == kWK3 || kind == kWK2) {
        bool couples = false;
        for (int d = 1; d < Q; d++)
          if (((L.g_iolet[g] >> (d - 1)) & 1u) && inv(d) == L.dir0[idx]) couples = true;
        if (couples) cpl_sites[idx].push_back({x, g});
      }
    }
    if (wall == kGZS && L.g_wall[g]) {
      // Slot d of a GZS wall link d with no rule behind it is pulled from the
      // fluid neighbour the virtual node extrapolates from; the slot writers
      // guarantee that neighbour exists, but it may be another shard's.
      for (int d = 1; d < Q; d++) {
        if (!((L.g_wall[g] >> (d - 1)) & 1u)) continue;
        const int i = inv(d);
        const bool bi = (L.g_iolet[g] >> (i - 1)) & 1u, bw = (L.g_wall[g] >> (i - 1)) & 1u;
        const float q = L.g_q[(size_t)(d - 1) * G + g];
        const int from = L.g_src[(size_t)(d - 1) * G + g];  // the site itself where no bulk pull fills the slot
        if (q < 0.75 && !bi && !bw && from == L.g_site[g])
          throw Error{HB_ERR_UNSUPPORTED, "GZS wall link without a fluid neighbour behind the site"};
        if (q < 0.75 && !bi && !bw && from >= n)
          throw Error{HB_ERR_UNSUPPORTED, "GZS wall link whose extrapolation neighbour lies in another shard"};
      }
    }
  }

  // Windkessel coupling slots in reference order, and the centre site
  // (BoundaryValues::IsIOletCentreOnThisProc, src/lb/iolets/BoundaryValues.cc:103-121).
  int slot = 0;
  L.couplings.clear();
  for (int idx = 0; idx < 32; idx++) {
    const int cnt = idx < 16 ? p.n_inlets : p.n_outlets;
    if ((idx % 16) >= cnt || (iolet_cfg(idx).kind != kWK3 && iolet_cfg(idx).kind != kWK2)) continue;
    auto& v = cpl_sites[idx];
    std::sort(v.begin(), v.end());
    Layout::Coupling c;
    c.iolet = idx;
    c.start = slot;
    c.count = (int)v.size();
    for (auto& pr : v) L.g_cpl[pr.second] = slot++;
    const hb_iolet& io = iolet_cfg(idx);
    for (int i = 0; i < n; i++) {  // owned sites only: a shard holds its own centre or none
      bool in = true;
      for (int k = 0; k < 3; k++) {
        const double cc = (double)t.coords[3 * i + k];
        if (!(cc >= io.position[k] - 1.0 && cc <= io.position[k] + 1.0)) in = false;
      }
      if (in) {
        c.centre_ref = i;
        break;
      }
    }
    for (auto& pr : v)
      if (pr.first == c.centre_ref) c.centre_couples = true;
    L.couplings.push_back(c);
  }
  L.cpl_total = slot;
}

namespace {
uint64_t fnv1a(const void* data, size_t bytes, uint64_t h = 1469598103934665603ull) {
  const unsigned char* b = static_cast<const unsigned char*>(data);
  for (size_t k = 0; k < bytes; k++) {
    h ^= b[k];
    h *= 1099511628211ull;
  }
  return h;
}
template <class T>
uint64_t fnv_vec(const std::vector<T>& v) {
  const size_t count = v.size();
  return fnv1a(v.data(), count * sizeof(T), fnv1a(&count, sizeof(count)));
}
}  // namespace

void layout_digest(const Layout& L, uint64_t out[32]) {
  for (int k = 0; k < 32; k++) out[k] = 0;
  const int64_t sc[] = {L.n, L.n_halo, L.np, L.axis, L.runs, L.bulk_sites, L.G, L.regular_general, L.cpl_total};
  uint64_t h = fnv1a(sc, sizeof(sc));
  h = fnv1a(L.kind_start, sizeof(L.kind_start), h);
  out[0] = fnv1a(L.dir0, sizeof(L.dir0), h);
  out[1] = fnv_vec(L.st2ref);
  out[2] = fnv_vec(L.ref2st);
  out[3] = fnv_vec(L.meta);
  out[4] = fnv_vec(L.run_off);
  out[5] = fnv_vec(L.g_site);
  out[6] = fnv_vec(L.g_run);
  out[7] = fnv_vec(L.g_src);
  out[8] = fnv_vec(L.g_io);
  out[9] = fnv_vec(L.g_cpl);
  out[10] = fnv_vec(L.g_xyz);
  out[11] = fnv_vec(L.g_kind);
  out[12] = fnv_vec(L.g_wall);
  out[13] = fnv_vec(L.g_iolet);
  out[14] = fnv_vec(L.g_q);
  out[15] = fnv_vec(L.g_nrm);
  uint64_t c = fnv1a(nullptr, 0);
  for (const auto& cp : L.couplings) {
    const int64_t v[] = {cp.iolet, cp.start, cp.count, cp.centre_ref, cp.centre_couples ? 1 : 0};
    c = fnv1a(v, sizeof(v), c);
  }
  out[16] = c;
}

}  // namespace hb
