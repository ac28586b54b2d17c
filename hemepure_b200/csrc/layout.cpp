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
#include <cmath>
#include <cstring>
#include <numeric>

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

Layout build_layout(const LatticeTables& t, const hb_params& p, int wall) {
  Layout L;
  const int64_t n64 = t.n;
  if (n64 <= 0) throw Error{HB_ERR_ARG, "lattice has no fluid sites"};
  if (n64 > (int64_t)1 << 30) throw Error{HB_ERR_UNSUPPORTED, "more than 2^30 sites in one lattice"};
  const int n = (int)n64;
  L.n = n;
  L.np = ((n64 + 63) / 64) * 64;
  const int64_t D[3] = {t.dims[0], t.dims[1], t.dims[2]};

  // Dense grid of reference indices.
  std::vector<int32_t> grid(D[0] * D[1] * D[2], -1);
  auto gidx = [&](int64_t x, int64_t y, int64_t z) { return (x * D[1] + y) * D[2] + z; };
  for (int i = 0; i < n; i++) grid[gidx(t.coords[3 * i], t.coords[3 * i + 1], t.coords[3 * i + 2])] = i;

  // Run axis: fewest sites whose predecessor along the axis is not fluid.
  int64_t best_runs = -1;
  for (int a = 0; a < 3; a++) {
    int64_t runs = 0;
    for (int i = 0; i < n; i++) {
      int64_t c[3] = {t.coords[3 * i], t.coords[3 * i + 1], t.coords[3 * i + 2]};
      c[a] -= 1;
      if (c[a] < 0 || grid[gidx(c[0], c[1], c[2])] < 0) runs++;
    }
    if (best_runs < 0 || runs < best_runs) {
      best_runs = runs;
      L.axis = a;
    }
  }
  const int a0 = L.axis, a1 = (a0 + 1) % 3, a2 = (a0 + 2) % 3;

  // Storage order.
  std::vector<int64_t> key(n);
  for (int i = 0; i < n; i++) {
    const int64_t* c = &t.coords[3 * i];
    key[i] = (c[a2] * D[a1] + c[a1]) * D[a0] + c[a0];
  }
  L.st2ref.resize(n);
  std::iota(L.st2ref.begin(), L.st2ref.end(), 0);
  std::sort(L.st2ref.begin(), L.st2ref.end(), [&](int x, int y) { return key[x] < key[y]; });
  L.ref2st.resize(n);
  for (int s = 0; s < n; s++) L.ref2st[L.st2ref[s]] = s;

  // Runs.
  std::vector<int> run_of(n);
  int runs = 0;
  for (int s = 0; s < n; s++) {
    if (s == 0 || key[L.st2ref[s]] != key[L.st2ref[s - 1]] + 1) runs++;
    run_of[s] = runs - 1;
  }
  L.runs = runs;

  // Slot writers from the push semantics.  src[s*19+i]: storage index of the
  // bulk source, -2 own boundary rule, -1 no writer yet.
  std::vector<int> src((size_t)n * Q, -1);
  std::vector<uint8_t> writers((size_t)n * Q, 0);
  for (int x = 0; x < n; x++) {
    const int ct = t.collision_type(x);
    const int sx = L.ref2st[x];
    for (int d = 0; d < Q; d++) {
      const bool io = d > 0 && ct >= 2 && ((t.iolet[x] >> (d - 1)) & 1u);
      const bool wl = d > 0 && (ct == 1 || ct >= 4) && ((t.wall[x] >> (d - 1)) & 1u);
      if (io || wl) {
        const size_t slot = (size_t)sx * Q + inv(d);
        writers[slot]++;
        src[slot] = -2;
      } else {
        const int64_t target = t.nbr[(size_t)x * Q + d];
        if (target == n64 * Q) continue;  // the rubbish slot
        if (target < 0 || target > n64 * Q || target % Q != d)
          throw Error{HB_ERR_BAD_INDEX, "neighbour index out of range or in the wrong direction"};
        const int y = (int)(target / Q);
        const size_t slot = (size_t)L.ref2st[y] * Q + d;
        writers[slot]++;
        src[slot] = sx;
      }
    }
  }
  for (size_t k = 0; k < writers.size(); k++) {
    if (writers[k] != 1)
      throw Error{HB_ERR_UNSUPPORTED, writers[k] == 0 ? "a distribution slot is never written in a step (inconsistent cut links)"
                                                      : "a distribution slot is written twice in a step (inconsistent cut links)"};
  }

  // Run offsets, per direction: from the first site of the run whose slot is a
  // bulk pull.  A site follows its run when every bulk slot matches them.
  L.run_off.assign((size_t)runs * 20, 0);
  std::vector<uint32_t> run_set(runs, 0u);
  L.meta.assign(n, 0);
  std::vector<char> plain(n, 0), regular(n, 0);
  for (int s = 0; s < n; s++) {
    const int r = run_of[s];
    int* off = &L.run_off[(size_t)r * 20];
    for (int i = 1; i < Q; i++) {
      const int v = src[(size_t)s * Q + i];
      if (v >= 0 && !((run_set[r] >> i) & 1u)) {
        off[i] = v - s;
        run_set[r] |= 1u << i;
      }
    }
  }
  for (int s = 0; s < n; s++) {
    const int r = run_of[s];
    const int* off = &L.run_off[(size_t)r * 20];
    bool ok = src[(size_t)s * Q] == s, all_bulk = true;
    for (int i = 1; i < Q; i++) {
      const int v = src[(size_t)s * Q + i];
      if (v < 0) all_bulk = false;
      else if (v - s != off[i]) ok = false;
    }
    regular[s] = ok;
    plain[s] = ok && all_bulk && t.collision_type(L.st2ref[s]) == 0;
  }

  // General sites, binned by collision type.
  std::vector<int> gl;
  for (int s = 0; s < n; s++)
    if (!plain[s]) gl.push_back(s);
  std::stable_sort(gl.begin(), gl.end(), [&](int u, int v) { return t.collision_type(L.st2ref[u]) < t.collision_type(L.st2ref[v]); });
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
  for (int k = 0; k < 7; k++) L.kind_start[k] = 0;

  // Iolet table index and the direction closest to each normal.
  for (int k = 0; k < 32; k++) L.dir0[k] = 0;
  for (int k = 0; k < p.n_inlets; k++) L.dir0[k] = closest_direction(p.inlets[k].normal);
  for (int k = 0; k < p.n_outlets; k++) L.dir0[16 + k] = closest_direction(p.outlets[k].normal);
  auto iolet_cfg = [&](int idx) -> const hb_iolet& { return idx < 16 ? p.inlets[idx] : p.outlets[idx - 16]; };

  std::vector<std::vector<std::pair<int, int>>> cpl_sites(32);  // (ref index, g)
  for (int g = 0; g < G; g++) {
    const int s = gl[g];
    const int x = L.st2ref[s];
    L.meta[s] = -(g + 1);
    L.g_site[g] = s;
    L.g_run[g] = regular[s] ? run_of[s] : -1;
    if (regular[s]) L.regular_general++;
    const int ct = t.collision_type(x);
    L.g_kind[g] = ct;
    L.kind_start[ct + 1]++;
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
      const int idx = grp * 16 + id;
      L.g_io[g] = idx;
      const int kind = iolet_cfg(idx).kind;
      if (kind == kWK3 || kind == kWK2) {
        bool couples = false;
        for (int d = 1; d < Q; d++)
          if (((L.g_iolet[g] >> (d - 1)) & 1u) && inv(d) == L.dir0[idx]) couples = true;
        if (couples) cpl_sites[idx].push_back({x, g});
      }
    }
    if (wall == kGZS && L.g_wall[g]) {
      for (int d = 1; d < Q; d++) {
        if (!((L.g_wall[g] >> (d - 1)) & 1u)) continue;
        const int i = inv(d);
        const bool bi = (L.g_iolet[g] >> (i - 1)) & 1u, bw = (L.g_wall[g] >> (i - 1)) & 1u;
        const double q = t.q[(size_t)18 * x + d - 1];
        if (q < 0.75 && !bi && !bw && src[(size_t)s * Q + d] < 0)
          throw Error{HB_ERR_UNSUPPORTED, "GZS wall link without a fluid neighbour behind the site"};
      }
    }
  }
  for (int k = 1; k < 7; k++) L.kind_start[k] += L.kind_start[k - 1];

  // Windkessel coupling slots in reference order, and the centre site
  // (BoundaryValues::IsIOletCentreOnThisProc, src/lb/iolets/BoundaryValues.cc:103-121).
  int slot = 0;
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
    for (int i = 0; i < n; i++) {
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
  return L;
}

}  // namespace hb
