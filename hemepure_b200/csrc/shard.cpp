// shard.cpp -- slab plan, shard tables and halo lists of the sharded form (shard.h).
#include "shard.h"

#include <algorithm>
#include <unordered_map>

namespace hb {

namespace {

// The streamer of a site's collision type sends link d to a delegate
// (iolet or wall) instead of pushing it to the neighbour (the same rule as the
// layout's slot writers, src/lb/streamers/StreamerTypeFactory.h:47-300).
bool link_to_delegate(const LatticeTables& t, int64_t x, int d) {
  const int ct = t.collision_type(x);
  const bool io = ct >= 2 && ((t.iolet[x] >> (d - 1)) & 1u);
  const bool wl = (ct == 1 || ct >= 4) && ((t.wall[x] >> (d - 1)) & 1u);
  return io || wl;
}

int c_of(int d, int axis) { return axis == 0 ? cx(d) : (axis == 1 ? cy(d) : cz(d)); }

}  // namespace

std::vector<int64_t> plan_slabs(const LatticeTables& t, int n_shards, int* axis) {
  if (n_shards < 1) throw Error{HB_ERR_ARG, "at least one shard"};
  if (t.n <= 0) throw Error{HB_ERR_ARG, "lattice has no fluid sites"};
  int64_t lo[3], hi[3];
  for (int a = 0; a < 3; a++) {
    lo[a] = t.coords[a];
    hi[a] = t.coords[a];
  }
  for (int64_t i = 0; i < t.n; i++)
    for (int a = 0; a < 3; a++) {
      lo[a] = std::min(lo[a], t.coords[3 * i + a]);
      hi[a] = std::max(hi[a], t.coords[3 * i + a]);
    }
  int a = *axis;
  if (a < 0) {
    a = 0;
    for (int k = 1; k < 3; k++)
      if (hi[k] - lo[k] > hi[a] - lo[a]) a = k;
  }
  if (a > 2) throw Error{HB_ERR_ARG, "axis must be 0, 1 or 2"};
  *axis = a;
  const int64_t planes = hi[a] - lo[a] + 1;
  if (planes < n_shards) throw Error{HB_ERR_ARG, "more shards than lattice planes along the axis"};
  std::vector<int64_t> count(planes + 1, 0);
  for (int64_t i = 0; i < t.n; i++) count[t.coords[3 * i + a] - lo[a] + 1]++;
  for (int64_t k = 0; k < planes; k++) count[k + 1] += count[k];
  std::vector<int64_t> b(n_shards + 1);
  b[0] = lo[a];
  b[n_shards] = hi[a] + 1;
  for (int k = 1; k < n_shards; k++) {
    const int64_t target = (t.n * k + n_shards / 2) / n_shards;
    int64_t c = 0;
    while (c < planes && count[c] < target) c++;  // first plane boundary with >= target sites below
    c = std::max<int64_t>(c, b[k - 1] - lo[a] + 1);
    c = std::min<int64_t>(c, planes - (n_shards - k));
    b[k] = lo[a] + c;
  }
  return b;
}

LatticeTables cut_shard(const LatticeTables& full, const hb_params& p, int axis, int64_t lo, int64_t hi) {
  if (axis < 0 || axis > 2 || !(lo < hi)) throw Error{HB_ERR_ARG, "shard: axis 0..2 and lo < hi"};
  const int64_t n = full.n;
  std::vector<int64_t> owned, halo;
  for (int64_t x = 0; x < n; x++) {
    const int64_t c = full.coords[3 * x + axis];
    if (c >= lo && c < hi) owned.push_back(x);
    else if (c == lo - 1 || c == hi) halo.push_back(x);
  }
  if (owned.empty()) throw Error{HB_ERR_ARG, "shard owns no fluid site"};

  // Windkessel iolets: their sites and their centre site in one shard.
  for (int grp = 0; grp < 2; grp++) {
    const int cnt = grp == 0 ? p.n_inlets : p.n_outlets;
    for (int k = 0; k < cnt; k++) {
      const hb_iolet& io = grp == 0 ? p.inlets[k] : p.outlets[k];
      if (io.kind != kWK3 && io.kind != kWK2) continue;
      int64_t in = 0, out = 0;
      for (int64_t x = 0; x < n; x++) {
        if (full.stype[x] != grp + 1 || full.iolet_id[x] != k) continue;
        const int64_t c = full.coords[3 * x + axis];
        (c >= lo && c < hi ? in : out)++;
      }
      int64_t centre = -1;
      for (int64_t x = 0; x < n && centre < 0; x++) {
        bool inside = true;
        for (int d = 0; d < 3; d++) {
          const double cc = (double)full.coords[3 * x + d];
          if (!(cc >= io.position[d] - 1.0 && cc <= io.position[d] + 1.0)) inside = false;
        }
        if (inside) centre = x;
      }
      const bool centre_here = centre >= 0 && full.coords[3 * centre + axis] >= lo && full.coords[3 * centre + axis] < hi;
      if ((in > 0 && out > 0) || (in > 0 && centre >= 0 && !centre_here) || (in == 0 && centre_here && out > 0))
        throw Error{HB_ERR_UNSUPPORTED, "a Windkessel iolet's sites or centre site span two shards"};
    }
  }

  LatticeTables t;
  const int64_t no = (int64_t)owned.size(), nt = no + (int64_t)halo.size();
  t.n = nt;
  t.n_owned = no;
  for (int d = 0; d < 3; d++) {
    t.dims[d] = full.dims[d];
    t.blocks[d] = full.blocks[d];
  }
  t.block_size = full.block_size;
  t.gid.resize(nt);
  std::vector<int64_t> map(n, -1);
  for (int64_t k = 0; k < no; k++) t.gid[k] = owned[k];
  for (int64_t k = 0; k < (int64_t)halo.size(); k++) t.gid[no + k] = halo[k];
  for (int64_t k = 0; k < nt; k++) map[t.gid[k]] = k;
  t.coords.resize(3 * nt);
  t.wall.resize(nt);
  t.iolet.resize(nt);
  t.stype.resize(nt);
  t.iolet_id.resize(nt);
  if (!full.q.empty()) t.q.resize(18 * nt);
  if (!full.normal.empty()) t.normal.resize(3 * nt);
  for (int64_t k = 0; k < nt; k++) {
    const int64_t x = t.gid[k];
    for (int d = 0; d < 3; d++) t.coords[3 * k + d] = full.coords[3 * x + d];
    t.wall[k] = full.wall[x];
    t.iolet[k] = full.iolet[x];
    t.stype[k] = full.stype[x];
    t.iolet_id[k] = full.iolet_id[x];
    if (!full.q.empty()) std::copy(&full.q[18 * x], &full.q[18 * x] + 18, &t.q[18 * k]);
    if (!full.normal.empty()) std::copy(&full.normal[3 * x], &full.normal[3 * x] + 3, &t.normal[3 * k]);
  }
  if (!full.nbr.empty()) {
    t.nbr.resize((size_t)nt * Q);
    for (int64_t k = 0; k < nt; k++)
      for (int d = 0; d < Q; d++) {
        const int64_t g = full.nbr[(size_t)t.gid[k] * Q + d];
        const int64_t y = g / Q;
        t.nbr[(size_t)k * Q + d] = (g >= n * Q || map[y] < 0) ? nt * Q : map[y] * Q + d;
      }
  }
  for (int64_t k = 0; k < no; k++) t.type_counts[t.collision_type(k)]++;
  return t;
}

HaloLists halo_lists(const LatticeTables& t, const Layout& L, int axis, int64_t lo, int64_t hi) {
  const int64_t n = L.n, nt = t.n, np = L.np;
  struct Item {
    int64_t gid;
    int dir;
    int64_t elem;
  };
  std::vector<Item> send[2], recv[2];

  // Received: every pull of an owned general record from a halo site.
  const int G = L.G;
  for (int g = 0; g < G; g++)
    for (int i = 1; i < Q; i++) {
      const int64_t v = L.g_src[(size_t)(i - 1) * G + g];
      if (v < n) continue;
      const int64_t x = v;  // halo sites keep their index as their storage index
      const int side = t.coords[3 * x + axis] < lo ? 0 : 1;
      recv[side].push_back({t.gid[x], i, (int64_t)i * np + v});
    }

  // Sent: the pushes of owned sites next to a cut into the halo planes.
  const int64_t D1 = t.dims[1], D2 = t.dims[2];
  auto key = [&](int64_t a, int64_t b, int64_t c) { return (a * D1 + b) * D2 + c; };
  std::unordered_map<int64_t, int64_t> halo_at;
  halo_at.reserve((size_t)(nt - n) * 2 + 1);
  for (int64_t x = n; x < nt; x++) halo_at[key(t.coords[3 * x], t.coords[3 * x + 1], t.coords[3 * x + 2])] = x;
  for (int64_t x = 0; x < n; x++) {
    const int64_t c = t.coords[3 * x + axis];
    for (int side = 0; side < 2; side++) {
      if ((side == 0 && c != lo) || (side == 1 && c != hi - 1)) continue;
      for (int i = 1; i < Q; i++) {
        if (c_of(i, axis) != (side == 0 ? -1 : 1) || link_to_delegate(t, x, i)) continue;
        bool lands = false;
        if (!t.nbr.empty()) {
          const int64_t g = t.nbr[(size_t)x * Q + i];
          lands = g < nt * Q && g / Q >= n;
        } else {
          lands = halo_at.count(key(t.coords[3 * x] + cx(i), t.coords[3 * x + 1] + cy(i), t.coords[3 * x + 2] + cz(i))) != 0;
        }
        if (lands) send[side].push_back({t.gid[x], i, (int64_t)i * np + L.ref2st[x]});
      }
    }
  }

  HaloLists h;
  auto emit = [](std::vector<Item>& v, std::vector<int64_t>& elem, std::vector<int64_t>& pairs) {
    std::sort(v.begin(), v.end(), [](const Item& a, const Item& b) { return a.gid != b.gid ? a.gid < b.gid : a.dir < b.dir; });
    elem.resize(v.size());
    pairs.resize(2 * v.size());
    for (size_t k = 0; k < v.size(); k++) {
      elem[k] = v[k].elem;
      pairs[2 * k] = v[k].gid;
      pairs[2 * k + 1] = v[k].dir;
    }
  };
  for (int side = 0; side < 2; side++) {
    emit(send[side], h.send[side], h.send_pairs[side]);
    emit(recv[side], h.recv[side], h.recv_pairs[side]);
  }
  return h;
}

}  // namespace hb
