// layout_device.cu -- the storage layout (layout.cpp) built on the GPU.
//
// The passes are those of build_layout, one kernel each, on the lattice tables
// already resident on the device (the device .gmy reader leaves them there):
//   a dense grid of site indices over the lattice box (two sites at one point
//   or a site outside the box is an error);
//   the run axis: for each axis the sites whose predecessor along it is not a
//   fluid site, the axis with the fewest wins (the first on a tie);
//   the storage order: rows along the run axis ordered by the other two
//   coordinates, a row's sites in order, and the runs (maximal segments);
//   the slot writers from the reference's push semantics
//   (src/lb/streamers/StreamerTypeFactory.h:47-300; LatticeData::
//   InitialiseNeighbourLookup, src/geometry/LatticeData.cc:366-443): each slot
//   of each site must have exactly one writer;
//   the run offsets (from the first site of a run whose slot is a bulk pull),
//   the plain/general classification, and the general records binned by
//   collision type in storage order.
// Every result equals the host passes' bit for bit (integer work only); the
// Windkessel couplings and centre sites, which touch a few sites, are left to
// finish_layout on the host.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "hb_common.h"
#include "layout.h"
#include "setup_pool.h"

namespace hb {
namespace {

constexpr int kT = 256;

// First error of a pass: code, then the site it was found at.
enum : int { kLayoutErrOutside = 1, kLayoutErrTwice, kLayoutErrNoWriter, kLayoutErrTwoWriters, kLayoutErrIolet };

struct LayoutDevArgs {
  int64_t n, nt;  // owned sites, all sites (owned, then halo)
  int64_t dims[3];
  const int64_t* coords;
  const uint32_t* wall;
  const uint32_t* iolet;
  const int32_t* stype;
  const int32_t* iolet_id;
  const float* q;       // may be null
  const float* normal;  // may be null
  int n_inlets, n_outlets;
};

// The general records, structure of arrays (Layout's g_* fields).
struct LayoutRecordsDev {
  int32_t *site, *run, *kind;
  uint32_t *wall, *iolet;
  int32_t *src, *xyz;
  float *q, *nrm;
  int32_t* io;
};

__device__ __forceinline__ int64_t gidx(const LayoutDevArgs& a, int64_t x, int64_t y, int64_t z) {
  return (x * a.dims[1] + y) * a.dims[2] + z;
}

__device__ __forceinline__ void set_err(int* err, int code, int where) {
  if (atomicCAS(err, 0, code) == 0) err[1] = where;
}

__device__ __forceinline__ int collision_type(uint32_t wall, int32_t st) {
  const bool w = wall != 0;
  return !w ? (st == 0 ? 0 : (st == 1 ? 2 : 3)) : (st == 0 ? 1 : (st == 1 ? 4 : 5));
}

__global__ void k_fill_i32(int32_t* p, int64_t n, int32_t v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}

__global__ void k_grid(const LayoutDevArgs a, int32_t* grid, int* err) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= a.nt) return;
  const int64_t* c = a.coords + 3 * i;
  if (c[0] < 0 || c[1] < 0 || c[2] < 0 || c[0] >= a.dims[0] || c[1] >= a.dims[1] || c[2] >= a.dims[2]) {
    set_err(err, kLayoutErrOutside, (int)i);
    return;
  }
  if (atomicCAS(grid + gidx(a, c[0], c[1], c[2]), -1, (int32_t)i) != -1) set_err(err, kLayoutErrTwice, (int)i);
}

// Sites of the first n (owned) whose predecessor along each axis is not owned.
__global__ void k_axis_runs(const LayoutDevArgs a, const int32_t* grid, unsigned long long* counts) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int r[3] = {0, 0, 0};
  if (i < a.n) {
    const int64_t* c = a.coords + 3 * i;
    for (int ax = 0; ax < 3; ax++) {
      int64_t p[3] = {c[0], c[1], c[2]};
      p[ax] -= 1;
      bool owned = false;
      if (p[ax] >= 0) {
        const int32_t g = grid[gidx(a, p[0], p[1], p[2])];
        owned = g >= 0 && g < a.n;
      }
      r[ax] = owned ? 0 : 1;
    }
  }
  for (int ax = 0; ax < 3; ax++) {
    const int v = __reduce_add_sync(0xffffffffu, r[ax]);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(counts + ax, (unsigned long long)v);
  }
}

__device__ __forceinline__ int32_t cell(const LayoutDevArgs& a, const int32_t* grid, int a0, int a1, int a2, int64_t row,
                                        int64_t k) {
  int64_t c[3];
  c[a2] = row / a.dims[a1];
  c[a1] = row % a.dims[a1];
  c[a0] = k;
  const int32_t g = grid[gidx(a, c[0], c[1], c[2])];
  return g < a.n ? g : -1;
}

__global__ void k_row_count(const LayoutDevArgs a, const int32_t* grid, int a0, int a1, int a2, int64_t R, int64_t* rc) {
  const int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (row >= R) return;
  int64_t m = 0;
  for (int64_t k = 0; k < a.dims[a0]; k++) m += cell(a, grid, a0, a1, a2, row, k) >= 0;
  rc[row + 1] = m;
}

__global__ void k_row_place(const LayoutDevArgs a, const int32_t* grid, int a0, int a1, int a2, int64_t R,
                            const int64_t* row_start, int32_t* st2ref, int32_t* ref2st, int32_t* start_flag) {
  const int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (row >= R) return;
  int64_t s = row_start[row];
  int32_t prev = -1;
  for (int64_t k = 0; k < a.dims[a0]; k++) {
    const int32_t x = cell(a, grid, a0, a1, a2, row, k);
    if (x >= 0) {
      st2ref[s] = x;
      ref2st[x] = (int32_t)s;
      start_flag[s] = (k == 0 || prev < 0) ? 1 : 0;
      s++;
    }
    prev = x;
  }
}

__global__ void k_halo_ref2st(int32_t* ref2st, int64_t n, int64_t nt) {
  const int64_t x = n + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (x < nt) ref2st[x] = (int32_t)x;
}

// Slot writers: src[s*19+i] = storage index of the bulk source, -2 for a slot a
// delegate of the site fills; writers counted per slot (one byte each, packed).
__global__ void k_writers(const LayoutDevArgs a, const int32_t* grid, const int32_t* ref2st, int32_t* src,
                          uint32_t* writers, int* err) {
  const int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (x >= a.nt) return;
  const int ct = collision_type(a.wall[x], a.stype[x]);
  const int32_t sx = ref2st[x];
  const bool halo = x >= a.n;
  const int64_t* c = a.coords + 3 * x;
  for (int d = 0; d < Q; d++) {
    const bool io = d > 0 && ct >= 2 && ((a.iolet[x] >> (d - 1)) & 1u);
    const bool wl = d > 0 && (ct == 1 || ct >= 4) && ((a.wall[x] >> (d - 1)) & 1u);
    int64_t slot;
    int32_t v;
    if (io || wl) {
      if (halo) continue;
      slot = (int64_t)sx * Q + inv(d);
      v = -2;
    } else {
      const int64_t px = c[0] + cx(d), py = c[1] + cy(d), pz = c[2] + cz(d);
      if (px < 0 || py < 0 || pz < 0 || px >= a.dims[0] || py >= a.dims[1] || pz >= a.dims[2]) continue;
      const int32_t y = grid[gidx(a, px, py, pz)];
      if (y < 0 || y >= a.n) continue;  // solid, or a halo site (another shard's slot)
      slot = (int64_t)ref2st[y] * Q + d;
      v = sx;
    }
    atomicAdd(writers + (slot >> 2), 1u << (8 * (slot & 3)));
    src[slot] = v;
  }
}

__global__ void k_check_writers(const uint32_t* writers, int64_t nslots, int* err) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= nslots) return;
  const uint32_t w = (writers[k >> 2] >> (8 * (k & 3))) & 0xffu;
  if (w == 0) set_err(err, kLayoutErrNoWriter, (int)(k / Q));
  else if (w != 1) set_err(err, kLayoutErrTwoWriters, (int)(k / Q));
}

// One thread per (run, direction): the first site of the run whose slot is a
// bulk pull from an owned site sets the offset.
__global__ void k_run_offsets(const int32_t* src, const int32_t* run_start, int runs, int64_t n, int32_t* run_off) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)runs * 19) return;
  const int r = (int)(t / 19), i = (int)(t % 19);
  if (i == 0) return;  // entry 0 (and the spare 19) stay 0
  for (int32_t s = run_start[r]; s < run_start[r + 1]; s++) {
    const int32_t v = src[(int64_t)s * Q + i];
    if (v >= 0 && v < n) {
      run_off[(int64_t)r * 20 + i] = v - s;
      return;
    }
  }
}

__global__ void k_classify(const LayoutDevArgs a, const int32_t* src, const int32_t* run_of, const int32_t* run_off,
                           const int32_t* st2ref, uint8_t* regular, int32_t* kind) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  const int32_t* off = run_off + (int64_t)run_of[s] * 20;
  bool ok = src[s * Q] == s, all_bulk = true;
  for (int i = 1; i < Q; i++) {
    const int32_t v = src[s * Q + i];
    if (v < 0) all_bulk = false;
    else if (v >= a.n || v - (int32_t)s != off[i]) ok = false;
  }
  regular[s] = ok;
  const int32_t x = st2ref[s];
  const int ct = collision_type(a.wall[x], a.stype[x]);
  const bool plain = ok && all_bulk && ct == 0;
  kind[s] = plain ? -1 : ct;  // -1 plain bulk, else the general record's bin
}

// Stable partition of the general sites by bin: per-block counts per bin...
__global__ void k_bin_counts(const int32_t* kind, int64_t n, int32_t* counts /* [blocks][6] */) {
  __shared__ int32_t c[6];
  if (threadIdx.x < 6) c[threadIdx.x] = 0;
  __syncthreads();
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s < n && kind[s] >= 0) atomicAdd(&c[kind[s]], 1);
  __syncthreads();
  if (threadIdx.x < 6) counts[(int64_t)blockIdx.x * 6 + threadIdx.x] = c[threadIdx.x];
}

// ...then each block places its general sites of every bin in storage order:
// a site's rank among the block's sites of its bin is its rank within its warp
// (lanes with the same bin) plus the counts of the warps before it.
__global__ void __launch_bounds__(kT) k_bin_place(const int32_t* kind, int64_t n, const int64_t* base /* [blocks][6] */,
                                                  int32_t* gl) {
  __shared__ int32_t wc[kT / 32][6];
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int my = s < n ? kind[s] : -1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned same = __match_any_sync(0xffffffffu, my);
  const int rank = __popc(same & ((1u << lane) - 1u));
  if (threadIdx.x < (kT / 32) * 6) (&wc[0][0])[threadIdx.x] = 0;
  __syncthreads();
  if (my >= 0 && rank == 0) wc[warp][my] = __popc(same);
  __syncthreads();
  if (my < 0) return;
  int before = rank;
  for (int w = 0; w < warp; w++) before += wc[w][my];
  gl[base[(int64_t)blockIdx.x * 6 + my] + before] = (int32_t)s;
}

__global__ void k_records(const LayoutDevArgs a, const int32_t* gl, int G, const int32_t* st2ref, const uint8_t* regular,
                          const int32_t* run_of, const int32_t* src, LayoutRecordsDev r, int32_t* meta, int* err) {
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= G) return;
  const int32_t s = gl[g];
  const int32_t x = st2ref[s];
  meta[s] = -(int32_t)(g + 1);
  r.site[g] = s;
  r.run[g] = regular[s] ? run_of[s] : -1;
  const int ct = collision_type(a.wall[x], a.stype[x]);
  r.kind[g] = ct;
  const uint32_t wm = (ct == 1 || ct >= 4) ? a.wall[x] : 0u;
  const uint32_t im = ct >= 2 ? a.iolet[x] : 0u;
  r.wall[g] = wm;
  r.iolet[g] = im;
  for (int i = 1; i < Q; i++) {
    const int32_t v = src[(int64_t)s * Q + i];
    r.src[(int64_t)(i - 1) * G + g] = v >= 0 ? v : s;
  }
  for (int c = 0; c < 3; c++) r.xyz[(int64_t)c * G + g] = (int32_t)a.coords[3 * (int64_t)x + c];
  for (int d = 0; d < 18; d++) r.q[(int64_t)d * G + g] = a.q ? a.q[(int64_t)18 * x + d] : 0.0f;
  for (int c = 0; c < 3; c++) r.nrm[(int64_t)c * G + g] = a.normal ? a.normal[(int64_t)3 * x + c] : 0.0f;
  int io = -1;
  if (im) {
    const int id = a.iolet_id[x];
    const int grp = a.stype[x] == 1 ? 0 : 1;
    const int cnt = grp == 0 ? a.n_inlets : a.n_outlets;
    if (id < 0 || id >= cnt) set_err(err, kLayoutErrIolet, (int)x);
    else io = grp * 16 + id;
  }
  r.io[g] = io;
}

__global__ void k_meta_plain(const int32_t* kind, const int32_t* run_of, int64_t n, int32_t* meta) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s < n && kind[s] < 0) meta[s] = run_of[s];
}

unsigned nblk(int64_t n) { return (unsigned)((n + kT - 1) / kT); }

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error{HB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

template <class T>
void download(std::vector<T>& out, const T* src, size_t count, cudaStream_t st) {
  out.resize(count);
  if (count) check(cudaMemcpyAsync(out.data(), src, count * sizeof(T), cudaMemcpyDeviceToHost, st), "layout download");
}

void raise_pass_error(const int herr[2]) {
  switch (herr[0]) {
    case 0: return;
    case kLayoutErrOutside: throw Error{HB_ERR_BAD_INDEX, "site coordinates outside the lattice"};
    case kLayoutErrTwice: throw Error{HB_ERR_BAD_INDEX, "two sites share coordinates"};
    case kLayoutErrNoWriter:
      throw Error{HB_ERR_UNSUPPORTED, "a distribution slot is never written in a step (inconsistent cut links)"};
    case kLayoutErrTwoWriters:
      throw Error{HB_ERR_UNSUPPORTED, "a distribution slot is written twice in a step (inconsistent cut links)"};
    case kLayoutErrIolet: throw Error{HB_ERR_BAD_INDEX, "site refers to an iolet that the case does not define"};
    default: throw Error{HB_ERR_CUDA, "layout pass error"};
  }
}

}  // namespace

Layout layout_on_device(const DeviceTables& d, const hb_params& p, void* stream) {
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  LayoutDevArgs a;
  a.nt = d.n;
  a.n = d.n_owned >= 0 ? d.n_owned : d.n;
  for (int k = 0; k < 3; k++) a.dims[k] = d.dims[k];
  a.coords = d.coords;
  a.wall = d.wall;
  a.iolet = d.iolet;
  a.stype = d.stype;
  a.iolet_id = d.iolet_id;
  a.q = d.q;
  a.normal = d.normal;
  a.n_inlets = p.n_inlets;
  a.n_outlets = p.n_outlets;
  if (a.n <= 0) throw Error{HB_ERR_ARG, "lattice has no fluid sites"};
  if (a.nt > (int64_t)1 << 30) throw Error{HB_ERR_UNSUPPORTED, "more than 2^30 sites in one lattice"};
  const int64_t n = a.n, nt = a.nt;
  const int64_t* D = a.dims;
  Layout L;
  L.n = (int)n;
  L.n_halo = (int)(nt - n);
  L.np = ((nt + 63) / 64) * 64;

  int device = 0;
  check(cudaGetDevice(&device), "cudaGetDevice");
  SetupPool P(device, st);
  int* err = P.get<int>(2);
  int herr[2] = {0, 0};
  auto sync_and_check = [&](const char* what) {
    check(cudaMemcpyAsync(herr, err, sizeof(herr), cudaMemcpyDeviceToHost, st), what);
    check(cudaStreamSynchronize(st), what);
    raise_pass_error(herr);
  };
  check(cudaMemsetAsync(err, 0, 2 * sizeof(int), st), "cudaMemset");

  // Dense grid of reference indices.
  const int64_t cells = D[0] * D[1] * D[2];
  int32_t* grid = P.get<int32_t>(cells);
  k_fill_i32<<<1184, kT, 0, st>>>(grid, cells, -1);
  k_grid<<<nblk(nt), kT, 0, st>>>(a, grid, err);
  check(cudaGetLastError(), "k_grid launch");
  sync_and_check("layout grid");  // every site inside the box, once, before the grid is read

  // Run axis: fewest owned sites whose predecessor along it is not owned (first on a tie).
  unsigned long long* axis_runs = P.get<unsigned long long>(3);
  check(cudaMemsetAsync(axis_runs, 0, 3 * sizeof(unsigned long long), st), "cudaMemset");
  k_axis_runs<<<nblk(n), kT, 0, st>>>(a, grid, axis_runs);
  unsigned long long hr[3];
  check(cudaMemcpyAsync(hr, axis_runs, sizeof(hr), cudaMemcpyDeviceToHost, st), "axis runs");
  check(cudaStreamSynchronize(st), "axis runs");
  L.axis = 0;
  for (int k = 1; k < 3; k++)
    if (hr[k] < hr[L.axis]) L.axis = k;
  const int a0 = L.axis, a1 = (a0 + 1) % 3, a2 = (a0 + 2) % 3;

  // Storage order: rows along a0 in (c[a2], c[a1]) order.
  const int64_t R = D[a2] * D[a1];
  int64_t* row_start = P.get<int64_t>(R + 1);
  check(cudaMemsetAsync(row_start, 0, sizeof(int64_t), st), "cudaMemset");
  k_row_count<<<nblk(R), kT, 0, st>>>(a, grid, a0, a1, a2, R, row_start);
  std::vector<int64_t> rc;
  download(rc, row_start, (size_t)R + 1, st);
  check(cudaStreamSynchronize(st), "row counts");
  for (int64_t r = 0; r < R; r++) rc[r + 1] += rc[r];
  check(cudaMemcpyAsync(row_start, rc.data(), rc.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st), "row starts");
  int32_t* st2ref = P.get<int32_t>(n);
  int32_t* ref2st = P.get<int32_t>(nt);
  int32_t* run_of = P.get<int32_t>(n);  // run start flags, then run numbers
  k_row_place<<<nblk(R), kT, 0, st>>>(a, grid, a0, a1, a2, R, row_start, st2ref, ref2st, run_of);
  if (nt > n) k_halo_ref2st<<<nblk(nt - n), kT, 0, st>>>(ref2st, n, nt);
  check(cudaGetLastError(), "k_row_place launch");

  // Runs numbered in storage order (on the host: one pass over the flags).
  std::vector<int32_t> flags;
  download(flags, run_of, (size_t)n, st);
  check(cudaStreamSynchronize(st), "run flags");
  std::vector<int32_t> run_start;
  int runs = 0;
  for (int64_t s = 0; s < n; s++) {
    if (flags[s]) {
      runs++;
      run_start.push_back((int32_t)s);
    }
    flags[s] = runs - 1;
  }
  run_start.push_back((int32_t)n);
  L.runs = runs;
  int32_t* d_run_start = P.get<int32_t>(run_start.size());
  check(cudaMemcpyAsync(run_of, flags.data(), (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, st), "run numbers");
  check(cudaMemcpyAsync(d_run_start, run_start.data(), run_start.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st),
        "run starts");

  // Slot writers and sources.
  const int64_t nslots = n * Q;
  int32_t* src = P.get<int32_t>(nslots);
  uint32_t* writers = P.get<uint32_t>((nslots + 3) / 4);
  k_fill_i32<<<1184, kT, 0, st>>>(src, nslots, -1);
  check(cudaMemsetAsync(writers, 0, (size_t)((nslots + 3) / 4) * sizeof(uint32_t), st), "cudaMemset");
  k_writers<<<nblk(nt), kT, 0, st>>>(a, grid, ref2st, src, writers, err);
  k_check_writers<<<nblk(nslots), kT, 0, st>>>(writers, nslots, err);
  check(cudaGetLastError(), "k_writers launch");

  // Run offsets, classification, bins.
  int32_t* run_off = P.get<int32_t>((size_t)runs * 20);
  check(cudaMemsetAsync(run_off, 0, (size_t)runs * 20 * sizeof(int32_t), st), "cudaMemset");
  k_run_offsets<<<nblk((int64_t)runs * 19), kT, 0, st>>>(src, d_run_start, runs, n, run_off);
  uint8_t* regular = P.get<uint8_t>(n);
  int32_t* kind = P.get<int32_t>(n);
  const unsigned nbk = nblk(n);
  int32_t* bin_counts = P.get<int32_t>((size_t)nbk * 6);
  k_classify<<<nbk, kT, 0, st>>>(a, src, run_of, run_off, st2ref, regular, kind);
  k_bin_counts<<<nbk, kT, 0, st>>>(kind, n, bin_counts);
  check(cudaGetLastError(), "k_classify launch");
  std::vector<int32_t> bc;
  download(bc, bin_counts, (size_t)nbk * 6, st);
  sync_and_check("layout writers");
  std::vector<int64_t> base((size_t)nbk * 6);
  {
    int64_t start[6], total = 0;
    for (int k = 0; k < 6; k++) {
      start[k] = total;
      for (unsigned b = 0; b < nbk; b++) total += bc[(size_t)b * 6 + k];
    }
    for (unsigned b = 0; b < nbk; b++)
      for (int k = 0; k < 6; k++) {
        base[(size_t)b * 6 + k] = start[k];
        start[k] += bc[(size_t)b * 6 + k];
      }
    if (total > n) throw Error{HB_ERR_CUDA, "layout bin counts exceed the sites"};
    L.G = (int)total;
  }
  const int G = L.G;
  L.bulk_sites = (int)n - G;
  int64_t* d_base = P.get<int64_t>(base.size());
  check(cudaMemcpyAsync(d_base, base.data(), base.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st), "bin bases");

  // General records.
  int32_t* gl = P.get<int32_t>(G);
  int32_t* meta = P.get<int32_t>(n);
  LayoutRecordsDev r;
  r.site = P.get<int32_t>(G);
  r.run = P.get<int32_t>(G);
  r.kind = P.get<int32_t>(G);
  r.wall = P.get<uint32_t>(G);
  r.iolet = P.get<uint32_t>(G);
  r.src = P.get<int32_t>((size_t)18 * G);
  r.xyz = P.get<int32_t>((size_t)3 * G);
  r.q = P.get<float>((size_t)18 * G);
  r.nrm = P.get<float>((size_t)3 * G);
  r.io = P.get<int32_t>(G);
  k_bin_place<<<nbk, kT, 0, st>>>(kind, n, d_base, gl);
  k_meta_plain<<<nbk, kT, 0, st>>>(kind, run_of, n, meta);
  if (G > 0) k_records<<<nblk(G), kT, 0, st>>>(a, gl, G, st2ref, regular, run_of, src, r, meta, err);
  check(cudaGetLastError(), "k_records launch");

  download(L.st2ref, st2ref, (size_t)n, st);
  download(L.ref2st, ref2st, (size_t)nt, st);
  download(L.meta, meta, (size_t)n, st);
  download(L.run_off, run_off, (size_t)runs * 20, st);
  download(L.g_site, r.site, (size_t)G, st);
  download(L.g_run, r.run, (size_t)G, st);
  download(L.g_kind, r.kind, (size_t)G, st);
  download(L.g_wall, r.wall, (size_t)G, st);
  download(L.g_iolet, r.iolet, (size_t)G, st);
  download(L.g_src, r.src, (size_t)18 * G, st);
  download(L.g_xyz, r.xyz, (size_t)3 * G, st);
  download(L.g_q, r.q, (size_t)18 * G, st);
  download(L.g_nrm, r.nrm, (size_t)3 * G, st);
  download(L.g_io, r.io, (size_t)G, st);
  sync_and_check("layout records");
  return L;
}

Layout build_layout_on_device(const LatticeTables& t, const hb_params& p, int wall, int device) {
  if (!t.nbr.empty()) return build_layout(t, p, wall);
  check(cudaSetDevice(device), "cudaSetDevice");
  cudaStream_t st;
  check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{st};
  SetupPool P(device, st);
  const int64_t n = t.n;
  DeviceTables d;
  d.n = n;
  d.n_owned = t.n_owned;
  for (int k = 0; k < 3; k++) d.dims[k] = t.dims[k];
  auto up = [&](const auto& v) {
    using T = typename std::decay_t<decltype(v)>::value_type;
    if (v.empty()) return (const T*)nullptr;
    T* ptr = P.get<T>(v.size());
    check(cudaMemcpyAsync(ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st), "table upload");
    return (const T*)ptr;
  };
  d.coords = up(t.coords);
  d.wall = up(t.wall);
  d.iolet = up(t.iolet);
  d.stype = up(t.stype);
  d.iolet_id = up(t.iolet_id);
  d.q = up(t.q);
  d.normal = up(t.normal);
  Layout L = layout_on_device(d, p, st);
  finish_layout(L, t, p, wall);
  return L;
}

}  // namespace hb
