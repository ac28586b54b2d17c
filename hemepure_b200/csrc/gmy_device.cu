// gmy_device.cu -- the .gmy v4 reader with its decode on the GPU.
//
// The same tables as read_gmy (config.cpp), bit for bit, from the same steps of
// the reference's GeometryReader and LatticeData (src/geometry/GeometryReader.cc:
// 382-444 preamble, 515-607 header, 800-946 inflate and site records;
// src/geometry/SiteDataBare.cc:24-172 classification; src/geometry/LatticeData.cc:
// 69-285 contiguous order, 366-443 neighbour table), split by where the work fits:
//
//   host   read the file, check the preamble and block header, inflate the
//          non-empty blocks with one zlib stream per block on a pool of threads
//          (each block lands 16-byte aligned in one buffer), copy it to the GPU;
//   GPU    k_decode   one thread per non-empty block walks its site records
//                     (big-endian words, bounds-checked against the block's own
//                     bytes) and writes each fluid site's masks, ids, cut
//                     distances and normal in read order, with the block's count
//                     of sites per collision type;
//          (host)     exclusive scan of those counts: the first contiguous index
//                     of each type in each block (a few KB);
//          k_place    one thread per block places its sites at their contiguous
//                     index: binned by collision type, block-traversal order
//                     within a type (read order is block-traversal order), and
//                     normalises the wall normals in float;
//   host   copy the tables back.  The neighbour table is not built here: the
//          storage layout looks neighbours up in its own coordinate grid, and
//          neighbour_table() derives the reference's table when it is asked for.
//
// Malformed input is reported through an error word the kernels set with
// atomicCAS (first error wins) and the host turns into hb::Error; no kernel
// reads outside its block's bytes or writes outside its block's output range.
#include <cuda_runtime.h>
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "config.h"
#include "layout.h"
#include "setup_pool.h"

namespace hb {
namespace {

enum GmyErr : int {
  kGmyOk = 0,
  kGmyTruncated = 1,     // a record runs past its block's bytes
  kGmyNormal = 2,        // normal flag disagrees with the wall links
  kGmyCount = 3,         // fluid-site count differs from the block header
};

struct BlockDev {
  int64_t raw_off;       // byte offset of the block's inflated records (16-byte aligned)
  int64_t out_base;      // first read-order index of the block's sites
  int64_t block;         // block index (bx * By + by) * Bz + bz
  uint32_t raw_len;      // inflated bytes
  uint32_t count;        // fluid sites the header declares
};

// Read-order records (structure of arrays).
struct RecDev {
  uint32_t* wall;
  uint32_t* iolet;
  int32_t* stype;
  int32_t* iolet_id;
  int32_t* local;        // site index within its block
  float* dist;           // [18][n]
  float* nrm;            // [3][n]
  uint8_t* has_nrm;
};

__device__ __forceinline__ uint32_t bswap32(uint32_t v) { return __byte_perm(v, 0, 0x0123); }

__device__ __forceinline__ void set_err(int* err, int code, int64_t where) {
  if (atomicCAS(err, 0, code) == 0) err[1] = (int)where;
}

// The 26 displacements in the .gmy's order (dx, dy, dz each -1..1, z fastest,
// the zero vector skipped) mapped to D3Q19 directions, or -1.
__device__ __forceinline__ int gmy_dir(int k) {
  const int j = k < 13 ? k : k + 1;
  const int dx = j / 9 - 1, dy = (j / 3) % 3 - 1, dz = j % 3 - 1;
  for (int d = 1; d < Q; d++)
    if (cx(d) == dx && cy(d) == dy && cz(d) == dz) return d;
  return -1;
}

__device__ __forceinline__ int collision_type_of(uint32_t wall, int stype) {
  return wall == 0 ? (stype == 0 ? 0 : (stype == 1 ? 2 : 3)) : (stype == 0 ? 1 : (stype == 1 ? 4 : 5));
}

__global__ void k_decode(const uint32_t* __restrict__ raw, const BlockDev* __restrict__ blocks, int nb, int bs3,
                         RecDev rec, int64_t n, int32_t* __restrict__ type_counts, int* err) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nb) return;
  const BlockDev B = blocks[k];
  const uint32_t* w = raw + B.raw_off / 4;
  const uint32_t nw = B.raw_len / 4;
  uint32_t pos = 0;
  bool bad = false;
  auto rd = [&]() -> uint32_t {
    if (pos >= nw) {
      bad = true;
      return 0u;
    }
    return bswap32(__ldg(w + pos++));
  };
  int32_t tc[6] = {0, 0, 0, 0, 0, 0};
  uint32_t count = 0;
  for (int s = 0; s < bs3 && !bad; s++) {
    if (!rd()) continue;
    if (count >= B.count) {
      set_err(err, kGmyCount, B.block);
      return;
    }
    const int64_t r = B.out_base + count;
    if (r >= n) {
      set_err(err, kGmyCount, B.block);
      return;
    }
    uint32_t wall = 0, iolet = 0;
    int32_t iolet_id = -1;
    bool gmy_wall = false, had_in = false, had_out = false;
    for (int d = 0; d < 18; d++) rec.dist[(int64_t)d * n + r] = -1.0f;
    // Every link is read whatever its direction; only D3Q19 directions are kept.
    int32_t ids[18];
    uint8_t types[18];
    for (int d = 0; d < 18; d++) {
      ids[d] = -1;
      types[d] = 0;
    }
    for (int l = 0; l < 26; l++) {
      const uint32_t ty = rd();
      float dist = -1.0f;
      int32_t iid = -1;
      if (ty == 1) {
        gmy_wall = true;
        dist = __uint_as_float(rd());
      } else if (ty != 0) {
        iid = (int32_t)rd();
        dist = __uint_as_float(rd());
      }
      const int d = gmy_dir(l);
      if (d > 0) {
        types[d - 1] = (uint8_t)ty;
        ids[d - 1] = iid;
        rec.dist[(int64_t)(d - 1) * n + r] = dist;
      }
    }
    const bool has_normal = rd() == 1u;
    if (has_normal != gmy_wall) {
      set_err(err, kGmyNormal, B.block);
      return;
    }
    float nv[3] = {0.0f, 0.0f, 0.0f};
    if (has_normal) {
      nv[0] = __uint_as_float(rd());
      nv[1] = __uint_as_float(rd());
      nv[2] = __uint_as_float(rd());
    }
    if (bad) break;
    // SiteData: wall and iolet bits; the iolet id and type of the last iolet link.
    for (int d = 1; d <= 18; d++) {
      const int ty = types[d - 1];
      if (ty == 1) wall |= 1u << (d - 1);
      else if (ty == 2 || ty == 3) iolet |= 1u << (d - 1);
      if (ty == 2) {
        iolet_id = ids[d - 1];
        had_in = true;
      } else if (ty == 3) {
        iolet_id = ids[d - 1];
        had_out = true;
      }
    }
    const int stype = had_in ? 1 : (had_out ? 2 : 0);
    rec.wall[r] = wall;
    rec.iolet[r] = iolet;
    rec.stype[r] = stype;
    rec.iolet_id[r] = iolet_id;
    rec.local[r] = s;
    rec.has_nrm[r] = has_normal ? 1 : 0;
    for (int c = 0; c < 3; c++) rec.nrm[(int64_t)c * n + r] = nv[c];
    tc[collision_type_of(wall, stype)]++;
    count++;
  }
  if (bad) {
    set_err(err, kGmyTruncated, B.block);
    return;
  }
  if (count != B.count) {
    set_err(err, kGmyCount, B.block);
    return;
  }
  for (int t = 0; t < 6; t++) type_counts[6 * (int64_t)k + t] = tc[t];
}

struct TablesDev {
  int64_t* coords;       // [n][3]
  uint32_t* wall;
  uint32_t* iolet;
  int32_t* stype;
  int32_t* iolet_id;
  float* q;              // [n][18]
  float* normal;         // [n][3]
};

// Vector3D<float>::GetNormalised, in float with the host's rounding.
__device__ __forceinline__ void normalised(const float in[3], float out[3]) {
  const float nx = in[0], ny = in[1], nz = in[2];
  if (nx == 0.0f && ny == 0.0f && nz == 0.0f) {
    out[0] = out[1] = out[2] = 0.0f;
    return;
  }
  const float m2 = __fadd_rn(__fadd_rn(__fmul_rn(nx, nx), __fmul_rn(ny, ny)), __fmul_rn(nz, nz));
  const float m = __fsqrt_rn(m2);
  out[0] = __fdiv_rn(nx, m);
  out[1] = __fdiv_rn(ny, m);
  out[2] = __fdiv_rn(nz, m);
}

__global__ void k_place(const BlockDev* __restrict__ blocks, int nb, const int64_t* __restrict__ first, RecDev rec,
                        int64_t n, int bs, int64_t by_blocks, int64_t bz_blocks, TablesDev t) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nb) return;
  const BlockDev B = blocks[k];
  int64_t next[6];
  for (int c = 0; c < 6; c++) next[c] = first[6 * (int64_t)k + c];
  const int64_t bxi = B.block / (by_blocks * bz_blocks), byi = (B.block / bz_blocks) % by_blocks,
                bzi = B.block % bz_blocks;
  for (uint32_t j = 0; j < B.count; j++) {
    const int64_t r = B.out_base + j;
    const uint32_t wall = rec.wall[r];
    const int32_t st = rec.stype[r];
    const int64_t c = next[collision_type_of(wall, st)]++;
    if (c < 0 || c >= n) return;
    const int s = rec.local[r];
    t.coords[3 * c] = bxi * bs + s / (bs * bs);
    t.coords[3 * c + 1] = byi * bs + (s / bs) % bs;
    t.coords[3 * c + 2] = bzi * bs + s % bs;
    t.wall[c] = wall;
    t.iolet[c] = rec.iolet[r];
    t.stype[c] = st;
    t.iolet_id[c] = rec.iolet_id[r];
    for (int d = 0; d < 18; d++) t.q[18 * c + d] = rec.dist[(int64_t)d * n + r];
    float nd[3];
    if (rec.has_nrm[r]) {
      const float nv[3] = {rec.nrm[r], rec.nrm[n + r], rec.nrm[2 * n + r]};
      normalised(nv, nd);
    } else {
      nd[0] = nd[1] = nd[2] = HUGE_VALF;
    }
    for (int e = 0; e < 3; e++) t.normal[3 * c + e] = nd[e];
  }
}

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error{HB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

uint32_t be32(const unsigned char* b) {
  return (uint32_t(b[0]) << 24) | (uint32_t(b[1]) << 16) | (uint32_t(b[2]) << 8) | uint32_t(b[3]);
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

cudaMemPool_t setup_pool(int device, bool fresh) {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  std::lock_guard<std::mutex> lock(mu);
  auto it = pools.find(device);
  if (it != pools.end() && !fresh) return it->second;
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  cudaMemPool_t pool = nullptr;
  cuda_check(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
  uint64_t keep = kSetupPoolKeep;
  cuda_check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
  pools[device] = pool;
  return pool;
}

LatticeTables read_gmy_device(const std::string& path, int device, GmyTiming* timing, const hb_params* params, int wall,
                              Layout* layout) {
  if (layout && !params) throw Error{HB_ERR_ARG, "the layout needs the case parameters"};
  auto t0 = std::chrono::steady_clock::now();
  GmyTiming tm{};
  std::ifstream in(path, std::ios::binary);
  if (!in) throw Error{HB_ERR_IO, "cannot open geometry file " + path};
  std::vector<unsigned char> buf((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  if (buf.size() < 32) throw Error{HB_ERR_FORMAT, "truncated preamble"};
  if (be32(&buf[0]) != 0x686c6221u) throw Error{HB_ERR_FORMAT, "This file does not start with the HemeLB magic number."};
  if (be32(&buf[4]) != 0x676d7904u) throw Error{HB_ERR_FORMAT, "This file does not have the geometry magic number."};
  if (be32(&buf[8]) != 4u) throw Error{HB_ERR_FORMAT, "Version number incorrect."};
  LatticeTables t;
  for (int d = 0; d < 3; d++) t.blocks[d] = be32(&buf[12 + 4 * d]);
  t.block_size = be32(&buf[24]);
  const int64_t bs = t.block_size, bs3 = bs * bs * bs;
  for (int d = 0; d < 3; d++) t.dims[d] = t.blocks[d] * bs;
  const int64_t nblocks = t.blocks[0] * t.blocks[1] * t.blocks[2];
  if (bs <= 0 || nblocks <= 0) throw Error{HB_ERR_FORMAT, "empty geometry"};
  if (bs3 > (1 << 20)) throw Error{HB_ERR_UNSUPPORTED, "block size above 128"};
  if (32 + 12 * (size_t)nblocks > buf.size()) throw Error{HB_ERR_FORMAT, "truncated header"};

  // Non-empty blocks: compressed source, 16-byte-aligned inflated destination,
  // read-order output base.
  std::vector<BlockDev> blocks;
  std::vector<size_t> src_off;
  std::vector<uint32_t> src_len;
  size_t off = 32 + 12 * (size_t)nblocks;
  int64_t raw_total = 0, n = 0;
  for (int64_t b = 0; b < nblocks; b++) {
    const unsigned char* h = &buf[32 + 12 * (size_t)b];
    const uint32_t fluid = be32(h), cb = be32(h + 4), ub = be32(h + 8);
    if (fluid == 0) continue;
    if (off + cb > buf.size()) throw Error{HB_ERR_FORMAT, "truncated block data"};
    if ((int64_t)fluid > bs3) throw Error{HB_ERR_FORMAT, "block fluid-site count does not match its header"};
    BlockDev B;
    B.raw_off = raw_total;
    B.raw_len = ub;
    B.block = b;
    B.count = fluid;
    B.out_base = n;
    blocks.push_back(B);
    src_off.push_back(off);
    src_len.push_back(cb);
    off += cb;
    raw_total += ((int64_t)ub + 15) / 16 * 16;
    n += fluid;
  }
  if (n > ((int64_t)1 << 31) - 1) throw Error{HB_ERR_UNSUPPORTED, "more than 2^31 sites"};
  const int nb = (int)blocks.size();
  tm.read_ms = ms_since(t0);

  // Inflate on a pool of host threads.
  auto t1 = std::chrono::steady_clock::now();
  // Left uninitialised: the inflating threads touch its pages first, in parallel.
  const size_t raw_size = (size_t)std::max<int64_t>(raw_total, 16);
  std::unique_ptr<unsigned char[]> raw(new unsigned char[raw_size]);
  std::atomic<int> next{0}, failed{-1};
  auto work = [&]() {
    for (int k = next++; k < nb; k = next++) {
      uLongf dl = blocks[k].raw_len;
      if (uncompress(raw.get() + blocks[k].raw_off, &dl, buf.data() + src_off[k], src_len[k]) != Z_OK) {
        int exp = -1;
        failed.compare_exchange_strong(exp, k);
        continue;
      }
      blocks[k].raw_len = (uint32_t)dl;  // the decoder stays inside what was inflated
    }
  };
  const int nthreads = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  for (int i = 1; i < nthreads; i++) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
  if (failed.load() >= 0) throw Error{HB_ERR_FORMAT, "Decompression error for block!"};
  tm.inflate_ms = ms_since(t1);

  cuda_check(cudaSetDevice(device), "cudaSetDevice");
  cudaStream_t st;
  cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{st};
  SetupPool P(device, st);
  auto t2 = std::chrono::steady_clock::now();
  uint32_t* d_raw = P.get<uint32_t>(raw_size / 4 + 1);
  BlockDev* d_blocks = P.get<BlockDev>(nb);
  cuda_check(cudaMemcpyAsync(d_raw, raw.get(), raw_size, cudaMemcpyHostToDevice, st), "copy of the inflated blocks");
  cuda_check(cudaMemcpyAsync(d_blocks, blocks.data(), sizeof(BlockDev) * nb, cudaMemcpyHostToDevice, st), "copy of the block table");
  cuda_check(cudaStreamSynchronize(st), "copy of the inflated blocks");
  tm.h2d_ms = ms_since(t2);

  auto t3 = std::chrono::steady_clock::now();
  RecDev rec;
  rec.wall = P.get<uint32_t>(n);
  rec.iolet = P.get<uint32_t>(n);
  rec.stype = P.get<int32_t>(n);
  rec.iolet_id = P.get<int32_t>(n);
  rec.local = P.get<int32_t>(n);
  rec.dist = P.get<float>(18 * (size_t)n);
  rec.nrm = P.get<float>(3 * (size_t)n);
  rec.has_nrm = P.get<uint8_t>(n);
  int32_t* d_tc = P.get<int32_t>(6 * (size_t)nb);
  int* d_err = P.get<int>(2);
  cuda_check(cudaMemsetAsync(d_err, 0, 2 * sizeof(int), st), "cudaMemset");
  const int tb = 128;
  if (nb > 0) k_decode<<<(nb + tb - 1) / tb, tb, 0, st>>>(d_raw, d_blocks, nb, (int)bs3, rec, n, d_tc, d_err);
  cuda_check(cudaGetLastError(), "k_decode launch");
  std::vector<int32_t> tc(6 * (size_t)nb);
  int herr[2] = {0, 0};
  cuda_check(cudaMemcpyAsync(tc.data(), d_tc, tc.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, st), "type counts");
  cuda_check(cudaMemcpyAsync(herr, d_err, sizeof(herr), cudaMemcpyDeviceToHost, st), "error word");
  cuda_check(cudaStreamSynchronize(st), "site record decode");
  auto raise = [&](int code, int where) {
    switch (code) {
      case kGmyTruncated: throw Error{HB_ERR_FORMAT, "truncated site record (block " + std::to_string(where) + ")"};
      case kGmyNormal: throw Error{HB_ERR_FORMAT, "Malformed GMY file, wall normal does not match the wall links (block " + std::to_string(where) + ")"};
      case kGmyCount: throw Error{HB_ERR_FORMAT, "block fluid-site count does not match its header (block " + std::to_string(where) + ")"};
      default: throw Error{HB_ERR_FORMAT, "geometry decode error"};
    }
  };
  if (herr[0]) raise(herr[0], herr[1]);

  // First contiguous index of each collision type in each block.
  for (int k = 0; k < nb; k++)
    for (int c = 0; c < 6; c++) t.type_counts[c] += tc[6 * (size_t)k + c];
  std::vector<int64_t> first(6 * (size_t)nb);
  {
    int64_t start[6];
    start[0] = 0;
    for (int c = 1; c < 6; c++) start[c] = start[c - 1] + t.type_counts[c - 1];
    for (int k = 0; k < nb; k++)
      for (int c = 0; c < 6; c++) {
        first[6 * (size_t)k + c] = start[c];
        start[c] += tc[6 * (size_t)k + c];
      }
  }
  int64_t* d_first = P.get<int64_t>(first.size());
  cuda_check(cudaMemcpyAsync(d_first, first.data(), first.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st), "type starts");
  TablesDev T;
  T.coords = P.get<int64_t>(3 * (size_t)n);
  T.wall = P.get<uint32_t>(n);
  T.iolet = P.get<uint32_t>(n);
  T.stype = P.get<int32_t>(n);
  T.iolet_id = P.get<int32_t>(n);
  T.q = P.get<float>(18 * (size_t)n);
  T.normal = P.get<float>(3 * (size_t)n);
  if (nb > 0) k_place<<<(nb + tb - 1) / tb, tb, 0, st>>>(d_blocks, nb, d_first, rec, n, (int)bs, t.blocks[1], t.blocks[2], T);
  cuda_check(cudaGetLastError(), "k_place launch");
  cuda_check(cudaStreamSynchronize(st), "k_place");
  tm.device_ms = ms_since(t3);

  auto t4 = std::chrono::steady_clock::now();
  t.n = n;
  // The tables come back to the host on a second stream and host thread while
  // the layout's passes (when asked for) run on the device copy.
  cudaStream_t st2;
  cuda_check(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking), "cudaStreamCreate");
  StreamGuard sg2{st2};
  cudaError_t d2h_err = cudaSuccess;
  auto download = [&]() {
    try {
      t.coords.resize(3 * (size_t)n);
      t.wall.resize(n);
      t.iolet.resize(n);
      t.stype.resize(n);
      t.iolet_id.resize(n);
      t.q.resize(18 * (size_t)n);
      t.normal.resize(3 * (size_t)n);
    } catch (const std::bad_alloc&) {
      d2h_err = cudaErrorMemoryAllocation;
      return;
    }
    // Pageable copies go through the driver's staging buffers and the host's
    // first touch of each page: a few host threads, each with its own stream and
    // a slice of every table, keep the copy engine busy.
    struct Part {
      void* dst;
      const void* src;
      size_t bytes, elem;
    };
    const Part parts[] = {{t.coords.data(), T.coords, t.coords.size() * sizeof(int64_t), sizeof(int64_t)},
                          {t.wall.data(), T.wall, (size_t)n * sizeof(uint32_t), sizeof(uint32_t)},
                          {t.iolet.data(), T.iolet, (size_t)n * sizeof(uint32_t), sizeof(uint32_t)},
                          {t.stype.data(), T.stype, (size_t)n * sizeof(int32_t), sizeof(int32_t)},
                          {t.iolet_id.data(), T.iolet_id, (size_t)n * sizeof(int32_t), sizeof(int32_t)},
                          {t.q.data(), T.q, t.q.size() * sizeof(float), sizeof(float)},
                          {t.normal.data(), T.normal, t.normal.size() * sizeof(float), sizeof(float)}};
    const int workers = (int)std::max<int64_t>(1, std::min<int64_t>(nthreads, n / 65536));
    std::vector<cudaError_t> errs(workers, cudaSuccess);
    auto work_slice = [&](int w) {
      cudaError_t e = cudaSetDevice(device);
      cudaStream_t ws = st2;
      if (e == cudaSuccess && w > 0) e = cudaStreamCreateWithFlags(&ws, cudaStreamNonBlocking);
      if (e != cudaSuccess) {
        errs[w] = e;
        return;
      }
      for (const Part& p : parts) {
        const size_t count = p.bytes / p.elem;
        const size_t b = count * w / workers, en = count * (w + 1) / workers;
        // First touch of this slice's pages here, in parallel with the other
        // workers, rather than inside the driver's copy.
        volatile char* c = static_cast<char*>(p.dst);
        for (size_t off = b * p.elem; off < en * p.elem; off += 4096) c[off] = 0;
        if (en > b && e == cudaSuccess)
          e = cudaMemcpyAsync(static_cast<char*>(p.dst) + b * p.elem, static_cast<const char*>(p.src) + b * p.elem,
                              (en - b) * p.elem, cudaMemcpyDeviceToHost, ws);
      }
      const cudaError_t se = cudaStreamSynchronize(ws);
      if (e == cudaSuccess) e = se;
      if (w > 0) cudaStreamDestroy(ws);
      errs[w] = e;
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < workers; w++) pool.emplace_back(work_slice, w);
    work_slice(0);
    for (auto& th : pool) th.join();
    for (cudaError_t e : errs)
      if (d2h_err == cudaSuccess) d2h_err = e;
  };
  if (!layout) {
    download();
  } else {
    std::thread th(download);
    struct Join {
      std::thread& th;
      ~Join() {
        if (th.joinable()) th.join();
      }
    } join{th};
    DeviceTables dt;
    dt.n = n;
    for (int d = 0; d < 3; d++) dt.dims[d] = t.dims[d];
    dt.coords = T.coords;
    dt.wall = T.wall;
    dt.iolet = T.iolet;
    dt.stype = T.stype;
    dt.iolet_id = T.iolet_id;
    dt.q = T.q;
    dt.normal = T.normal;
    *layout = layout_on_device(dt, *params, st);
    th.join();
  }
  if (d2h_err == cudaErrorMemoryAllocation) throw Error{HB_ERR_OOM, "host memory for the tables"};
  cuda_check(d2h_err, "copy of the tables");
  if (layout) finish_layout(*layout, t, *params, wall);
  tm.d2h_ms = ms_since(t4);
  if (timing) *timing = tm;
  return t;
}

}  // namespace hb
