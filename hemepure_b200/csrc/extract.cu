// extract.cu -- extraction sites selected on the device.
//
// The reference evaluates a geometry selector per site when it sets up a
// property output (GeometrySelector::Include, src/extraction/GeometrySelector.cc;
// PlaneGeometrySelector.cc:50, StraightLineGeometrySelector.cc, SphereGeometrySelector.cc,
// InletSelector.cc, OutletSelector.cc, GeometrySurfaceSelector.cc,
// SurfaceWithinSphereSelector.cc, SurfacePointSelector.cc:24) and writes only
// the selected sites.  Here the selector runs in a kernel over the sites in
// the reference's order, the selected sites are compacted into an index list
// in that order, and the fields of those sites alone are gathered into a
// compact buffer, so an output step downloads the selected sites only.
//
// Compiled with -fmad=false: the selectors' util::Vector3D<float> arithmetic
// rounds every product and sum, as the host's (extraction.cpp) does, so the
// device and the host select the same sites.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/hemeb200.h"
#include "device.h"
#include "hb_common.h"

namespace hb {
namespace {

constexpr int kThreads = 256;

struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 vsub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 vadd(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 vmul(V3 a, float k) { return {a.x * k, a.y * k, a.z * k}; }
__device__ __forceinline__ V3 vdiv(V3 a, float k) { return {a.x / k, a.y / k, a.z / k}; }
__device__ __forceinline__ float vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float vmag(V3 a) { return sqrtf(vdot(a, a)); }

__global__ void __launch_bounds__(kThreads) k_select(const SelectArgs s, uint8_t* mask) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  const bool wall = s.wall[i] != 0;
  // Vector3D<float>(location) * voxel + origin, in double, stored as float.
  const V3 c = {(float)((double)(float)s.coords[3 * i] * s.voxel + s.origin[0]),
                (float)((double)(float)s.coords[3 * i + 1] * s.voxel + s.origin[1]),
                (float)((double)(float)s.coords[3 * i + 2] * s.voxel + s.origin[2])};
  const V3 point = {s.point[0], s.point[1], s.point[2]}, normal = {s.normal[0], s.normal[1], s.normal[2]};
  bool take = false;
  switch (s.type) {
    case HB_SELECT_WHOLE:
      take = true;
      break;
    case HB_SELECT_PLANE: {
      const float perp = vdot(vsub(c, point), normal);
      if (fabs((double)perp) > 0.5 * s.voxel) break;
      if (s.radius <= 0.) {
        take = true;
        break;
      }
      const V3 q = vsub(vsub(c, vmul(normal, perp)), point);
      take = vdot(q, q) <= s.radius * s.radius;
      break;
    }
    case HB_SELECT_LINE: {
      const V3 line = {s.line[0], s.line[1], s.line[2]};
      const float along = vdot(line, vsub(c, point)) / s.line_len;
      if (along < 0. || along > s.line_len) break;
      const V3 d = vsub(vadd(point, vdiv(vmul(line, along), s.line_len)), c);
      take = (double)vdot(d, d) <= 2.0 * 0.5 * 0.5 * s.voxel * s.voxel;
      break;
    }
    case HB_SELECT_SPHERE:
      take = vmag(vsub(c, point)) <= s.radius;
      break;
    case HB_SELECT_INLET:
      take = s.stype[i] == 1;
      break;
    case HB_SELECT_OUTLET:
      take = s.stype[i] == 2;
      break;
    case HB_SELECT_SURFACE:
      take = wall;
      break;
    case HB_SELECT_SURFACE_WITHIN_SPHERE:
      take = wall && vmag(vsub(c, point)) <= s.radius;
      break;
    case HB_SELECT_SURFACE_POINT: {
      if (!wall) break;
      const float d = (float)((double)vmag(vsub(c, point)) / s.voxel);
      take = d <= s.max_surface_dist;
      break;
    }
    default:
      break;
  }
  mask[i] = take ? 1 : 0;
}

// Stream compaction of the mask, keeping order: per-block counts, an exclusive
// scan of the counts in one block, then each block writes its selected indices
// at its offset (a block-wide scan of its own flags).
__global__ void __launch_bounds__(kThreads) k_count(const uint8_t* mask, int64_t n, int* counts) {
  __shared__ int warp_sum[kThreads / 32];
  const int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  const int v = i < n ? mask[i] : 0;
  const int w = __reduce_add_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = w;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int k = 0; k < kThreads / 32; k++) t += warp_sum[k];
    counts[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(1024) k_scan_counts(int* counts, int nblocks, int* total) {
  // One block: each thread scans a contiguous chunk, then the chunk totals.
  __shared__ int part[1024];
  const int per = (nblocks + 1023) / 1024;
  const int b = threadIdx.x * per, e = min(nblocks, b + per);
  int acc = 0;
  for (int k = b; k < e; k++) acc += counts[k];
  part[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int k = 0; k < 1024; k++) {
      const int v = part[k];
      part[k] = run;
      run += v;
    }
    *total = run;
  }
  __syncthreads();
  int run = part[threadIdx.x];
  for (int k = b; k < e; k++) {
    const int v = counts[k];
    counts[k] = run;
    run += v;
  }
}

__global__ void __launch_bounds__(kThreads) k_scatter_idx(const uint8_t* mask, int64_t n, const int* offsets, int* idx) {
  __shared__ int warp_off[kThreads / 32];
  const int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  const int v = i < n ? mask[i] : 0;
  const unsigned ballot = __ballot_sync(0xffffffffu, v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) warp_off[warp] = __popc(ballot);
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int k = 0; k < kThreads / 32; k++) {
      const int c = warp_off[k];
      warp_off[k] = run;
      run += c;
    }
  }
  __syncthreads();
  if (v) idx[offsets[blockIdx.x] + warp_off[warp] + __popc(ballot & ((1u << lane) - 1u))] = (int)i;
}

// out[k * width + j] = src[j * stride + st[idx[k]]] for the selected sites
// (a field stored per storage index, `width` values `stride` apart).
__global__ void __launch_bounds__(kThreads) k_gather_sel(const double* src, int64_t stride, int width, const int* idx,
                                                         const int* ref2st, int m, double* out) {
  const int64_t t = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  if (t >= (int64_t)m * width) return;
  const int k = (int)(t / width), j = (int)(t % width);
  out[t] = src[(int64_t)j * stride + ref2st[idx[k]]];
}

// out[k * width + j] = aos[idx[k] * width + j]: rows of an AoS array in reference order.
__global__ void __launch_bounds__(kThreads) k_gather_rows(const double* aos, int width, const int* idx, int m, double* out) {
  const int64_t t = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  if (t >= (int64_t)m * width) return;
  const int k = (int)(t / width), j = (int)(t % width);
  out[t] = aos[(int64_t)idx[k] * width + j];
}

unsigned blocks_for(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

}  // namespace

int select_blocks(int64_t n) { return (int)blocks_for(n); }

void launch_select(const SelectArgs& s, uint8_t* mask, int* counts, int* total, int* idx, void* stream) {
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned nb = blocks_for(s.n);
  if (nb == 0) return;
  k_select<<<nb, kThreads, 0, st>>>(s, mask);
  k_count<<<nb, kThreads, 0, st>>>(mask, s.n, counts);
  k_scan_counts<<<1, 1024, 0, st>>>(counts, (int)nb, total);
  k_scatter_idx<<<nb, kThreads, 0, st>>>(mask, s.n, counts, idx);
}

void launch_gather_selected(const double* src, int64_t stride, int width, const int* idx, const int* ref2st, int m,
                            double* out, void* stream) {
  if (m <= 0) return;
  k_gather_sel<<<blocks_for((int64_t)m * width), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(src, stride, width,
                                                                                                    idx, ref2st, m, out);
}

void launch_gather_rows(const double* aos, int width, const int* idx, int m, double* out, void* stream) {
  if (m <= 0) return;
  k_gather_rows<<<blocks_for((int64_t)m * width), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(aos, width, idx, m,
                                                                                                     out);
}

}  // namespace hb
