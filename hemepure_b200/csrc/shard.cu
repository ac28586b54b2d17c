// shard.cu -- halo pack and unpack of the sharded form: the values crossing a
// slab cut are copied between a distribution buffer and a contiguous exchange
// buffer through an element-index list (shard.h).  The copies move the stored
// elements bit for bit (FP64, or the shifted FP32 / FP16 storage), so a shard
// pulls exactly what the single lattice would have held there.
#include <cuda_runtime.h>

#include <cstdint>

#include "device.h"

namespace hb {
namespace {

constexpr int kThreads = 256;

template <class T>
__global__ void __launch_bounds__(kThreads) k_halo_pack(const T* __restrict__ f, const int64_t* __restrict__ idx,
                                                        int64_t m, T* __restrict__ out) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x)
    out[k] = f[__ldg(idx + k)];
}

template <class T>
__global__ void __launch_bounds__(kThreads) k_halo_unpack(const T* __restrict__ in, const int64_t* __restrict__ idx,
                                                          int64_t m, T* __restrict__ f) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x)
    f[__ldg(idx + k)] = in[k];
}

int grid_for(int64_t m) {
  const int64_t b = (m + kThreads - 1) / kThreads;
  return (int)(b < 148 * 8 ? (b > 0 ? b : 1) : 148 * 8);
}

}  // namespace

void launch_halo_pack(const void* f, const int64_t* idx, int64_t m, void* out, int elem_bytes, void* stream) {
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int g = grid_for(m);
  if (elem_bytes == 8)
    k_halo_pack<<<g, kThreads, 0, st>>>(static_cast<const double*>(f), idx, m, static_cast<double*>(out));
  else if (elem_bytes == 4)
    k_halo_pack<<<g, kThreads, 0, st>>>(static_cast<const float*>(f), idx, m, static_cast<float*>(out));
  else
    k_halo_pack<<<g, kThreads, 0, st>>>(static_cast<const uint16_t*>(f), idx, m, static_cast<uint16_t*>(out));
}

void launch_halo_unpack(const void* in, const int64_t* idx, int64_t m, void* f, int elem_bytes, void* stream) {
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int g = grid_for(m);
  if (elem_bytes == 8)
    k_halo_unpack<<<g, kThreads, 0, st>>>(static_cast<const double*>(in), idx, m, static_cast<double*>(f));
  else if (elem_bytes == 4)
    k_halo_unpack<<<g, kThreads, 0, st>>>(static_cast<const float*>(in), idx, m, static_cast<float*>(f));
  else
    k_halo_unpack<<<g, kThreads, 0, st>>>(static_cast<const uint16_t*>(in), idx, m, static_cast<uint16_t*>(f));
}

}  // namespace hb
