// setup_pool.h -- device memory of the set-up passes (geometry decode, storage
// layout): stream-ordered allocations from a memory pool of the library's own,
// one per device.  Freeing returns the memory to the pool instead of unmapping
// it, which made a case's set-up take from 0.3 to 1 s by the frees alone; the
// pool keeps up to kSetupPoolKeep bytes between set-ups (what a lattice of
// about eight million sites needs) and gives the rest back at the next
// synchronisation.  Allocations of one set-up come from a SetupPool object,
// returned on every path.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "hb_common.h"

namespace hb {

constexpr uint64_t kSetupPoolKeep = (uint64_t)4 << 30;

// The library's pool on `device` (created on first use; `fresh` makes a new one,
// for a device whose context was replaced since).
cudaMemPool_t setup_pool(int device, bool fresh = false);

class SetupPool {
 public:
  SetupPool(int device, cudaStream_t stream) : device_(device), pool_(setup_pool(device)), stream_(stream) {}
  SetupPool(const SetupPool&) = delete;
  SetupPool& operator=(const SetupPool&) = delete;
  ~SetupPool() {
    for (void* p : ptrs_) cudaFreeAsync(p, stream_);
  }
  template <class T>
  T* get(size_t count) {
    void* p = nullptr;
    const size_t bytes = (count ? count : 1) * sizeof(T);
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool_, stream_);
    if (e != cudaSuccess && e != cudaErrorMemoryAllocation && ptrs_.empty()) {
      cudaGetLastError();
      pool_ = setup_pool(device_, true);
      e = cudaMallocFromPoolAsync(&p, bytes, pool_, stream_);
    }
    if (e != cudaSuccess)
      throw Error{e == cudaErrorMemoryAllocation ? HB_ERR_OOM : HB_ERR_CUDA,
                  std::string("device memory for set-up: ") + cudaGetErrorString(e)};
    ptrs_.push_back(p);
    return static_cast<T*>(p);
  }

 private:
  int device_;
  cudaMemPool_t pool_;
  cudaStream_t stream_;
  std::vector<void*> ptrs_;
};

}  // namespace hb
