// noalloc.cu -- conserved sums for callers that cannot allocate device memory.
//
// hb_moment_sums (solver.cpp) reduces with a scratch buffer the handle allocates.
// Some callers may not have the library allocate anything: a process whose
// device memory is all pre-committed to its own pool or to a fixed HBM budget
// (the serving layer's admission control accounts for every byte it admits), or
// an embedding framework that owns allocation.  For them,
// hb_moment_sums_noalloc runs the same two-pass reduction on buffers the caller
// owns, with its scratch in the file-scope array below instead of cudaMalloc.
//
// The array is kNoAllocMaxBlocks x 4 doubles (256 KiB); every GPU that loads
// the library holds it until the process exits.  Each block of 2048 sites takes
// one 4-double slot, so one call covers at most kNoAllocMaxBlocks * 2048 =
// 16,777,216 sites; larger calls are rejected.  All calls share the array: two
// calls whose kernels overlap on the same GPU race on it.  Every slot a call
// reads is written earlier in that call, so nothing needs clearing between calls.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/hemeb200.h"
#include "device.h"

namespace hb {
void set_last_error(const std::string& msg);  // capi.cpp
}

namespace {

constexpr int kNoAllocMaxBlocks = 8192;
constexpr int64_t kNoAllocMaxSites = (int64_t)kNoAllocMaxBlocks * hb::kSumSitesPerBlock;

static __device__ __align__(256) double g_sum_scratch[kNoAllocMaxBlocks * 4];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of g_sum_scratch on the current device, looked up once per
// device.  In host code the symbol itself is only a host-side stand-in.
int scratch_for_current_device(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    hb::set_last_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return HB_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    hb::set_last_error("device ordinal out of range");
    return HB_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_sum_scratch);
    if (e != cudaSuccess || !p) {
      hb::set_last_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return HB_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return HB_OK;
}

}  // namespace

extern "C" int hb_moment_sums_noalloc(const double* f, int64_t dir_stride, int64_t site_stride, int64_t n_sites,
                                      double* sums, void* stream) {
  if (!f || !sums || dir_stride <= 0 || site_stride <= 0 || n_sites <= 0) {
    hb::set_last_error("hb_moment_sums_noalloc: null pointer or non-positive size or stride");
    return HB_ERR_ARG;
  }
  if (n_sites > kNoAllocMaxSites) {
    hb::set_last_error("hb_moment_sums_noalloc: " + std::to_string(n_sites) + " sites exceed the fixed scratch limit of " +
                       std::to_string(kNoAllocMaxSites) + " sites per call");
    return HB_ERR_ARG;
  }
  double* scratch = nullptr;
  const int rc = scratch_for_current_device(&scratch);
  if (rc != HB_OK) return rc;
  hb::launch_moment_sums(f, dir_stride, site_stride, n_sites, scratch, sums, stream);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    hb::set_last_error(std::string("hb_moment_sums_noalloc launch: ") + cudaGetErrorString(e));
    return HB_ERR_CUDA;
  }
  return HB_OK;
}
