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
// the library holds it until the process exits.  Under CUDA's lazy module
// loading (the default since CUDA 12) the array comes into being on a device
// when the library's module is loaded there, at the latest when the first call
// looks up its address: a caller that commits all of its device memory should
// make one call (a warm-up) before doing so.  Each block of 2048 sites takes
// one 4-double slot, so one call covers at most kNoAllocMaxBlocks * 2048 =
// 16,777,216 sites; larger calls are rejected.  All calls share the array: two
// calls whose kernels overlap on the same GPU race on it.  Every slot a call
// reads is written earlier in that call, so nothing needs clearing between calls.
//
// The device address is looked up once per device and kept.  A device reset
// (cudaDeviceReset) replaces the device's context and reloads the module,
// possibly elsewhere; the kept address is therefore tagged with the context's
// identifier (cuCtxGetId) and looked up again when the current context differs.
#include <cuda.h>
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
unsigned long long g_scratch_ctx[kMaxDevices] = {0};  // context identifier the address belongs to (0: unknown)

// Identifier of the calling thread's current context (0 when the driver entry
// points are unavailable; the address is then kept per device only).
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    void* a = nullptr;
    void* b = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, nullptr) == cudaSuccess &&
        cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, nullptr) == cudaSuccess) {
      get_current = reinterpret_cast<GetCurrent>(a);
      get_id = reinterpret_cast<GetId>(b);
    }
    looked_up = true;
  }
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of g_sum_scratch on the current device, looked up once per
// device (and again after the device's context was replaced).  In host code the
// symbol itself is only a host-side stand-in.
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
    // First use on this device: make the runtime's context current, so that the
    // context identifier below names the context the address belongs to.
    e = cudaFree(nullptr);
    if (e != cudaSuccess) {
      hb::set_last_error(std::string("cudaFree(0): ") + cudaGetErrorString(e));
      return HB_ERR_CUDA;
    }
  }
  const unsigned long long ctx = current_context_id();
  if (!g_scratch_ptr[dev] || (ctx != 0 && ctx != g_scratch_ctx[dev])) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_sum_scratch);
    if (e != cudaSuccess || !p) {
      hb::set_last_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return HB_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<double*>(p);
    g_scratch_ctx[dev] = ctx;
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
