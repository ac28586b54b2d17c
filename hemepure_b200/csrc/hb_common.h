// hb_common.h -- D3Q19 constants and shared host/device definitions.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#ifdef __CUDACC__
#define HB_HD __host__ __device__ __forceinline__
#else
#define HB_HD inline
#endif

namespace hb {

constexpr int Q = 19;
// FP16 shifted storage holds (f - w) * kHalfScale: non-equilibrium parts of
// order 1e-4..1e-2 then sit in FP16's normal range.
constexpr float kHalfScale = 1024.0f;

// D3Q19 velocity set, weights and inverse directions (src/lb/lattices/D3Q19.cc:15-33).
HB_HD constexpr int cx(int i) {
  return (i == 1 || i == 7 || i == 9 || i == 11 || i == 13) ? 1
         : (i == 2 || i == 8 || i == 10 || i == 12 || i == 14) ? -1 : 0;
}
HB_HD constexpr int cy(int i) {
  return (i == 3 || i == 7 || i == 10 || i == 15 || i == 17) ? 1
         : (i == 4 || i == 8 || i == 9 || i == 16 || i == 18) ? -1 : 0;
}
HB_HD constexpr int cz(int i) {
  return (i == 5 || i == 11 || i == 14 || i == 15 || i == 18) ? 1
         : (i == 6 || i == 12 || i == 13 || i == 16 || i == 17) ? -1 : 0;
}
HB_HD constexpr int cc(int axis, int i) { return axis == 0 ? cx(i) : (axis == 1 ? cy(i) : cz(i)); }
HB_HD constexpr int inv(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }
HB_HD constexpr double weight(int i) { return i == 0 ? 1.0 / 3.0 : (i < 7 ? 1.0 / 18.0 : 1.0 / 36.0); }

constexpr double kCs2 = 1.0 / 3.0;
constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kNoValue = 1.7976931348623157e308;  // std::numeric_limits<double>::max()

enum Kernel { kLBGK = 0, kTRT = 1, kLES = 2, kLBGKSL = 3, kTRTSL = 4 };
// The kernels with a per-site sponge relaxation time.
constexpr bool is_sponge(int k) { return k == kLES || k == kLBGKSL || k == kTRTSL; }
enum Wall { kSBB = 0, kBFL = 1, kGZS = 2 };
enum IoletKind { kCosine = 0, kWK3 = 1, kParabolic = 2, kWK2 = 3, kFile = 4, kFileVelocity = 5, kWomersley = 6 };
// Velocity iolets take the Ladd streamer; the others the Nash zeroth-order pressure streamer.
HB_HD constexpr bool is_velocity_iolet(int kind) { return kind == kParabolic || kind == kFileVelocity || kind == kWomersley; }

// Host-side error carrying one of the HB_ERR_* codes.
struct Error {
  int code;
  std::string msg;
};

}  // namespace hb
