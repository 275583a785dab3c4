// Shared helpers for the ves3d_b200 CUDA library: status codes, thread-local error
// text, a global launch counter, and device helpers.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <cstdio>
#include <string>

#include "../../include/ves3d_b200.h"

namespace ves3d {

void set_error(const char* fmt, ...);
std::atomic<long long>& launch_counter();

inline int cuda_status(cudaError_t e, const char* what, const char* file, int line) {
  if (e == cudaSuccess) return VES3D_OK;
  set_error("%s failed at %s:%d: %s", what, file, line, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? VES3D_ERR_NOMEM : VES3D_ERR_CUDA;
}

#define VES3D_CK(call)                                                          \
  do {                                                                          \
    int _st = ::ves3d::cuda_status((call), #call, __FILE__, __LINE__);          \
    if (_st != VES3D_OK) return _st;                                            \
  } while (0)

// Check the launch that was just issued and count it.
#define VES3D_LAUNCHED()                                                        \
  do {                                                                          \
    ::ves3d::launch_counter().fetch_add(1, std::memory_order_relaxed);          \
    int _st = ::ves3d::cuda_status(cudaGetLastError(), "kernel launch", __FILE__, __LINE__); \
    if (_st != VES3D_OK) return _st;                                            \
  } while (0)

#define VES3D_ARG(cond, msg)                                                    \
  do {                                                                          \
    if (!(cond)) {                                                              \
      ::ves3d::set_error("invalid argument: %s", msg);                          \
      return VES3D_ERR_ARG;                                                     \
    }                                                                           \
  } while (0)

// NVTX range over a scope ("ves3d <phase>"), for timelines in a profiler; without one
// attached the push and pop do nothing (NVTX 3 is header-only).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

constexpr double kInv8Pi = 0.039788735772973836;  // 1/(8 pi)
constexpr double kDl = 0.238732414637843;         // 3/(4 pi), the double-layer kernel's constant

// Hardware reciprocal square root in its flush-to-zero form (PTX rsqrt.approx.ftz.f32):
// no subnormal handling around the MUFU op. Every caller passes squared distances far
// inside FP32's normal range; for those it equals rsqrtf.
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// 1/sqrt(r2) in FP64 for r2 > 0: single-precision hardware seed refined by one
// third-order Newton/Householder step y <- y (1 + e/2 + 3e^2/8), e = 1 - r2 y^2
// (Householder's method of order 3 applied to f(y) = y^-2 - r2). The seed's relative
// error (~2^-23) becomes O(2^-66), i.e. the result is within rounding of 1/sqrt(r2).
// Valid for FLT_MIN < r2 < FLT_MAX. (The flush-to-zero seed gives the same bits here and
// measured no faster in the FP64 far field, which is bound by its FP64 pipe.)
// The same refinement from a seed formed without FP64 conversions: the FP32 operand is
// cut from the double's bits (exponent rebased, significand truncated to 23 bits) and the
// hardware result put back into a double by integer operations, so the FP64 pipe only
// sees the refinement (two conversions fewer per call; the seed's relative error stays
// ~2^-22, within the refinement's reach). Valid for FLT_MIN <= r2 < FLT_MAX; a caller
// treats smaller r2 (below 2^-126) as a coincident pair.
__device__ __forceinline__ double rsqrt_f64_int_seed(double r2) {
  constexpr int kRebias = (1023 - 127) << 20;  // exponent bias difference, in the high word
  const unsigned fb = __funnelshift_l((unsigned)__double2loint(r2), (unsigned)(__double2hiint(r2) - kRebias), 3);
  const unsigned yb = __float_as_uint(rsqrt_ftz(__uint_as_float(fb)));
  const double y = __hiloint2double((int)((yb >> 3) + kRebias), (int)(yb << 29));
  const double e = fma(-r2 * y, y, 1.0);
  const double c = fma(e, 0.375, 0.5);
  return fma(y * e, c, y);
}

// Coincidence test on the high word of a squared distance: true for r2 >= 2^-126.
__device__ __forceinline__ bool r2_normal(double r2) { return __double2hiint(r2) >= 0x38100000; }

__device__ __forceinline__ double rsqrt_f64(double r2) {
  double y = (double)rsqrtf((float)r2);
  double e = fma(-r2 * y, y, 1.0);
  double c = fma(e, 0.375, 0.5);
  return fma(y * e, c, y);
}

}  // namespace ves3d
