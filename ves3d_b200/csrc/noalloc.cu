// All-to-all Stokes interaction that allocates nothing.
//
// Some callers of this library cannot call cudaMalloc: host programs whose device
// memory is owned by another allocator (a pool that has already reserved the GPU, or a
// framework that forbids raw cudaMalloc/cudaFree churn between time steps).
// ves3d_stokes_alltoall_f64 stages its inputs through a workspace it allocates on first
// use; this variant stages them through a fixed, file-scope device array instead.
//
// The call is synchronous: it copies host arrays in, runs the sum and waits for the
// result on the caller's stream before it returns.
//
// The array holds VES3D_NOALLOC_MAX_POINTS points (source, density and result, three
// doubles each: 36 MiB). Every GPU that loads the library holds it until the process
// exits. Every call shares it and it keeps the last call's contents; nothing in it has
// to start at zero (each call overwrites the parts it reads). Calls whose GPU work
// overlaps (other host threads, or streams that run concurrently) race on the array.
// The first call on each device does the set-up: with that device current it looks up
// the array's device address (cudaGetSymbolAddress; host code may not use the array's
// name as a device pointer) and keeps it for the life of the process. Make that first
// call before any stream capture. The kept address does not survive cudaDeviceReset.
#include <cmath>
#include <mutex>

#include "common.cuh"
#include "kernels.h"

namespace ves3d {

// sources [max][3], densities [max][3], results [max][3]
static __device__ __align__(256) double g_noalloc_scratch[(size_t)VES3D_NOALLOC_MAX_POINTS * 9];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_addr[kMaxDevices] = {nullptr};

// Device address of the array on the current device, looked up once per device.
int scratch_address(double** out) {
  int dev = 0;
  VES3D_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device index %d beyond the %d devices this entry point supports", dev, kMaxDevices);
    return VES3D_ERR_NODEV;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    VES3D_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_addr[dev] = (double*)p;
  }
  *out = g_addr[dev];
  return VES3D_OK;
}
}  // namespace

}  // namespace ves3d

using namespace ves3d;

namespace {
// Copies in, the sum, the copy out and the wait; a failure returns at once (the caller
// fills the result with NaN after waiting for what was queued).
int noalloc_body(const double* src, const double* den, size_t np, double* pot, cudaStream_t st) {
  double* base = nullptr;
  int s = scratch_address(&base);
  if (s) return s;
  double* dsrc = base;
  double* dden = base + (size_t)3 * VES3D_NOALLOC_MAX_POINTS;
  double* dpot = base + (size_t)6 * VES3D_NOALLOC_MAX_POINTS;
  VES3D_CK(cudaMemcpyAsync(dsrc, src, 3 * np * sizeof(double), cudaMemcpyHostToDevice, st));
  VES3D_CK(cudaMemcpyAsync(dden, den, 3 * np * sizeof(double), cudaMemcpyHostToDevice, st));
  if ((s = launch_alltoall_f64(dsrc, dden, (long)np, dpot, st))) return s;
  VES3D_CK(cudaMemcpyAsync(pot, dpot, 3 * np * sizeof(double), cudaMemcpyDeviceToHost, st));
  VES3D_CK(cudaStreamSynchronize(st));
  return VES3D_OK;
}
}  // namespace

extern "C" int ves3d_stokes_alltoall_noalloc_f64(const double* src, const double* den, size_t np, double* pot,
                                                 void* stream) {
  // like ves3d_stokes_alltoall_f64: on any error pot (when given) is filled with NaN
  const auto fail_nan = [&](int status) {
    if (pot)
      for (size_t i = 0; i < 3 * np; i++) pot[i] = NAN;
    return status;
  };
  if (!(src && den && pot)) {
    set_error("invalid argument: null pointer");
    return fail_nan(VES3D_ERR_ARG);
  }
  if (np == 0) return VES3D_OK;  // nothing to compute; pot is left as it is
  if (np > (size_t)VES3D_NOALLOC_MAX_POINTS) {
    set_error("invalid argument: np = %zu exceeds VES3D_NOALLOC_MAX_POINTS = %d, the capacity of the fixed "
              "device array this entry point uses; call ves3d_stokes_alltoall_f64 instead",
              np, VES3D_NOALLOC_MAX_POINTS);
    return fail_nan(VES3D_ERR_ARG);
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int s = noalloc_body(src, den, np, pot, st);
  if (s) {
    // let copies already queued on the stream finish before the host result is touched
    cudaStreamSynchronize(st);
    return fail_nan(s);
  }
  return VES3D_OK;
}
