// All-to-all Stokes interaction that allocates nothing.
//
// Some callers of this library cannot call cudaMalloc: host programs whose device
// memory is owned by another allocator (a pool that has already reserved the GPU, or a
// framework that forbids raw cudaMalloc/cudaFree churn between time steps).
// ves3d_stokes_alltoall_f64 stages its inputs through a workspace it allocates on first
// use; this variant stages them through a fixed, file-scope device array instead.
//
// The call is synchronous: it copies host arrays in, runs the sum and waits for the
// result on the caller's stream before it returns, so it cannot be recorded into a
// CUDA graph.
//
// The array holds VES3D_NOALLOC_MAX_POINTS points (source, density and result, three
// doubles each: 36 MiB). Every GPU that loads the library holds it until the process
// exits. Every call shares it and it keeps the last call's contents; nothing in it has
// to start at zero (each call overwrites the parts it reads). Calls whose GPU work
// overlaps (other host threads, or streams that run concurrently) race on the array.
// The array's address is looked up on every call, so the entry point keeps working after
// the device's context is torn down and rebuilt (cudaDeviceReset).
#include <cmath>

#include "common.cuh"
#include "kernels.h"

namespace ves3d {

// sources [max][3], densities [max][3], results [max][3]
static __device__ __align__(256) double g_noalloc_scratch[(size_t)VES3D_NOALLOC_MAX_POINTS * 9];

namespace {
// Device address of the array on the current device, looked up on every call (cheap; a
// cached address would go stale when the device's context is torn down and rebuilt).
int scratch_address(double** out) {
  void* p = nullptr;
  VES3D_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
  *out = (double*)p;
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
