// FMA-throughput probe: measures the FP64 / FP32 CUDA-core FMA peak of the device it
// runs on, the denominator of the roofline of the direct-sum kernels (which are bound
// by those pipes, not by HBM or tensor cores). Eight independent FMA chains per
// thread, enough CTAs to fill every SM several times over.
#include "common.cuh"
#include "kernels.h"

namespace ves3d {

template <class T>
__global__ void __launch_bounds__(256) k_fma_probe(T* out, int iters, T a, T b) {
  T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
      x0 = fma(x0, a, b);
      x1 = fma(x1, a, b);
      x2 = fma(x2, a, b);
      x3 = fma(x3, a, b);
      x4 = fma(x4, a, b);
      x5 = fma(x5, a, b);
      x6 = fma(x6, a, b);
      x7 = fma(x7, a, b);
    }
  }
  T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == (T)-1.2345) out[blockIdx.x] = s;  // keeps the chains live
}

}  // namespace ves3d

using namespace ves3d;

extern "C" int ves3d_measure_fma_peak(int fp64, double* tflops) {
  VES3D_ARG(tflops != nullptr, "tflops is null");
  int dev = 0, nsm = 0;
  VES3D_CK(cudaGetDevice(&dev));
  VES3D_CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = nsm * 8, threads = 256, iters = 2048;
  void* out = nullptr;
  VES3D_CK(cudaMalloc(&out, blocks * sizeof(double)));
  cudaEvent_t e0, e1;
  VES3D_CK(cudaEventCreate(&e0));
  VES3D_CK(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int rep = 0; rep < 4; rep++) {
    VES3D_CK(cudaEventRecord(e0));
    if (fp64)
      k_fma_probe<double><<<blocks, threads>>>((double*)out, iters, 0.999999, 1e-7);
    else
      k_fma_probe<float><<<blocks, threads>>>((float*)out, iters, 0.999999f, 1e-7f);
    VES3D_LAUNCHED();
    VES3D_CK(cudaEventRecord(e1));
    VES3D_CK(cudaEventSynchronize(e1));
    float ms = 0;
    VES3D_CK(cudaEventElapsedTime(&ms, e0, e1));
    if (rep > 0 && ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
  *tflops = flops / (best * 1e-3) / 1e12;
  return VES3D_OK;
}
