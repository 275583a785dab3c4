// FMA-throughput probe of the benchmark (not part of the library: built on its own into
// ves3d_b200/libves3d_peak.so and loaded by bench.py only). It measures the FP64 / FP32
// CUDA-core FMA peak of the device it runs on, the denominator of the roofline of the
// direct-sum kernels (which are bound by those pipes, not by HBM or tensor cores). Eight
// independent FMA chains per thread, enough CTAs to fill every SM several times over.
#include <cuda_runtime.h>

namespace {

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

}  // namespace

// Returns 0 and the measured TFLOP/s (2 flops per FMA) in *tflops, or the CUDA error code.
extern "C" int ves3d_bench_fma_peak(int fp64, double* tflops) {
  if (!tflops) return -1;
  int dev = 0, nsm = 0;
  cudaError_t e;
  if ((e = cudaGetDevice(&dev)) || (e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev))) return e;
  const int blocks = nsm * 8, threads = 256, iters = 2048;
  void* out = nullptr;
  if ((e = cudaMalloc(&out, blocks * sizeof(double)))) return e;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float best = 1e30f;
  if (!(e = cudaEventCreate(&e0)) && !(e = cudaEventCreate(&e1))) {
    for (int rep = 0; rep < 4 && !e; rep++) {
      cudaEventRecord(e0);
      if (fp64)
        k_fma_probe<double><<<blocks, threads>>>((double*)out, iters, 0.999999, 1e-7);
      else
        k_fma_probe<float><<<blocks, threads>>>((float*)out, iters, 0.999999f, 1e-7f);
      if ((e = cudaGetLastError())) break;
      cudaEventRecord(e1);
      if ((e = cudaEventSynchronize(e1))) break;
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0 && ms < best) best = ms;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(out);
  if (e) return e;
  const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
  *tflops = flops / (best * 1e-3) / 1e12;
  return 0;
}
