// Device<GPU> primitives of the reference's plugin surface (include/Device.h:81-253) that a
// caller of the operators uses around them: axpy, AlgebraicDot, Transpose, Reduce (the
// smooth surface integral of GLIntegrator) and gemm (column-major BLAS semantics, cuBLAS).
// Device pointers, the given stream; every entry point returns when its work is done.
#include <cublas_v2.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace ves3d {

// out[j * height + i] = in[i * width + j] through 32 x 33 shared-memory tiles (coalesced
// reads and writes); grid-stride over tiles
__global__ void k_transpose(const double* __restrict__ in, long height, long width, double* __restrict__ out) {
  __shared__ double tile[32][33];
  const long tiles_h = (height + 31) / 32, tiles_w = (width + 31) / 32;
  for (long tix = blockIdx.x; tix < tiles_h * tiles_w; tix += gridDim.x) {
    const long ti = tix / tiles_w, tj = tix - ti * tiles_w;
    const long i0 = ti * 32, j0 = tj * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const long i = i0 + r, j = j0 + threadIdx.x;
      tile[r][threadIdx.x] = (i < height && j < width) ? in[i * width + j] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const long j = j0 + r, i = i0 + threadIdx.x;
      if (j < width && i < height) out[j * height + i] = tile[threadIdx.x][r];
    }
    __syncthreads();
  }
}

// x_dw[s * x_dim + d] = sum_i x[(s * x_dim + d) * stride + i] w[s * stride + i] qw[i], or with
// x null sum_i w[s * stride + i] qw[i] (Device<CPU>::Reduce, src/DeviceCPU.cc:444-497): one
// CTA per (surface, component), fixed-order tree (deterministic)
__global__ void k_reduce(const double* __restrict__ x, int x_dim, const double* __restrict__ w,
                         const double* __restrict__ qw, long stride, double* __restrict__ x_dw) {
  __shared__ double red[256];
  const long s = blockIdx.x / x_dim;
  const int d = (int)(blockIdx.x - s * x_dim);
  double acc = 0.0;
  for (long i = threadIdx.x; i < stride; i += blockDim.x) {
    const double v = w[s * stride + i] * qw[i];
    acc += x ? x[(s * x_dim + d) * stride + i] * v : v;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) x_dw[blockIdx.x] = red[0];
}

// Device::AggregateRotation for one longitude jj and one operand (include/Device.h:234-237,
// src/DeviceCPU.cc:646-680): res = Permute(mat, jj) . vec in column-major BLAS terms, where
// Permute shifts the columns of every latitude block of the np x np matrix mat by jj
// (CircShift / PermuteGpu, src/CudaKernels.cu:2286-2310). Equivalently
//   res[s][row] = sum_c mat[c][row] vec[s][lat(c) nlong + (lon(c) + jj) mod nlong],
// computed here without forming the permuted matrix: one thread per (row, column s), the
// shifted column s staged in shared memory, mat read column by column (coalesced rows).
__global__ void k_aggregate_rotation(const double* __restrict__ mat, int nlat, int nlong, int jj,
                                     const double* __restrict__ vec, double* __restrict__ res) {
  extern __shared__ double sw[];  // [np] shifted column
  const int np = nlat * nlong;
  const long sc = blockIdx.y;
  for (int c = threadIdx.x; c < np; c += blockDim.x) {
    const int lat = c / nlong, lon = c - lat * nlong;
    sw[c] = vec[sc * np + lat * nlong + (lon + jj) % nlong];
  }
  __syncthreads();
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= np) return;
  double a0 = 0.0, a1 = 0.0;
  int c = 0;
  for (; c + 1 < np; c += 2) {
    a0 = fma(mat[(long)c * np + row], sw[c], a0);
    a1 = fma(mat[(long)(c + 1) * np + row], sw[c + 1], a1);
  }
  if (c < np) a0 = fma(mat[(long)c * np + row], sw[c], a0);
  res[sc * np + row] = a0 + a1;
}

int launch_aggregate_rotation(const double* mat, int nlat, int nlong, int jj, const double* vec, int nsub,
                              double* res, cudaStream_t st) {
  const int np = nlat * nlong;
  if (np <= 0 || nsub <= 0) return VES3D_OK;
  dim3 grid((np + 127) / 128, nsub);
  k_aggregate_rotation<<<grid, 128, np * sizeof(double), st>>>(mat, nlat, nlong, jj, vec, res);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

namespace {

// one cuBLAS handle per device, created on first use and kept until exit; a mutex
// serialises its use (the stream is set per call)
struct BlasHandles {
  std::mutex mu;
  cublasHandle_t h[64] = {};
};

BlasHandles& blas_handles() {
  static BlasHandles* b = new BlasHandles();  // intentionally never freed
  return *b;
}

int blas_status(cublasStatus_t s, const char* what) {
  if (s == CUBLAS_STATUS_SUCCESS) return VES3D_OK;
  set_error("%s failed (cuBLAS status %d)", what, (int)s);
  return s == CUBLAS_STATUS_INVALID_VALUE ? VES3D_ERR_ARG : VES3D_ERR_CUDA;
}

bool blas_op(char c, cublasOperation_t* op) {
  if (c == 'N' || c == 'n') *op = CUBLAS_OP_N;
  else if (c == 'T' || c == 't') *op = CUBLAS_OP_T;
  else if (c == 'C' || c == 'c') *op = CUBLAS_OP_C;
  else return false;
  return true;
}

}  // namespace

}  // namespace ves3d

using namespace ves3d;

extern "C" {

int ves3d_dev_axpy(double a, const double* x, const double* y, size_t length, double* out, void* stream) {
  VES3D_ARG(x && y && out, "null pointer");
  if (length == 0) return VES3D_OK;
  cudaStream_t st = (cudaStream_t)stream;
  int s = lincomb_f64((long)length, a, x, 1.0, y, 0.0, nullptr, out, st);
  if (s) return s;
  VES3D_CK(cudaStreamSynchronize(st));
  return VES3D_OK;
}

int ves3d_dev_algebraic_dot(const double* x, const double* y, size_t length, double* result, void* stream) {
  VES3D_ARG(x && y && result, "null pointer");
  if (length == 0) {
    *result = 0.0;
    return VES3D_OK;
  }
  double* scratch = nullptr;
  VES3D_CK(cudaMalloc((void**)&scratch, 1024 * sizeof(double)));  // the dot's block partials
  const int s = dot_f64(x, y, (long)length, scratch, result, (cudaStream_t)stream);
  cudaFree(scratch);
  return s;
}

int ves3d_dev_transpose(const double* in, size_t height, size_t width, double* out, void* stream) {
  VES3D_ARG(in && out, "null pointer");
  VES3D_ARG(in != out || height * width == 0, "transpose is out of place");
  if (height == 0 || width == 0) return VES3D_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const long tiles = (long)((height + 31) / 32) * (long)((width + 31) / 32);
  const unsigned grid = (unsigned)std::min(tiles, 65535L);
  k_transpose<<<grid, dim3(32, 8), 0, st>>>(in, (long)height, (long)width, out);
  VES3D_LAUNCHED();
  VES3D_CK(cudaStreamSynchronize(st));
  return VES3D_OK;
}

int ves3d_dev_reduce(const double* x, int x_dim, const double* w, const double* quad_w, size_t stride, size_t ns,
                     double* x_dw, void* stream) {
  VES3D_ARG(w && quad_w && x_dw, "null pointer");
  VES3D_ARG(x == nullptr || x_dim >= 1, "x_dim must be >= 1");
  if (ns == 0) return VES3D_OK;
  const int dim = x ? x_dim : 1;
  VES3D_ARG((double)ns * dim < 2147483647.0, "too many integrals");
  cudaStream_t st = (cudaStream_t)stream;
  k_reduce<<<(unsigned)(ns * dim), 256, 0, st>>>(x, dim, w, quad_w, (long)stride, x_dw);
  VES3D_LAUNCHED();
  VES3D_CK(cudaStreamSynchronize(st));
  return VES3D_OK;
}

int ves3d_dev_gemm(char trans_a, char trans_b, int m, int n, int k, double alpha, const double* A, int lda,
                   const double* B, int ldb, double beta, double* C, int ldc, void* stream) {
  cublasOperation_t oa, ob;
  VES3D_ARG(blas_op(trans_a, &oa) && blas_op(trans_b, &ob), "trans must be 'N', 'T' or 'C'");
  VES3D_ARG(m >= 0 && n >= 0 && k >= 0, "negative dimension");
  VES3D_ARG(C != nullptr && (k == 0 || (A && B)), "null pointer");
  if (m == 0 || n == 0) return VES3D_OK;
  int dev = 0;
  VES3D_CK(cudaGetDevice(&dev));
  BlasHandles& bh = blas_handles();
  std::lock_guard<std::mutex> lk(bh.mu);
  cublasHandle_t& h = bh.h[(unsigned)dev % 64];
  int s;
  if (!h && (s = blas_status(cublasCreate(&h), "cublasCreate"))) {
    h = nullptr;
    return s;
  }
  cudaStream_t st = (cudaStream_t)stream;
  if ((s = blas_status(cublasSetStream(h, st), "cublasSetStream"))) return s;
  if ((s = blas_status(cublasDgemm(h, oa, ob, m, n, k, &alpha, A, lda, B, ldb, &beta, C, ldc), "cublasDgemm")))
    return s;
  VES3D_CK(cudaStreamSynchronize(st));
  return VES3D_OK;
}

int ves3d_dev_aggregate_rotation(int sh_order, int nlat, int nlong, int n_vec, const int* n_sub, const double* mat,
                                 const double* const* vec, double* const* wrk, double* const* res, int n_stream,
                                 void* stream) {
  (void)wrk;  // the permuted matrices are never formed (see k_aggregate_rotation)
  (void)n_stream;
  VES3D_ARG(sh_order >= 1 && nlat == sh_order + 1 && nlong == 2 * sh_order, "grid must be (p + 1) x 2p");
  VES3D_ARG(n_vec >= 0, "n_vec < 0");
  if (n_vec == 0) return VES3D_OK;
  VES3D_ARG(n_sub && mat && vec && res, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  for (int jj = 0; jj < nlong; jj++)
    for (int ii = 0; ii < n_vec; ii++) {
      VES3D_ARG(n_sub[ii] >= 0, "n_sub < 0");
      VES3D_ARG(n_sub[ii] == 0 || (vec[ii] && res[n_vec * jj + ii]), "null operand or result");
      const int s = launch_aggregate_rotation(mat, nlat, nlong, jj, vec[ii], n_sub[ii], res[n_vec * jj + ii], st);
      if (s) return s;
    }
  VES3D_CK(cudaStreamSynchronize(st));
  return VES3D_OK;
}

}  // extern "C"
