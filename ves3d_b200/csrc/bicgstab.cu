// BiCGStab on device vectors (FP64), the reference's iteration
// (BiCGStab<Container, MatVec, Precond>::operator(), src/BiCGStab.cc:45-138): right
// preconditioning phat = P p, shat = P s (identity when no preconditioner is given), same
// update order, same tests on the unpreconditioned residual (initial residual <= tol;
// afterwards s- and r-residuals < tol), same breakdown codes (BiCGSReturn,
// include/BiCGStab.h:19-23). Dot products are two-pass block reductions in a fixed
// order, so a solve is deterministic run to run. Scalars come back to the host once per
// dot product (the loop is host-driven; the matvec is the expensive part).
#include <cmath>

#include "common.cuh"
#include "kernels.h"

namespace ves3d {

constexpr int kDotBlocks = 592;  // 4 per SM on a B200
constexpr int kDotThreads = 256;

__global__ void __launch_bounds__(kDotThreads) k_dot_partial(const double* __restrict__ x, const double* __restrict__ y,
                                                             long n, double* __restrict__ part) {
  __shared__ double red[kDotThreads / 32];
  double s = 0.0;
  for (long i = (long)blockIdx.x * kDotThreads + threadIdx.x; i < n; i += (long)gridDim.x * kDotThreads)
    s = fma(x[i], y[i], s);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kDotThreads / 32; w++) t += red[w];
    part[blockIdx.x] = t;
  }
}

__global__ void k_dot_final(const double* __restrict__ part, int np, double* __restrict__ out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) s += part[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (blockDim.x + 31) / 32; w++) t += red[w];
    *out = t;
  }
}

// out = a*x + b*y (+ c*z if z)
__global__ void k_lincomb(long n, double a, const double* __restrict__ x, double b, const double* __restrict__ y,
                          double c, const double* __restrict__ z, double* __restrict__ out) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double s = a * x[i] + b * y[i];
    if (z) s += c * z[i];
    out[i] = s;
  }
}

// p = r + beta (p - omega v)
__global__ void k_p_update(long n, const double* __restrict__ r, double beta, double omega, const double* __restrict__ v,
                           double* __restrict__ p) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    p[i] = r[i] + beta * (p[i] - omega * v[i]);
}

static unsigned grid_for(long n) {
  long b = (n + 255) / 256;
  return (unsigned)(b < 1184 ? (b < 1 ? 1 : b) : 1184);
}

int dot_f64(const double* x, const double* y, long n, double* scratch, double* result, cudaStream_t st) {
  k_dot_partial<<<kDotBlocks, kDotThreads, 0, st>>>(x, y, n, scratch);
  VES3D_LAUNCHED();
  k_dot_final<<<1, 256, 0, st>>>(scratch, kDotBlocks, scratch + kDotBlocks);
  VES3D_LAUNCHED();
  VES3D_CK(cudaMemcpyAsync(result, scratch + kDotBlocks, sizeof(double), cudaMemcpyDeviceToHost, st));
  VES3D_CK(cudaStreamSynchronize(st));
  return VES3D_OK;
}

int lincomb_f64(long n, double a, const double* x, double b, const double* y, double c, const double* z, double* out,
                cudaStream_t st) {
  if (n <= 0) return VES3D_OK;
  k_lincomb<<<grid_for(n), 256, 0, st>>>(n, a, x, b, y, c, z, out);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

size_t bicgstab_workspace_doubles(long n) { return (size_t)9 * n + kDotBlocks + 8; }

double* bicgstab_dot_scratch(double* ws, long n) { return ws + 9 * n; }

int bicgstab_run(MatVecFn A, void* ctx, double* x, const double* b, long n, double* tol, int* max_iter, int* code,
                 double* ws, cudaStream_t st, MatVecFn P, void* pctx) {
  double* p = ws;
  double* s = ws + n;
  double* t = ws + 2 * n;
  double* v = ws + 3 * n;
  double* r = ws + 4 * n;
  double* rt = ws + 5 * n;
  double* ax = ws + 6 * n;
  double* phat = P ? ws + 7 * n : p;
  double* shat = P ? ws + 8 * n : s;
  double* dscr = bicgstab_dot_scratch(ws, n);
  int st_;
  const double tol_in = *tol;
  const int iter_max = *max_iter;
  double nb2 = 0;
  if ((st_ = dot_f64(b, b, n, dscr, &nb2, st))) return st_;
  double normb = std::sqrt(nb2);
  if (normb == 0.0) normb = 1.0;
  if ((st_ = A(ctx, x, ax))) return st_;
  if ((st_ = lincomb_f64(n, 1.0, b, -1.0, ax, 0, nullptr, r, st))) return st_;
  VES3D_CK(cudaMemcpyAsync(rt, r, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  double rr = 0;
  if ((st_ = dot_f64(r, r, n, dscr, &rr, st))) return st_;
  double resid = std::sqrt(rr) / normb;
  if (resid <= tol_in) {
    *tol = resid;
    *max_iter = 0;
    *code = 100;
    return VES3D_OK;
  }
  double rho2 = 1.0, alpha = 1.0, omega = 1.0;
  for (int i = 1; i <= iter_max; i++) {
    if (resid != resid) {
      *tol = resid;
      *max_iter = i;
      *code = 104;
      return VES3D_OK;
    }
    double rho1 = 0;
    if ((st_ = dot_f64(rt, r, n, dscr, &rho1, st))) return st_;
    if (rho1 == 0) {
      if ((st_ = dot_f64(r, r, n, dscr, &rr, st))) return st_;
      *tol = std::sqrt(rr) / normb;
      *max_iter = i;
      *code = 102;
      return VES3D_OK;
    }
    if (i == 1) {
      VES3D_CK(cudaMemcpyAsync(p, r, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    } else {
      const double beta = (rho1 / rho2) * (alpha / omega);
      k_p_update<<<grid_for(n), 256, 0, st>>>(n, r, beta, omega, v, p);
      VES3D_LAUNCHED();
    }
    if (P && (st_ = P(pctx, p, phat))) return st_;
    if ((st_ = A(ctx, phat, v))) return st_;
    double rtv = 0;
    if ((st_ = dot_f64(rt, v, n, dscr, &rtv, st))) return st_;
    alpha = rho1 / rtv;
    if ((st_ = lincomb_f64(n, 1.0, r, -alpha, v, 0, nullptr, s, st))) return st_;
    double ss = 0;
    if ((st_ = dot_f64(s, s, n, dscr, &ss, st))) return st_;
    resid = std::sqrt(ss) / normb;
    if (resid < tol_in) {
      if ((st_ = lincomb_f64(n, 1.0, x, alpha, phat, 0, nullptr, x, st))) return st_;
      *tol = resid;
      *max_iter = i;
      *code = 100;
      return VES3D_OK;
    }
    if (P && (st_ = P(pctx, s, shat))) return st_;
    if ((st_ = A(ctx, shat, t))) return st_;
    double ts = 0, tt = 0;
    if ((st_ = dot_f64(t, s, n, dscr, &ts, st))) return st_;
    if ((st_ = dot_f64(t, t, n, dscr, &tt, st))) return st_;
    omega = ts / tt;
    if ((st_ = lincomb_f64(n, 1.0, x, alpha, phat, omega, shat, x, st))) return st_;
    if ((st_ = lincomb_f64(n, 1.0, s, -omega, t, 0, nullptr, r, st))) return st_;
    rho2 = rho1;
    if ((st_ = dot_f64(r, r, n, dscr, &rr, st))) return st_;
    resid = std::sqrt(rr) / normb;
    if (resid < tol_in) {
      *tol = resid;
      *max_iter = i;
      *code = 100;
      return VES3D_OK;
    }
    if (omega == 0) {
      *tol = resid;
      *max_iter = i;
      *code = 103;
      return VES3D_OK;
    }
  }
  *tol = resid;
  *max_iter = iter_max;
  *code = 101;
  return VES3D_OK;
}

}  // namespace ves3d

using namespace ves3d;

extern "C" int ves3d_bicgstab_f64(ves3d_matvec_fn A, void* ctx, double* x, const double* b, size_t n, double* tol,
                                  int* max_iter, int* code, void* stream) {
  VES3D_ARG(A && x && b && tol && max_iter && code, "null argument");
  VES3D_ARG(n > 0 && *max_iter >= 0, "bad sizes");
  cudaStream_t st = (cudaStream_t)stream;
  double* ws = nullptr;
  VES3D_CK(cudaMalloc((void**)&ws, bicgstab_workspace_doubles((long)n) * sizeof(double)));
  int s = bicgstab_run(A, ctx, x, b, (long)n, tol, max_iter, code, ws, st, nullptr, nullptr);
  // an asynchronous fault of the last queued work surfaces here; report it unless the
  // solve already failed
  const cudaError_t e = cudaStreamSynchronize(st);
  cudaFree(ws);
  if (!s && e != cudaSuccess) {
    set_error("CUDA error %s after the solve", cudaGetErrorString(e));
    s = VES3D_ERR_CUDA;
  }
  return s;
}
