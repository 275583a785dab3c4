// FP64 direct Stokes single-layer sums (plain form) and the far-field source packing.
//
// Pair kernel (StokesAlltoAll, src/CPUKernels.cc:1011-1057; DirectStokesKernel, :123-178):
//   r = x_s - x_t,  u_t += [ d_s / |r| + (r . d_s) r / |r|^3 ] / (8 pi),
// and a coincident pair (|r| = 0) contributes nothing.
//
// (The far field with same-vesicle exclusion is in far_kernels.cu.)
#include "common.cuh"
#include "kernels.h"

namespace ves3d {

constexpr int kFarBS = 128;

struct PairAcc {
  double x = 0.0, y = 0.0, z = 0.0;
};

__device__ __forceinline__ void pair_f64(double tx, double ty, double tz, double sx, double sy, double sz, double dx_,
                                         double dy_, double dz_, bool skip, PairAcc& a) {
  const double dx = sx - tx, dy = sy - ty, dz = sz - tz;
  const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
  double rinv = rsqrt_f64(r2);
  rinv = (skip || r2 == 0.0) ? 0.0 : rinv;
  const double cc = fma(dz, dz_, fma(dy, dy_, dx * dx_)) * rinv * rinv;
  a.x = fma(fma(cc, dx, dx_), rinv, a.x);
  a.y = fma(fma(cc, dy, dy_), rinv, a.y);
  a.z = fma(fma(cc, dz, dz_), rinv, a.z);
}

// All pairs, point-major in and out.
__global__ void __launch_bounds__(kFarBS) k_alltoall_f64(const double* __restrict__ pos, const double* __restrict__ den,
                                                         long N, double* __restrict__ pot) {
  __shared__ double sp[kFarBS * 3];
  __shared__ double sd[kFarBS * 3];
  const long g = (long)blockIdx.x * kFarBS + threadIdx.x;
  const bool active = g < N;
  double tx = 0, ty = 0, tz = 0;
  if (active) {
    tx = pos[3 * g];
    ty = pos[3 * g + 1];
    tz = pos[3 * g + 2];
  }
  PairAcc acc;
  for (long s0 = 0; s0 < N; s0 += kFarBS) {
    const int ns = (int)min((long)kFarBS, N - s0);
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * ns; i += kFarBS) {
      sp[i] = pos[3 * s0 + i];
      sd[i] = den[3 * s0 + i];
    }
    __syncthreads();
    if (!active) continue;
#pragma unroll 4
    for (int k = 0; k < ns; k++)
      pair_f64(tx, ty, tz, sp[3 * k], sp[3 * k + 1], sp[3 * k + 2], sd[3 * k], sd[3 * k + 1], sd[3 * k + 2], false,
               acc);
  }
  if (!active) return;
  pot[3 * g] = acc.x * kInv8Pi;
  pot[3 * g + 1] = acc.y * kInv8Pi;
  pot[3 * g + 2] = acc.z * kInv8Pi;
}

int launch_alltoall_f64(const double* pos, const double* den, long np, double* pot, cudaStream_t st) {
  if (np <= 0) return VES3D_OK;
  k_alltoall_f64<<<(unsigned)((np + kFarBS - 1) / kFarBS), kFarBS, 0, st>>>(pos, den, np, pot);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

// Device<GPU>::DirectStokes / cuda_stokes (src/CudaKernels.cu:1840-1916, 1996-2006):
// per surface v, targets t in [t_head, t_tail) of T[v] (stride trg_m), sources all
// src_m points of S[v] with density D * Q. grid = (target chunks, n surfaces).
__global__ void __launch_bounds__(kFarBS) k_direct_stokes_f64(int src_m, int trg_m, int t_head, int t_tail,
                                                              const double* __restrict__ T,
                                                              const double* __restrict__ S,
                                                              const double* __restrict__ D, double* __restrict__ U,
                                                              const double* __restrict__ Q) {
  __shared__ double sp[kFarBS * 3];
  __shared__ double sd[kFarBS * 3];
  const long v = blockIdx.y;
  const int t = t_head + blockIdx.x * kFarBS + threadIdx.x;
  const bool active = t < t_tail;
  const double* Tv = T + v * 3 * (long)trg_m;
  const double* Sv = S + v * 3 * (long)src_m;
  const double* Dv = D + v * 3 * (long)src_m;
  double tx = 0, ty = 0, tz = 0;
  if (active) {
    tx = Tv[t];
    ty = Tv[trg_m + t];
    tz = Tv[2 * trg_m + t];
  }
  PairAcc acc;
  for (int s0 = 0; s0 < src_m; s0 += kFarBS) {
    const int ns = min(kFarBS, src_m - s0);
    __syncthreads();
    for (int i = threadIdx.x; i < ns; i += kFarBS) {
      const int s = s0 + i;
      const double q = Q ? Q[s] : 1.0;
      sp[3 * i] = Sv[s];
      sp[3 * i + 1] = Sv[src_m + s];
      sp[3 * i + 2] = Sv[2 * src_m + s];
      sd[3 * i] = Dv[s] * q;
      sd[3 * i + 1] = Dv[src_m + s] * q;
      sd[3 * i + 2] = Dv[2 * src_m + s] * q;
    }
    __syncthreads();
    if (!active) continue;
    for (int k = 0; k < ns; k++)
      pair_f64(tx, ty, tz, sp[3 * k], sp[3 * k + 1], sp[3 * k + 2], sd[3 * k], sd[3 * k + 1], sd[3 * k + 2], false,
               acc);
  }
  if (!active) return;
  double* Uv = U + v * 3 * (long)trg_m;
  Uv[t] = acc.x * kInv8Pi;
  Uv[trg_m + t] = acc.y * kInv8Pi;
  Uv[2 * trg_m + t] = acc.z * kInv8Pi;
}

int launch_direct_stokes_f64(int src_m, int trg_m, int n, int t_head, int t_tail, const double* T,
                             const double* S, const double* D, double* U, const double* Q, cudaStream_t st) {
  if (n <= 0 || t_tail <= t_head) return VES3D_OK;
  dim3 grid((t_tail - t_head + kFarBS - 1) / kFarBS, n);
  k_direct_stokes_f64<<<grid, kFarBS, 0, st>>>(src_m, trg_m, t_head, t_tail, T, S, D, U, Q);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

// The single-precision overload of cuda_stokes (src/CudaKernels.cu:594-761, the kernel
// `stokes` on float arrays, used by SINGLE_PREC builds of the reference): FP32 inputs and
// outputs and FP32 pair arithmetic (hardware reciprocal square root, a coincident pair
// contributes nothing), each thread's FP32 sum over a tile of 128 sources added into an
// FP64 accumulator. Q may be NULL (unit weights), as in the reference's second kernel.
__global__ void __launch_bounds__(kFarBS) k_direct_stokes_f32(int src_m, int trg_m, int t_head, int t_tail,
                                                              const float* __restrict__ T,
                                                              const float* __restrict__ S,
                                                              const float* __restrict__ D, float* __restrict__ U,
                                                              const float* __restrict__ Q) {
  __shared__ float sp[kFarBS * 3];
  __shared__ float sd[kFarBS * 3];
  const long v = blockIdx.y;
  const int t = t_head + blockIdx.x * kFarBS + threadIdx.x;
  const bool active = t < t_tail;
  const float* Tv = T + v * 3 * (long)trg_m;
  const float* Sv = S + v * 3 * (long)src_m;
  const float* Dv = D + v * 3 * (long)src_m;
  float tx = 0.f, ty = 0.f, tz = 0.f;
  if (active) {
    tx = Tv[t];
    ty = Tv[trg_m + t];
    tz = Tv[2 * trg_m + t];
  }
  double ax = 0.0, ay = 0.0, az = 0.0;
  for (int s0 = 0; s0 < src_m; s0 += kFarBS) {
    const int ns = min(kFarBS, src_m - s0);
    __syncthreads();
    for (int i = threadIdx.x; i < ns; i += kFarBS) {
      const int s = s0 + i;
      const float q = Q ? Q[s] : 1.f;
      sp[3 * i] = Sv[s];
      sp[3 * i + 1] = Sv[src_m + s];
      sp[3 * i + 2] = Sv[2 * src_m + s];
      sd[3 * i] = Dv[s] * q;
      sd[3 * i + 1] = Dv[src_m + s] * q;
      sd[3 * i + 2] = Dv[2 * src_m + s] * q;
    }
    __syncthreads();
    if (!active) continue;
    float ux = 0.f, uy = 0.f, uz = 0.f;
    for (int k = 0; k < ns; k++) {
      const float dx = sp[3 * k] - tx, dy = sp[3 * k + 1] - ty, dz = sp[3 * k + 2] - tz;
      const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
      const float rinv = r2 > 0.f ? rsqrtf(r2) : 0.f;
      const float cc = fmaf(dz, sd[3 * k + 2], fmaf(dy, sd[3 * k + 1], dx * sd[3 * k])) * rinv * rinv;
      ux = fmaf(fmaf(cc, dx, sd[3 * k]), rinv, ux);
      uy = fmaf(fmaf(cc, dy, sd[3 * k + 1]), rinv, uy);
      uz = fmaf(fmaf(cc, dz, sd[3 * k + 2]), rinv, uz);
    }
    ax += ux;
    ay += uy;
    az += uz;
  }
  if (!active) return;
  float* Uv = U + v * 3 * (long)trg_m;
  Uv[t] = (float)(ax * kInv8Pi);
  Uv[trg_m + t] = (float)(ay * kInv8Pi);
  Uv[2 * trg_m + t] = (float)(az * kInv8Pi);
}

int launch_direct_stokes_f32(int src_m, int trg_m, int n, int t_head, int t_tail, const float* T, const float* S,
                             const float* D, float* U, const float* Q, cudaStream_t st) {
  if (n <= 0 || t_tail <= t_head) return VES3D_OK;
  dim3 grid((t_tail - t_head + kFarBS - 1) / kFarBS, n);
  k_direct_stokes_f32<<<grid, kFarBS, 0, st>>>(src_m, trg_m, t_head, t_tail, T, S, D, U, Q);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

// Double-layer pair (DirectStokesDoubleLayerKernel, src/CPUKernels.cc:1060-1120;
// stokes_double_layer, src/CudaKernels.cu:783-868): r = x_t - x_s,
// u_t += (r . n_s)(r . d_s) r / |r|^5, scaled by 3/(4 pi) after the sum; a coincident pair
// contributes nothing.
__device__ __forceinline__ void pair_dl_f64(double tx, double ty, double tz, const double* sp, const double* sn,
                                            const double* sd, PairAcc& a) {
  const double dx = tx - sp[0], dy = ty - sp[1], dz = tz - sp[2];
  const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
  double rinv = rsqrt_f64(r2);
  rinv = r2 > 0.0 ? rinv : 0.0;
  const double rinv2 = rinv * rinv;
  const double q = fma(dz, sn[2], fma(dy, sn[1], dx * sn[0])) * fma(dz, sd[2], fma(dy, sd[1], dx * sd[0])) *
                   (rinv2 * rinv2 * rinv);
  a.x = fma(dx, q, a.x);
  a.y = fma(dy, q, a.y);
  a.z = fma(dz, q, a.z);
}

// Device<GPU>::DirectStokesDoubleLayer / cuda_stokes_double_layer (src/CudaKernels.cu:895-918,
// src/DeviceGPU.cc:263-271): per surface v, targets t in [t_head, t_tail) of T[v] (stride
// trg_m), sources all src_m points of S[v] with normals N and densities D (times Q when
// given). grid = (target chunks, n surfaces).
__global__ void __launch_bounds__(kFarBS) k_direct_stokes_dl_f64(int src_m, int trg_m, int t_head, int t_tail,
                                                                 const double* __restrict__ T,
                                                                 const double* __restrict__ S,
                                                                 const double* __restrict__ N,
                                                                 const double* __restrict__ D, double* __restrict__ U,
                                                                 const double* __restrict__ Q) {
  __shared__ double sp[kFarBS * 3];
  __shared__ double sn[kFarBS * 3];
  __shared__ double sd[kFarBS * 3];
  const long v = blockIdx.y;
  const int t = t_head + blockIdx.x * kFarBS + threadIdx.x;
  const bool active = t < t_tail;
  const double* Tv = T + v * 3 * (long)trg_m;
  const double* Sv = S + v * 3 * (long)src_m;
  const double* Nv = N + v * 3 * (long)src_m;
  const double* Dv = D + v * 3 * (long)src_m;
  double tx = 0, ty = 0, tz = 0;
  if (active) {
    tx = Tv[t];
    ty = Tv[trg_m + t];
    tz = Tv[2 * trg_m + t];
  }
  PairAcc acc;
  for (int s0 = 0; s0 < src_m; s0 += kFarBS) {
    const int ns = min(kFarBS, src_m - s0);
    __syncthreads();
    for (int i = threadIdx.x; i < ns; i += kFarBS) {
      const int s = s0 + i;
      const double q = Q ? Q[s] : 1.0;
      sp[3 * i] = Sv[s];
      sp[3 * i + 1] = Sv[src_m + s];
      sp[3 * i + 2] = Sv[2 * src_m + s];
      sn[3 * i] = Nv[s];
      sn[3 * i + 1] = Nv[src_m + s];
      sn[3 * i + 2] = Nv[2 * src_m + s];
      sd[3 * i] = Dv[s] * q;
      sd[3 * i + 1] = Dv[src_m + s] * q;
      sd[3 * i + 2] = Dv[2 * src_m + s] * q;
    }
    __syncthreads();
    if (!active) continue;
    for (int k = 0; k < ns; k++) pair_dl_f64(tx, ty, tz, sp + 3 * k, sn + 3 * k, sd + 3 * k, acc);
  }
  if (!active) return;
  double* Uv = U + v * 3 * (long)trg_m;
  Uv[t] = acc.x * kDl;
  Uv[trg_m + t] = acc.y * kDl;
  Uv[2 * trg_m + t] = acc.z * kDl;
}

int launch_direct_stokes_dl_f64(int src_m, int trg_m, int n, int t_head, int t_tail, const double* T,
                                const double* S, const double* N, const double* D, double* U, const double* Q,
                                cudaStream_t st) {
  if (n <= 0 || t_tail <= t_head) return VES3D_OK;
  dim3 grid((t_tail - t_head + kFarBS - 1) / kFarBS, n);
  k_direct_stokes_dl_f64<<<grid, kFarBS, 0, st>>>(src_m, trg_m, t_head, t_tail, T, S, N, D, U, Q);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

// Velocity at M off-surface targets (point-major) from all N surface points (point-major):
// the single layer of den and, with nrm, the double layer of unit normals nrm and densities
// dden (both densities times area and weights). One target per thread, sources staged in
// shared memory.
__global__ void __launch_bounds__(kFarBS) k_targets_f64(const double* __restrict__ pos, const double* __restrict__ den,
                                                        const double* __restrict__ nrm, const double* __restrict__ dden,
                                                        long N, const double* __restrict__ trg, long M,
                                                        double* __restrict__ out) {
  __shared__ double sp[kFarBS * 3];
  __shared__ double sd[kFarBS * 3];
  __shared__ double sn[kFarBS * 3];
  __shared__ double sg[kFarBS * 3];
  const long m = (long)blockIdx.x * kFarBS + threadIdx.x;
  const bool active = m < M;
  const bool dl = nrm != nullptr;
  double tx = 0, ty = 0, tz = 0;
  if (active) {
    tx = trg[3 * m];
    ty = trg[3 * m + 1];
    tz = trg[3 * m + 2];
  }
  PairAcc a, b;
  for (long s0 = 0; s0 < N; s0 += kFarBS) {
    const int ns = (int)min((long)kFarBS, N - s0);
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * ns; i += kFarBS) {
      sp[i] = pos[3 * s0 + i];
      sd[i] = den[3 * s0 + i];
      if (dl) {
        sn[i] = nrm[3 * s0 + i];
        sg[i] = dden[3 * s0 + i];
      }
    }
    __syncthreads();
    if (!active) continue;
    for (int k = 0; k < ns; k++) {
      pair_f64(tx, ty, tz, sp[3 * k], sp[3 * k + 1], sp[3 * k + 2], sd[3 * k], sd[3 * k + 1], sd[3 * k + 2], false,
               a);
      if (dl) pair_dl_f64(tx, ty, tz, sp + 3 * k, sn + 3 * k, sg + 3 * k, b);
    }
  }
  if (!active) return;
  out[3 * m] = a.x * kInv8Pi + (dl ? b.x * kDl : 0.0);
  out[3 * m + 1] = a.y * kInv8Pi + (dl ? b.y * kDl : 0.0);
  out[3 * m + 2] = a.z * kInv8Pi + (dl ? b.z * kDl : 0.0);
}

int launch_targets_f64(const double* pos, const double* den, const double* nrm, const double* dden, long N,
                       const double* trg, long M, double* out, cudaStream_t st) {
  if (M <= 0) return VES3D_OK;
  k_targets_f64<<<(unsigned)((M + kFarBS - 1) / kFarBS), kFarBS, 0, st>>>(pos, den, nrm, dden, N, trg, M, out);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

// Unit outward normals, point-major (src/StokesVelocity.cc:245-275).
__global__ void k_unit_normals(const double* __restrict__ Xt, const double* __restrict__ Xp, long nv, int p0,
                               double* __restrict__ nrm) {
  const int ng = 2 * p0 * (p0 + 1);
  const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nv * ng) return;
  const long v = g / ng;
  const int k = (int)(g - v * ng);
  const long b = v * 3 * ng + k;
  const double ax = Xt[b], ay = Xt[b + ng], az = Xt[b + 2 * ng];
  const double bx = Xp[b], by = Xp[b + ng], bz = Xp[b + 2 * ng];
  const double nx = ay * bz - az * by, ny = az * bx - ax * bz, nz = ax * by - ay * bx;
  const double inv = 1.0 / sqrt(nx * nx + ny * ny + nz * nz);
  nrm[3 * g] = nx * inv;
  nrm[3 * g + 1] = ny * inv;
  nrm[3 * g + 2] = nz * inv;
}

int launch_unit_normals(const double* Xt, const double* Xp, long nv, int p0, double* nrm, cudaStream_t st) {
  const long N = nv * ngrid_(p0);
  if (N <= 0) return VES3D_OK;
  k_unit_normals<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(Xt, Xp, nv, p0, nrm);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

// area = |X_theta x X_phi|; pos point-major; den = f * area * w[lat].
__global__ void k_far_sources(const double* __restrict__ X, const double* __restrict__ f,
                              const double* __restrict__ Xt, const double* __restrict__ Xp, long nv, int p0,
                              const double* __restrict__ w, double* __restrict__ area, double* __restrict__ pos,
                              double* __restrict__ den) {
  const int ng = 2 * p0 * (p0 + 1);
  const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nv * ng) return;
  const long v = g / ng;
  const int k = (int)(g - v * ng);
  const long b = v * 3 * ng + k;
  const double ax = Xt[b], ay = Xt[b + ng], az = Xt[b + 2 * ng];
  const double bx = Xp[b], by = Xp[b + ng], bz = Xp[b + 2 * ng];
  const double nx = ay * bz - az * by, ny = az * bx - ax * bz, nz = ax * by - ay * bx;
  const double a = sqrt(nx * nx + ny * ny + nz * nz);
  area[g] = a;
  const double q = a * w[k / (2 * p0)];
  pos[3 * g] = X[b];
  pos[3 * g + 1] = X[b + ng];
  pos[3 * g + 2] = X[b + 2 * ng];
  if (f) {
    den[3 * g] = f[b] * q;
    den[3 * g + 1] = f[b + ng] * q;
    den[3 * g + 2] = f[b + 2 * ng] * q;
  }
}

int launch_far_sources(const double* X, const double* f, const double* Xt, const double* Xp, long nv, int p0,
                       const double* smooth_w, double* area, double* pos, double* den, cudaStream_t st) {
  const long N = nv * ngrid_(p0);
  if (N <= 0) return VES3D_OK;
  k_far_sources<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(X, f, Xt, Xp, nv, p0, smooth_w, area, pos, den);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

__global__ void k_far_density(const double* __restrict__ f, const double* __restrict__ area, long nv, int p0,
                              const double* __restrict__ w, double* __restrict__ den) {
  const int ng = 2 * p0 * (p0 + 1);
  const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nv * ng) return;
  const long v = g / ng;
  const int k = (int)(g - v * ng);
  const long b = v * 3 * ng + k;
  const double q = area[g] * w[k / (2 * p0)];
  den[3 * g] = f[b] * q;
  den[3 * g + 1] = f[b + ng] * q;
  den[3 * g + 2] = f[b + 2 * ng] * q;
}

int launch_far_density(const double* f, const double* area, long nv, int p0, const double* smooth_w, double* den,
                       cudaStream_t st) {
  const long N = nv * ngrid_(p0);
  if (N <= 0) return VES3D_OK;
  k_far_density<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(f, area, nv, p0, smooth_w, den);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

__global__ void k_scale_vesicles(const double* __restrict__ x, long n, long per, const double* __restrict__ c, long nc,
                                 const double* __restrict__ z, double beta, double* __restrict__ out) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v = c[(i / per) % nc] * x[i];
  out[i] = z ? fma(beta, z[i], v) : v;
}

int launch_scale_vesicles(const double* x, long n, long per, const double* c, long nc, const double* z, double beta,
                          double* out, cudaStream_t st) {
  if (n <= 0) return VES3D_OK;
  k_scale_vesicles<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, n, per, c, nc, z, beta, out);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

__global__ void k_add(const double* __restrict__ a, const double* __restrict__ b, long n, double* __restrict__ out) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] + b[i];
}

int launch_add(const double* a, const double* b, long n, double* out, cudaStream_t st) {
  if (n <= 0) return VES3D_OK;
  k_add<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, b, n, out);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

}  // namespace ves3d
