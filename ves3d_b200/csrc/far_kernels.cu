// Far field of the StokesVelocity path: for every surface point t, the Stokeslet sum
// over the points s of all OTHER vesicles,
//     u_t = 1/(8 pi) sum_s [ d_s / |r| + (r . d_s) r / |r|^3 ],   r = x_s - x_t,
// d_s = f_s * area_s * qw_s (StokesAlltoAll - DirectStokesKernel, src/CPUKernels.cc:
// 123-178, 1011-1057, composed in src/InterfacialVelocity.cc:1261-1291).
//
// Work decomposition: one CTA per (source segment, target vesicle). All targets of a
// CTA belong to one vesicle, so the excluded same-vesicle sources form one contiguous
// index range and every source tile is swept as at most two unmasked sub-ranges.
// Sources are staged in shared memory, two targets per thread. Each CTA writes FP64
// partial sums for its segment; k_far_reduce adds the segments in a fixed order (the
// result is deterministic) and fuses the addition of the self part.
//
// FP64 form: two independent FP64 chains per thread; 1/sqrt from an FP32 hardware seed
// refined in FP64; a coincident pair (|r| = 0) contributes nothing, as in the reference.
// Mixed form: coordinates relative to the target vesicle's centroid (differences taken
// in FP64, rounded to FP32 once per source per CTA), the pair arithmetic in packed FP32
// (Blackwell f32x2 FMA: both targets of a thread in one instruction), the unrefined
// hardware reciprocal square root, and the FP32 partial of every 120-source sub-tile added into
// FP64 accumulators. A coincident pair of distinct vesicles (equal FP32 coordinates) makes
// the unguarded sum non-finite; such a target's segment is summed again with the pair
// skipped, as in the reference, so the guard costs one finiteness test per target and
// segment instead of a select per pair.
#include <atomic>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace ves3d {

constexpr int kTileF64 = 512;  // 24.6 KB staged per barrier pair (2% faster than 256 at 512 vesicles)
// FP32 form: 960 sources staged per pair of barriers (46 KB of shared memory, three CTAs
// per SM), summed in FP32 over sub-tiles of 120 and the sub-tile sums added in FP64.
// Measured against 512-source tiles summed whole in FP32: 12% shorter launches at 512
// vesicles, and the far field's error against FP64 about halved (worst of five small
// suspensions 5.4e-7 instead of 1.09e-6; a sub-tile of 480 gave 1.13e-6 at the same speed)
constexpr int kTileF32 = 960;
constexpr int kSubF32 = 120;

// Source sub-ranges of tile [s0, s0 + ns) that lie outside the excluded range [e0, e1).
__device__ __forceinline__ void split_tile(long s0, int ns, long e0, long e1, int& a0, int& a1, int& b0, int& b1) {
  const long lo = max(e0 - s0, 0L), hi = min(e1 - s0, (long)ns);
  if (hi <= lo) {  // no overlap
    a0 = 0; a1 = ns; b0 = b1 = 0;
  } else {
    a0 = 0; a1 = (int)lo; b0 = (int)hi; b1 = ns;
  }
}

// ------------------------------------------------------------------------------------
// FP64
// ------------------------------------------------------------------------------------
struct Acc64 {
  double x = 0.0, y = 0.0, z = 0.0;
};

__device__ __forceinline__ void pair64(const double* s, double tx, double ty, double tz, Acc64& a) {
  const double dx = s[0] - tx, dy = s[1] - ty, dz = s[2] - tz;
  const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
  double rinv = rsqrt_f64(r2);
  rinv = r2 > 0.0 ? rinv : 0.0;
  const double cc = fma(dz, s[5], fma(dy, s[4], dx * s[3])) * rinv * rinv;
  a.x = fma(fma(cc, dx, s[3]), rinv, a.x);
  a.y = fma(fma(cc, dy, s[4]), rinv, a.y);
  a.z = fma(fma(cc, dz, s[5]), rinv, a.z);
}

// grid (segments, vesicles, target chunks of 2*blockDim targets); pos/den point-major
// [N][3]; part [seg][N][3].
__global__ void __launch_bounds__(512) k_far_f64_seg(const double* __restrict__ pos, const double* __restrict__ den,
                                                     const long* __restrict__ off, long N, int seg_tiles, int v0,
                                                     double* __restrict__ part) {
  __shared__ __align__(16) double sm[kTileF64 * 6];
  const int v = v0 + blockIdx.y, seg = blockIdx.x;
  const long t0 = off[v], nt = off[v + 1] - t0;
  const int nthr = blockDim.x;
  const long c0 = (long)blockIdx.z * 2 * nthr;
  const long ia = t0 + c0 + threadIdx.x, ib = ia + nthr;
  const bool va = c0 + threadIdx.x < nt, vb = c0 + threadIdx.x + nthr < nt;
  const long la = va ? ia : t0, lb = vb ? ib : t0;
  const double ax_ = pos[3 * la], ay_ = pos[3 * la + 1], az_ = pos[3 * la + 2];
  const double bx_ = pos[3 * lb], by_ = pos[3 * lb + 1], bz_ = pos[3 * lb + 2];
  Acc64 A, B;
  const long ntiles = (N + kTileF64 - 1) / kTileF64;
  const long tb = (long)seg * seg_tiles, te = min(tb + seg_tiles, ntiles);
  for (long tile = tb; tile < te; tile++) {
    const long s0 = tile * kTileF64;
    const int ns = (int)min((long)kTileF64, N - s0);
    __syncthreads();
    for (int i = threadIdx.x; i < ns; i += nthr) {
      const long s = s0 + i;
      double* d = sm + 6 * i;
      d[0] = pos[3 * s];
      d[1] = pos[3 * s + 1];
      d[2] = pos[3 * s + 2];
      d[3] = den[3 * s];
      d[4] = den[3 * s + 1];
      d[5] = den[3 * s + 2];
    }
    __syncthreads();
    int a0, a1, b0, b1;
    split_tile(s0, ns, t0, t0 + nt, a0, a1, b0, b1);
#pragma unroll 2
    for (int k = a0; k < a1; k++) {
      pair64(sm + 6 * k, ax_, ay_, az_, A);
      pair64(sm + 6 * k, bx_, by_, bz_, B);
    }
#pragma unroll 2
    for (int k = b0; k < b1; k++) {
      pair64(sm + 6 * k, ax_, ay_, az_, A);
      pair64(sm + 6 * k, bx_, by_, bz_, B);
    }
  }
  double* P = part + (long)seg * 3 * N;
  if (va) {
    P[3 * ia] = A.x;
    P[3 * ia + 1] = A.y;
    P[3 * ia + 2] = A.z;
  }
  if (vb) {
    P[3 * ib] = B.x;
    P[3 * ib + 1] = B.y;
    P[3 * ib + 2] = B.z;
  }
}

// ------------------------------------------------------------------------------------
// Double layer, FP64 (stokes_dl_uKernel, src/PVFMMInterface.cc:285-360, over the points of
// the other vesicles): with r = x_t - x_s, u_t = 3/(4 pi) sum_s (r . n_s)(r . d_s) r / |r|^5,
// n_s the unit outward normal and d_s the density times area and smooth weight; a coincident
// pair contributes nothing. Same decomposition as k_far_f64_seg; nine values per staged
// source (position, normal, density) and the partial sums left unscaled.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void pair_dl64(const double* s, double tx, double ty, double tz, Acc64& a) {
  const double dx = tx - s[0], dy = ty - s[1], dz = tz - s[2];
  const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
  double rinv = rsqrt_f64(r2);
  rinv = r2 > 0.0 ? rinv : 0.0;
  const double rinv2 = rinv * rinv;
  const double q = fma(dz, s[5], fma(dy, s[4], dx * s[3])) * fma(dz, s[8], fma(dy, s[7], dx * s[6])) *
                   (rinv2 * rinv2 * rinv);
  a.x = fma(dx, q, a.x);
  a.y = fma(dy, q, a.y);
  a.z = fma(dz, q, a.z);
}

// grid (segments, vesicles, target chunks of 2*blockDim targets); pos, nrm, dden
// point-major [N][3]; part [seg][N][3].
__global__ void __launch_bounds__(512) k_far_dl_f64_seg(const double* __restrict__ pos, const double* __restrict__ nrm,
                                                        const double* __restrict__ dden, const long* __restrict__ off,
                                                        long N, int seg_tiles, int v0, double* __restrict__ part) {
  __shared__ __align__(16) double sm[kTileF64 * 9];
  const int v = v0 + blockIdx.y, seg = blockIdx.x;
  const long t0 = off[v], nt = off[v + 1] - t0;
  const int nthr = blockDim.x;
  const long c0 = (long)blockIdx.z * 2 * nthr;
  const long ia = t0 + c0 + threadIdx.x, ib = ia + nthr;
  const bool va = c0 + threadIdx.x < nt, vb = c0 + threadIdx.x + nthr < nt;
  const long la = va ? ia : t0, lb = vb ? ib : t0;
  const double ax_ = pos[3 * la], ay_ = pos[3 * la + 1], az_ = pos[3 * la + 2];
  const double bx_ = pos[3 * lb], by_ = pos[3 * lb + 1], bz_ = pos[3 * lb + 2];
  Acc64 A, B;
  const long ntiles = (N + kTileF64 - 1) / kTileF64;
  const long tb = (long)seg * seg_tiles, te = min(tb + seg_tiles, ntiles);
  for (long tile = tb; tile < te; tile++) {
    const long s0 = tile * kTileF64;
    const int ns = (int)min((long)kTileF64, N - s0);
    __syncthreads();
    for (int i = threadIdx.x; i < ns; i += nthr) {
      const long s = s0 + i;
      double* d = sm + 9 * i;
      d[0] = pos[3 * s];
      d[1] = pos[3 * s + 1];
      d[2] = pos[3 * s + 2];
      d[3] = nrm[3 * s];
      d[4] = nrm[3 * s + 1];
      d[5] = nrm[3 * s + 2];
      d[6] = dden[3 * s];
      d[7] = dden[3 * s + 1];
      d[8] = dden[3 * s + 2];
    }
    __syncthreads();
    int a0, a1, b0, b1;
    split_tile(s0, ns, t0, t0 + nt, a0, a1, b0, b1);
    for (int k = a0; k < a1; k++) {
      pair_dl64(sm + 9 * k, ax_, ay_, az_, A);
      pair_dl64(sm + 9 * k, bx_, by_, bz_, B);
    }
    for (int k = b0; k < b1; k++) {
      pair_dl64(sm + 9 * k, ax_, ay_, az_, A);
      pair_dl64(sm + 9 * k, bx_, by_, bz_, B);
    }
  }
  double* P = part + (long)seg * 3 * N;
  if (va) {
    P[3 * ia] = A.x;
    P[3 * ia + 1] = A.y;
    P[3 * ia + 2] = A.z;
  }
  if (vb) {
    P[3 * ib] = B.x;
    P[3 * ib + 1] = B.y;
    P[3 * ib + 2] = B.z;
  }
}

// Four targets per thread (a launch shape the autotuner may pick): twice the independent
// FP64 chains and half the shared-memory reads per pair, at 98 registers.
template <int TPT>
__global__ void __launch_bounds__(512) k_far_f64_segT(const double* __restrict__ pos, const double* __restrict__ den,
                                                     const long* __restrict__ off, long N, int seg_tiles, int v0,
                                                     double* __restrict__ part) {
  __shared__ __align__(16) double sm[kTileF64 * 6];
  const int v = v0 + blockIdx.y, seg = blockIdx.x;
  const long t0 = off[v], nt = off[v + 1] - t0;
  const int nthr = blockDim.x;
  const long c0 = (long)blockIdx.z * TPT * nthr;
  // TPT targets per thread (independent FP64 chains; one shared-memory read per source)
  double tx[TPT], ty[TPT], tz[TPT];
  Acc64 acc[TPT];
#pragma unroll
  for (int q = 0; q < TPT; q++) {
    const long i = c0 + threadIdx.x + (long)q * nthr;
    const long l = t0 + (i < nt ? i : 0);
    tx[q] = pos[3 * l];
    ty[q] = pos[3 * l + 1];
    tz[q] = pos[3 * l + 2];
  }
  const long ntiles = (N + kTileF64 - 1) / kTileF64;
  const long tb = (long)seg * seg_tiles, te = min(tb + seg_tiles, ntiles);
  for (long tile = tb; tile < te; tile++) {
    const long s0 = tile * kTileF64;
    const int ns = (int)min((long)kTileF64, N - s0);
    __syncthreads();
    for (int i = threadIdx.x; i < ns; i += nthr) {
      const long s = s0 + i;
      double* d = sm + 6 * i;
      d[0] = pos[3 * s];
      d[1] = pos[3 * s + 1];
      d[2] = pos[3 * s + 2];
      d[3] = den[3 * s];
      d[4] = den[3 * s + 1];
      d[5] = den[3 * s + 2];
    }
    __syncthreads();
    int a0, a1, b0, b1;
    split_tile(s0, ns, t0, t0 + nt, a0, a1, b0, b1);
#pragma unroll 2
    for (int k = a0; k < a1; k++) {
#pragma unroll
      for (int q = 0; q < TPT; q++) pair64(sm + 6 * k, tx[q], ty[q], tz[q], acc[q]);
    }
#pragma unroll 2
    for (int k = b0; k < b1; k++) {
#pragma unroll
      for (int q = 0; q < TPT; q++) pair64(sm + 6 * k, tx[q], ty[q], tz[q], acc[q]);
    }
  }
  double* P = part + (long)seg * 3 * N;
#pragma unroll
  for (int q = 0; q < TPT; q++) {
    const long i = c0 + threadIdx.x + (long)q * nthr;
    if (i < nt) {
      P[3 * (t0 + i)] = acc[q].x;
      P[3 * (t0 + i) + 1] = acc[q].y;
      P[3 * (t0 + i) + 2] = acc[q].z;
    }
  }
}

// ------------------------------------------------------------------------------------
// Mixed (packed FP32 pairs, FP64 accumulation)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// One target's sum over the sources [s0, s1) outside [e0, e1) with coincident pairs
// skipped (|r| = 0 contributes nothing, as in StokesAlltoAll, src/CPUKernels.cc:1030-1040),
// in the pair arithmetic of the mixed kernel (FP32 coordinates relative to the centroid
// (cx, cy, cz), FP32 sums per 120 sources, FP64 across them); (tx, ty, tz) is the negated
// target. The slow path of a target whose segment sum came out non-finite.
__device__ __forceinline__ double3 far_f32_guarded(const double* __restrict__ pos, const double* __restrict__ den,
                                                long s0, long s1, long e0, long e1, double cx, double cy, double cz,
                                                float tx, float ty, float tz) {
  double ax = 0.0, ay = 0.0, az = 0.0;
  float ux = 0.f, uy = 0.f, uz = 0.f;
  int cnt = 0;
  for (long s = s0; s < s1; s++) {
    if (s >= e0 && s < e1) continue;
    const float rx = (float)(pos[3 * s] - cx) + tx, ry = (float)(pos[3 * s + 1] - cy) + ty,
                rz = (float)(pos[3 * s + 2] - cz) + tz;
    const float dx = (float)den[3 * s], dy = (float)den[3 * s + 1], dz = (float)den[3 * s + 2];
    const float r2 = rx * rx + ry * ry + rz * rz;
    if (r2 > 0.f) {
      const float y = rsqrt_ftz(r2);
      const float c = (rx * dx + ry * dy + rz * dz) * y * y;
      ux += (c * rx + dx) * y;
      uy += (c * ry + dy) * y;
      uz += (c * rz + dz) * y;
    }
    if (++cnt == kSubF32) {
      ax += ux; ay += uy; az += uz;
      ux = uy = uz = 0.f;
      cnt = 0;
    }
  }
  return make_double3(ax + ux, ay + uy, az + uz);
}

// NP packed target pairs per thread (2 NP targets): target j of thread i in chunk c0 is
// c0 + i + j * blockDim.x. NP = 2 reads each staged source once for four targets and gives
// the scheduler two independent chains per source.
template <int NP>
__global__ void __launch_bounds__(512) k_far_f32_segT(const double* __restrict__ pos, const double* __restrict__ den,
                                                      const long* __restrict__ off, long N, int seg_tiles, int v0,
                                                      double* __restrict__ part) {
  // one source = 6 broadcast float2: (x,x) (y,y) (z,z) (dx,dx) (dy,dy) (dz,dz)
  __shared__ __align__(16) float2 sm[kTileF32 * 6];
  __shared__ double cen[3];
  __shared__ double red[3][32];
  constexpr int T = 2 * NP;
  const int v = v0 + blockIdx.y, seg = blockIdx.x;
  const long t0 = off[v], nt = off[v + 1] - t0;
  const int nthr = blockDim.x;
  // centroid of the target vesicle (FP64), the origin of this CTA's FP32 coordinates
  {
    double cx = 0, cy = 0, cz = 0;
    for (long i = threadIdx.x; i < nt; i += nthr) {
      cx += pos[3 * (t0 + i)];
      cy += pos[3 * (t0 + i) + 1];
      cz += pos[3 * (t0 + i) + 2];
    }
    for (int o = 16; o > 0; o >>= 1) {
      cx += __shfl_down_sync(0xffffffffu, cx, o);
      cy += __shfl_down_sync(0xffffffffu, cy, o);
      cz += __shfl_down_sync(0xffffffffu, cz, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
      red[0][w] = cx;
      red[1][w] = cy;
      red[2][w] = cz;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
      double s = 0;
      for (int i = 0; i < (nthr + 31) / 32; i++) s += red[threadIdx.x][i];
      cen[threadIdx.x] = s / (double)nt;
    }
    __syncthreads();
  }
  const double cx = cen[0], cy = cen[1], cz = cen[2];
  const long c0 = (long)blockIdx.z * T * nthr;
  // negated targets, packed (lane x = target 2q, lane y = target 2q + 1 of the thread)
  float2 ntx[NP], nty[NP], ntz[NP];
#pragma unroll
  for (int q = 0; q < NP; q++) {
    const long ja = c0 + threadIdx.x + (long)(2 * q) * nthr, jb = ja + nthr;
    const long la = t0 + (ja < nt ? ja : 0), lb = t0 + (jb < nt ? jb : 0);
    ntx[q] = make_float2((float)(cx - pos[3 * la]), (float)(cx - pos[3 * lb]));
    nty[q] = make_float2((float)(cy - pos[3 * la + 1]), (float)(cy - pos[3 * lb + 1]));
    ntz[q] = make_float2((float)(cz - pos[3 * la + 2]), (float)(cz - pos[3 * lb + 2]));
  }
  double A[T][3];
#pragma unroll
  for (int j = 0; j < T; j++) A[j][0] = A[j][1] = A[j][2] = 0.0;
  const long ntiles = (N + kTileF32 - 1) / kTileF32;
  const long tb = (long)seg * seg_tiles, te = min(tb + seg_tiles, ntiles);
  for (long tile = tb; tile < te; tile++) {
    const long s0 = tile * kTileF32;
    const int ns = (int)min((long)kTileF32, N - s0);
    __syncthreads();
    for (int i = threadIdx.x; i < ns; i += nthr) {
      const long s = s0 + i;
      float2* d = sm + 6 * i;
      d[0] = f2((float)(pos[3 * s] - cx));
      d[1] = f2((float)(pos[3 * s + 1] - cy));
      d[2] = f2((float)(pos[3 * s + 2] - cz));
      d[3] = f2((float)den[3 * s]);
      d[4] = f2((float)den[3 * s + 1]);
      d[5] = f2((float)den[3 * s + 2]);
    }
    __syncthreads();
    int r0[2], r1[2];
    split_tile(s0, ns, t0, t0 + nt, r0[0], r1[0], r0[1], r1[1]);
    for (int sb = 0; sb < ns; sb += kSubF32) {
      const int se = min(sb + kSubF32, ns);
      float2 ux[NP], uy[NP], uz[NP];
#pragma unroll
      for (int q = 0; q < NP; q++) ux[q] = uy[q] = uz[q] = f2(0.f);
#pragma unroll
      for (int part_i = 0; part_i < 2; part_i++) {
        const int k0 = max(r0[part_i], sb), k1 = min(r1[part_i], se);
#pragma unroll 4
        for (int k = k0; k < k1; k++) {
          const float4* qs = reinterpret_cast<const float4*>(sm + 6 * k);
          const float4 q0 = qs[0], q1 = qs[1], q2 = qs[2];
          const float2 sx = make_float2(q0.x, q0.y), sy = make_float2(q0.z, q0.w);
          const float2 sz = make_float2(q1.x, q1.y), dx_ = make_float2(q1.z, q1.w);
          const float2 dy_ = make_float2(q2.x, q2.y), dz_ = make_float2(q2.z, q2.w);
#pragma unroll
          for (int q = 0; q < NP; q++) {
            // the differences as scalar adds: the packed ops keep one FMA pipe busy (76% of
            // cycles) and the scalar ones can go to the other (measured 1% faster)
            const float2 rx = make_float2(__fadd_rn(sx.x, ntx[q].x), __fadd_rn(sx.y, ntx[q].y));
            const float2 ry = make_float2(__fadd_rn(sy.x, nty[q].x), __fadd_rn(sy.y, nty[q].y));
            const float2 rz = make_float2(__fadd_rn(sz.x, ntz[q].x), __fadd_rn(sz.y, ntz[q].y));
            float2 r2 = __fmul2_rn(rx, rx);
            r2 = __ffma2_rn(ry, ry, r2);
            r2 = __ffma2_rn(rz, rz, r2);
            // unrefined hardware reciprocal square root: its error (a few 1e-7 relative per
            // pair) averages out in the sum and stays below the FP32 rounding of the
            // coordinates; a Newton step would cost ~20% more FP32 instructions per pair
            const float2 y = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
            const float2 y2 = __fmul2_rn(y, y);
            float2 dot = __fmul2_rn(rx, dx_);
            dot = __ffma2_rn(ry, dy_, dot);
            dot = __ffma2_rn(rz, dz_, dot);
            const float2 cc = __fmul2_rn(dot, y2);
            ux[q] = __ffma2_rn(__ffma2_rn(cc, rx, dx_), y, ux[q]);
            uy[q] = __ffma2_rn(__ffma2_rn(cc, ry, dy_), y, uy[q]);
            uz[q] = __ffma2_rn(__ffma2_rn(cc, rz, dz_), y, uz[q]);
          }
        }
      }
#pragma unroll
      for (int q = 0; q < NP; q++) {
        A[2 * q][0] += ux[q].x;
        A[2 * q][1] += uy[q].x;
        A[2 * q][2] += uz[q].x;
        A[2 * q + 1][0] += ux[q].y;
        A[2 * q + 1][1] += uy[q].y;
        A[2 * q + 1][2] += uz[q].y;
      }
    }
  }
  // A coincident pair left a target's segment sum non-finite: sum the segment again for
  // that target with coincident pairs skipped (non-finite inputs stay non-finite). One
  // test per target and segment; no instruction in the pair loop.
#pragma unroll
  for (int j = 0; j < T; j++) {
    const long jj = c0 + threadIdx.x + (long)j * nthr;
    if (jj < nt && !isfinite(A[j][0] + A[j][1] + A[j][2])) {
      const long g = t0 + jj;
      // the centroid from shared memory again: keeping it in registers across the pair
      // loop would cost the loop registers
      const double gx = cen[0], gy = cen[1], gz = cen[2];
      const double3 a = far_f32_guarded(pos, den, tb * kTileF32, min(te * kTileF32, N), t0, t0 + nt, gx, gy, gz,
                                        (float)(gx - pos[3 * g]), (float)(gy - pos[3 * g + 1]),
                                        (float)(gz - pos[3 * g + 2]));
      A[j][0] = a.x;
      A[j][1] = a.y;
      A[j][2] = a.z;
    }
  }
  double* P = part + (long)seg * 3 * N;
#pragma unroll
  for (int j = 0; j < T; j++) {
    const long jj = c0 + threadIdx.x + (long)j * nthr;
    if (jj < nt) {
      const long g = t0 + jj;
      P[3 * g] = A[j][0];
      P[3 * g + 1] = A[j][1];
      P[3 * g + 2] = A[j][2];
    }
  }
}

// out (AxisMajor per vesicle) = add + (1/8pi) sum over segments in order. One CTA per
// vesicle; vesicle v holds points [off[v], off[v+1]) as [3][n_v] from 3*off[v].
__global__ void k_far_reduce(const double* __restrict__ part, int nseg, const long* __restrict__ off, long N,
                             const double* __restrict__ add, double* __restrict__ out, double* __restrict__ far_out,
                             const double* __restrict__ part2, int nseg2, double scale2) {
  const int v = blockIdx.x;
  const long t0 = off[v], nt = off[v + 1] - t0;
  for (long i = threadIdx.x; i < 3 * nt; i += blockDim.x) {
    const long k = i / 3;
    const int c = (int)(i - 3 * k);
    const long g = t0 + k;
    double s = 0.0;
    for (int q = 0; q < nseg; q++) s += part[(long)q * 3 * N + 3 * g + c];
    s *= kInv8Pi;
    if (part2) {  // a second set of partials (the double layer) with its own constant
      double s2 = 0.0;
      for (int q = 0; q < nseg2; q++) s2 += part2[(long)q * 3 * N + 3 * g + c];
      s += s2 * scale2;
    }
    const long o = 3 * t0 + c * nt + k;
    if (far_out) far_out[o] = s;
    out[o] = (add ? add[o] : 0.0) + s;
  }
}

// Launch shape of the far field: how many waves of CTAs the source range is split into
// (segments), and how many targets of a vesicle one CTA takes (two per thread).
struct FarShape {
  int waves = 8;
  int chunk_max = 1024;
  int tpt = 2;  // targets per thread, 2 or 4 (the FP32 form packs them in pairs)
};

int far_segments(long nves, long N, int tile, int nthr, int waves, int* seg_tiles) {
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long ntiles = (N + tile - 1) / tile;
  const int per_sm = max(1, 2048 / max(nthr, 32));  // resident CTAs per SM if threads limit
  const long want = (long)nsm * per_sm * waves;
  long nseg = (want + nves - 1) / nves;
  if (nseg < 1) nseg = 1;
  if (nseg > ntiles) nseg = ntiles;
  *seg_tiles = (int)((ntiles + nseg - 1) / nseg);
  return (int)((ntiles + *seg_tiles - 1) / *seg_tiles);
}

int launch_far_reduce(const double* part, int nseg, const long* off, long nves, long N, const double* add, double* out,
                      double* far_out, cudaStream_t st, const double* part2, int nseg2, double scale2) {
  k_far_reduce<<<(unsigned)nves, 256, 0, st>>>(part, nseg, off, N, add, out, far_out, part2, nseg2, scale2);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

static void chunking(int nt, int chunk_max, int tpt, int* nchunk, int* nthr) {
  // targets of a vesicle in chunks of at most chunk_max (tpt per thread)
  *nchunk = (nt + chunk_max - 1) / chunk_max;
  const int per_chunk = (nt + *nchunk - 1) / *nchunk;
  *nthr = 32 * ((((per_chunk + tpt - 1) / tpt) + 31) / 32);
}

// With nseg_out null the segments' partials are reduced on st; otherwise the segments
// alone are launched and their count returned, for a launch_far_reduce elsewhere.
static int launch_far_shape(const FarShape& sh, bool mixed, const double* pos, const double* den, const long* off,
                            long nves, long N, const FarGroup* groups, int ngroups, const double* add, double* out,
                            double* far_out, double* part, long part_cap_segments, cudaStream_t st,
                            int* nseg_out = nullptr) {
  const int tile = mixed ? kTileF32 : kTileF64;
  // one segment layout for all groups, sized by the average vesicle
  long nthr_sum = 0, nchunk_tot = 0;
  for (int g = 0; g < ngroups; g++) {
    int nc, nt;
    chunking(groups[g].nt, sh.chunk_max, sh.tpt, &nc, &nt);
    nthr_sum += (long)nt * groups[g].nv;
    nchunk_tot += (long)nc * groups[g].nv;
  }
  const int nthr_avg = (int)(nthr_sum / nves);
  int seg_tiles = 1;
  int nseg = far_segments(nchunk_tot, N, tile, nthr_avg, sh.waves, &seg_tiles);
  if (nseg > part_cap_segments) {
    const long ntiles = (N + tile - 1) / tile;
    seg_tiles = (int)((ntiles + part_cap_segments - 1) / part_cap_segments);
    nseg = (int)((ntiles + seg_tiles - 1) / seg_tiles);
  }
  for (int g = 0; g < ngroups; g++) {
    if (groups[g].nv <= 0) continue;
    int nchunk, nthr;
    chunking(groups[g].nt, sh.chunk_max, sh.tpt, &nchunk, &nthr);
    dim3 grid(nseg, (unsigned)groups[g].nv, nchunk);
    if (mixed && sh.tpt == 4)
      k_far_f32_segT<2><<<grid, nthr, 0, st>>>(pos, den, off, N, seg_tiles, (int)groups[g].v0, part);
    else if (mixed)
      k_far_f32_segT<1><<<grid, nthr, 0, st>>>(pos, den, off, N, seg_tiles, (int)groups[g].v0, part);
    else if (sh.tpt == 4)
      k_far_f64_segT<4><<<grid, nthr, 0, st>>>(pos, den, off, N, seg_tiles, (int)groups[g].v0, part);
    else
      k_far_f64_seg<<<grid, nthr, 0, st>>>(pos, den, off, N, seg_tiles, (int)groups[g].v0, part);
    VES3D_LAUNCHED();
  }
  if (nseg_out) {
    *nseg_out = nseg;
    return VES3D_OK;
  }
  return launch_far_reduce(part, nseg, off, nves, N, add, out, far_out, st);
}

// ---- autotuner of the launch shape ----------------------------------------------------
// On the first launch of a configuration (precision, N, vesicles, group structure) with
// autotuning on, every candidate shape is launched once and timed with CUDA events on the
// caller's stream; the fastest is cached for the process. Off by default and never during
// stream capture. Candidates differ only in how the source range is split, i.e. in the
// grouping of the FP64 partial sums (results agree to rounding); a tuned configuration
// always uses its one shape afterwards, so repeated evaluations stay bitwise identical.
struct FarTuneEntry {
  FarShape shape;
  float ms = 0;
};

static std::mutex g_tune_mu;
static std::map<std::string, FarTuneEntry> g_tuned;
static std::atomic<int> g_autotune{-1};

static bool autotune_on() {
  int v = g_autotune.load();
  if (v < 0) {
    const char* e = getenv("VES3D_AUTOTUNE");
    v = (e && e[0] == '1') ? 1 : 0;
    g_autotune.store(v);
  }
  return v == 1;
}

static std::string tune_key(bool mixed, long nves, long N, const FarGroup* groups, int ngroups) {
  std::string k = mixed ? "f32" : "f64";
  k += ":N=" + std::to_string(N) + ":v=" + std::to_string(nves);
  for (int g = 0; g < ngroups; g++) k += ":" + std::to_string(groups[g].nv) + "x" + std::to_string(groups[g].nt);
  return k;
}

static FarShape g_forced{0, 0, 0};  // a caller-fixed shape (waves 0 = none)

int set_far_shape(int waves, int chunk_max, int tpt) {
  if (waves == 0) {
    g_forced = FarShape{0, 0, 0};
    return VES3D_OK;
  }
  if ((waves != 4 && waves != 8 && waves != 16) || (chunk_max != 512 && chunk_max != 1024) ||
      (tpt != 2 && tpt != 4)) {
    set_error("far shape: waves in {4, 8, 16}, chunk in {512, 1024}, targets per thread in {2, 4}");
    return VES3D_ERR_ARG;
  }
  g_forced = FarShape{waves, chunk_max, tpt};
  return VES3D_OK;
}

int launch_far_groups(bool mixed, const double* pos, const double* den, const long* off, long nves, long N,
                      const FarGroup* groups, int ngroups, const double* add, double* out, double* far_out,
                      double* part, long part_cap_segments, cudaStream_t st, int* nseg_out) {
  if (N <= 0) return VES3D_OK;
  FarShape shape;
  if (g_forced.waves) {
    shape = g_forced;
  } else if (autotune_on()) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    VES3D_CK(cudaStreamIsCapturing(st, &cap));
    const std::string key = tune_key(mixed, nves, N, groups, ngroups);
    bool have = false;
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tuned.find(key);
      if (it != g_tuned.end()) {
        shape = it->second.shape;
        have = true;
      }
    }
    if (!have && cap == cudaStreamCaptureStatusNone) {
      std::vector<FarShape> cands;
      for (int tpt : {2, 4}) {
        for (int chunk : {1024, 512})
          for (int waves : {4, 8, 16}) cands.push_back(FarShape{waves, chunk, tpt});
      }
      cudaEvent_t e0, e1;
      VES3D_CK(cudaEventCreate(&e0));
      VES3D_CK(cudaEventCreate(&e1));
      FarTuneEntry best;
      best.ms = 1e30f;
      int s = VES3D_OK;
      for (const FarShape& c : cands) {
        cudaEventRecord(e0, st);
        // candidates are timed on their segment kernels alone (the reduce is the same
        // for every shape, and its outputs may not be given when the caller reduces later)
        int cand_nseg = 0;
        s = launch_far_shape(c, mixed, pos, den, off, nves, N, groups, ngroups, add, out, far_out, part,
                             part_cap_segments, st, &cand_nseg);
        if (s) break;
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best.ms) {
          best.ms = ms;
          best.shape = c;
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      if (s) return s;
      {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned[key] = best;
      }
      shape = best.shape;
    }
  }
  return launch_far_shape(shape, mixed, pos, den, off, nves, N, groups, ngroups, add, out, far_out, part,
                          part_cap_segments, st, nseg_out);
}

int set_autotune(int on) {
  g_autotune.store(on ? 1 : 0);
  return VES3D_OK;
}

// "key waves chunk ms" per tuned configuration, one per line
std::string autotune_report() {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  std::string r;
  for (const auto& kv : g_tuned)
    r += kv.first + " waves=" + std::to_string(kv.second.shape.waves) + " chunk=" +
         std::to_string(kv.second.shape.chunk_max) + " tpt=" + std::to_string(kv.second.shape.tpt) +
         " ms=" + std::to_string(kv.second.ms) + "\n";
  return r;
}

// The far double layer of a suspension in order groups: one launch per group (its own
// target chunking and block shape), one segment layout for all, as launch_far_shape.
int launch_far_dl_groups(const double* pos, const double* nrm, const double* dden, const long* off, long nves, long N,
                         const FarGroup* groups, int ngroups, double* part, long part_cap_segments, cudaStream_t st,
                         int* nseg_out) {
  *nseg_out = 0;
  if (N <= 0 || nves <= 0) return VES3D_OK;
  long nthr_sum = 0, nchunk_tot = 0;
  for (int g = 0; g < ngroups; g++) {
    int nc, nt;
    chunking(groups[g].nt, 1024, 2, &nc, &nt);
    nthr_sum += (long)nt * groups[g].nv;
    nchunk_tot += (long)nc * groups[g].nv;
  }
  int seg_tiles = 1;
  int nseg = far_segments(nchunk_tot, N, kTileF64, (int)(nthr_sum / nves), 8, &seg_tiles);
  if (nseg > part_cap_segments) {
    const long ntiles = (N + kTileF64 - 1) / kTileF64;
    seg_tiles = (int)((ntiles + part_cap_segments - 1) / part_cap_segments);
    nseg = (int)((ntiles + seg_tiles - 1) / seg_tiles);
  }
  for (int g = 0; g < ngroups; g++) {
    if (groups[g].nv <= 0) continue;
    int nchunk, nthr;
    chunking(groups[g].nt, 1024, 2, &nchunk, &nthr);
    dim3 grid(nseg, (unsigned)groups[g].nv, nchunk);
    k_far_dl_f64_seg<<<grid, nthr, 0, st>>>(pos, nrm, dden, off, N, seg_tiles, (int)groups[g].v0, part);
    VES3D_LAUNCHED();
  }
  *nseg_out = nseg;
  return VES3D_OK;
}

int launch_far_dl(const double* pos, const double* nrm, const double* dden, const long* off, long nves, long N,
                  int max_nt, double* part, long part_cap_segments, cudaStream_t st, int* nseg_out) {
  FarGroup g{0, nves, max_nt};
  return launch_far_dl_groups(pos, nrm, dden, off, nves, N, &g, 1, part, part_cap_segments, st, nseg_out);
}

int launch_far(bool mixed, const double* pos, const double* den, const long* off, long nves, long N, int max_nt,
               const double* add, double* out, double* far_out, double* part, long part_cap_segments,
               cudaStream_t st, int* nseg_out) {
  FarGroup g{0, nves, max_nt};
  return launch_far_groups(mixed, pos, den, off, nves, N, &g, 1, add, out, far_out, part, part_cap_segments, st,
                           nseg_out);
}

}  // namespace ves3d
