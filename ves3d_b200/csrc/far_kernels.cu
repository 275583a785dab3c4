// Far field of the StokesVelocity path: for every surface point t, the Stokeslet sum
// over the points s of all OTHER vesicles,
//     u_t = 1/(8 pi) sum_s [ d_s / |r| + (r . d_s) r / |r|^3 ],   r = x_s - x_t,
// d_s = f_s * area_s * qw_s (StokesAlltoAll - DirectStokesKernel, src/CPUKernels.cc:
// 123-178, 1011-1057, composed in src/InterfacialVelocity.cc:1261-1291).
//
// Work decomposition: one CTA per (source segment, chunk of 2 x threads consecutive
// targets). A chunk may span several vesicles of any sizes, so one launch covers a
// polydisperse suspension and every lane holds a target. Sources outside the chunk's
// vesicles are swept unmasked (each tile as at most two sub-ranges); the chunk's own
// vesicles' sources are swept after, each target skipping its own vesicle. Sources are
// staged in shared memory, two targets per thread. Each CTA writes FP64 partial sums for
// its segment; k_far_reduce adds the segments in a fixed order (the result is
// deterministic) and fuses the addition of the self part.
//
// FP64 form: two independent FP64 chains per thread; 1/sqrt from an FP32 hardware seed
// refined in FP64; a coincident pair (|r| = 0) contributes nothing, as in the reference.
// Mixed form: coordinates relative to the centroid of the chunk's targets (differences
// taken in FP64, rounded to FP32 once per source per CTA), the pair arithmetic in packed
// FP32 (Blackwell f32x2 FMA: both targets of a thread in one instruction), the unrefined
// hardware reciprocal square root, and the FP32 partial of every 120-source sub-tile added
// into FP64 accumulators. A coincident pair of distinct vesicles (equal FP32 coordinates)
// makes the unguarded sum non-finite; such a target's segment is summed again with the pair
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
// FP32 form: 960 sources staged per pair of barriers (46 KB of shared memory), summed in
// FP32 over sub-tiles of 120 and the sub-tile sums added in FP64. Measured against
// 512-source tiles summed whole in FP32: 12% shorter launches at 512 vesicles, and the far
// field's error against FP64 about halved (worst of five small suspensions 5.4e-7 instead
// of 1.09e-6; a sub-tile of 480 gave 1.13e-6 at the same speed)
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

// Vesicle holding point g (off[v] <= g < off[v + 1]).
__device__ __forceinline__ long vesicle_of(const long* __restrict__ off, long nves, long g) {
  long lo = 0, hi = nves;
  while (hi - lo > 1) {
    const long mid = (lo + hi) >> 1;
    if (off[mid] <= g) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Work decomposition shared by every far-field kernel: CTA (segment, chunk) takes the
// targets [c0, c0 + 2 NT) of the concatenated points, whichever vesicles they belong to
// (a chunk may span several; every lane has a target but in the last chunk), and the
// sources of its segment of tiles. Sources outside the chunk's vesicles [u0, u1) are swept
// unmasked, tile by tile; the chunk's own vesicles' sources that fall in the segment are
// swept after, each target skipping the points of its own vesicle. One launch covers a
// suspension of any vesicle sizes (every SH order of a polydisperse suspension).
struct ChunkRange {
  long c0, c1;  // targets
  long u0, u1;  // their vesicles' points
};

template <int NT>
__device__ __forceinline__ void chunk_range(const long* __restrict__ off, long nves, long N, ChunkRange* cr) {
  if (threadIdx.x == 0) {
    const long c0 = (long)blockIdx.y * 2 * NT, c1 = min(N, c0 + 2L * NT);
    cr->c0 = c0;
    cr->c1 = c1;
    cr->u0 = off[vesicle_of(off, nves, c0)];
    cr->u1 = off[vesicle_of(off, nves, c1 - 1) + 1];
  }
  __syncthreads();
}

// ------------------------------------------------------------------------------------
// FP64
// ------------------------------------------------------------------------------------
struct Acc64 {
  double x = 0.0, y = 0.0, z = 0.0;
};

// One pair: 1/sqrt from the integer-cut seed, a coincident pair (|r|^2 below 2^-126)
// contributes nothing, as in the reference.
__device__ __forceinline__ void pair64(const double* s, double tx, double ty, double tz, Acc64& a) {
  const double dx = s[0] - tx, dy = s[1] - ty, dz = s[2] - tz;
  const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
  double rinv = rsqrt_f64_int_seed(r2);
  rinv = r2_normal(r2) ? rinv : 0.0;
  const double cc = fma(dz, s[5], fma(dy, s[4], dx * s[3])) * rinv * rinv;
  a.x = fma(fma(cc, dx, s[3]), rinv, a.x);
  a.y = fma(fma(cc, dy, s[4]), rinv, a.y);
  a.z = fma(fma(cc, dz, s[5]), rinv, a.z);
}

// Stage sources [s0, s0 + ns) into shared memory, W doubles each from the three point-major
// arrays a, b (and c when W == 9).
template <int W, int NT>
__device__ __forceinline__ void stage64(double* sm, const double* __restrict__ a, const double* __restrict__ b,
                                        const double* __restrict__ c, long s0, int ns) {
#pragma unroll 1
  for (int i = threadIdx.x; i < ns; i += NT) {
    const long s = s0 + i;
    double* d = sm + W * i;
    d[0] = a[3 * s];
    d[1] = a[3 * s + 1];
    d[2] = a[3 * s + 2];
    d[3] = b[3 * s];
    d[4] = b[3 * s + 1];
    d[5] = b[3 * s + 2];
    if (W == 9) {
      d[6] = c[3 * s];
      d[7] = c[3 * s + 1];
      d[8] = c[3 * s + 2];
    }
  }
}

// grid (segments, target chunks of 2 NT); pos/den point-major [N][3]; part [seg][N][3].
// 384 threads at 56 registers: three CTAs (36 warps) per SM, measured 16% faster at 512
// vesicles than one vesicle per CTA at 288 threads and 63 registers.
template <int NT>
__global__ void __launch_bounds__(NT, 1152 / NT) k_far_f64_flat(const double* __restrict__ pos,
                                                                 const double* __restrict__ den,
                                                                 const long* __restrict__ off, long nves, long N,
                                                                 int seg_tiles, double* __restrict__ part) {
  __shared__ __align__(16) double sm[kTileF64 * 6];
  __shared__ ChunkRange cr;
  chunk_range<NT>(off, nves, N, &cr);
  const int seg = blockIdx.x;
  const long c0 = cr.c0, c1 = cr.c1;
  const long ia = c0 + threadIdx.x, ib = ia + NT;
  const long la = ia < c1 ? ia : c0, lb = ib < c1 ? ib : c0;
  const double ax_ = pos[3 * la], ay_ = pos[3 * la + 1], az_ = pos[3 * la + 2];
  const double bx_ = pos[3 * lb], by_ = pos[3 * lb + 1], bz_ = pos[3 * lb + 2];
  Acc64 A, B;
  const long ntiles = (N + kTileF64 - 1) / kTileF64;
  const long tb = (long)seg * seg_tiles, te = min(tb + seg_tiles, ntiles);
  for (long tile = tb; tile < te; tile++) {
    const long s0 = tile * kTileF64;
    const int ns = (int)min((long)kTileF64, N - s0);
    __syncthreads();
    stage64<6, NT>(sm, pos, den, nullptr, s0, ns);
    __syncthreads();
    int a0, a1, b0, b1;
    split_tile(s0, ns, cr.u0, cr.u1, a0, a1, b0, b1);
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
  // the chunk's own vesicles within this segment: each target skips its own vesicle
  const long g0 = max(cr.u0, tb * kTileF64), g1 = min(cr.u1, min(te * kTileF64, N));
  if (g0 < g1) {
    const long va = vesicle_of(off, nves, la), vb = vesicle_of(off, nves, lb);
    const long ea0 = off[va], ea1 = off[va + 1], eb0 = off[vb], eb1 = off[vb + 1];
    for (long s0 = g0; s0 < g1; s0 += kTileF64) {
      const int ns = (int)min((long)kTileF64, g1 - s0);
      __syncthreads();
      stage64<6, NT>(sm, pos, den, nullptr, s0, ns);
      __syncthreads();
      for (int k = 0; k < ns; k++) {
        const long s = s0 + k;
        if (s < ea0 || s >= ea1) pair64(sm + 6 * k, ax_, ay_, az_, A);
        if (s < eb0 || s >= eb1) pair64(sm + 6 * k, bx_, by_, bz_, B);
      }
    }
  }
  double* P = part + (long)seg * 3 * N;
  if (ia < c1) {
    P[3 * ia] = A.x;
    P[3 * ia + 1] = A.y;
    P[3 * ia + 2] = A.z;
  }
  if (ib < c1) {
    P[3 * ib] = B.x;
    P[3 * ib + 1] = B.y;
    P[3 * ib + 2] = B.z;
  }
}

// ------------------------------------------------------------------------------------
// Double layer, FP64 (stokes_dl_uKernel, src/PVFMMInterface.cc:285-360, over the points of
// the other vesicles): with r = x_t - x_s, u_t = 3/(4 pi) sum_s (r . n_s)(r . d_s) r / |r|^5,
// n_s the unit outward normal and d_s the density times area and smooth weight; a coincident
// pair contributes nothing. Same decomposition as k_far_f64_flat; nine values per staged
// source (position, normal, density) and the partial sums left unscaled.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void pair_dl64(const double* s, double tx, double ty, double tz, Acc64& a) {
  const double dx = tx - s[0], dy = ty - s[1], dz = tz - s[2];
  const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
  double rinv = rsqrt_f64_int_seed(r2);
  rinv = r2_normal(r2) ? rinv : 0.0;
  const double rinv2 = rinv * rinv;
  const double q = fma(dz, s[5], fma(dy, s[4], dx * s[3])) * fma(dz, s[8], fma(dy, s[7], dx * s[6])) *
                   (rinv2 * rinv2 * rinv);
  a.x = fma(dx, q, a.x);
  a.y = fma(dy, q, a.y);
  a.z = fma(dz, q, a.z);
}

template <int NT>
__global__ void __launch_bounds__(NT, 1152 / NT) k_far_dl_f64_flat(const double* __restrict__ pos,
                                                                    const double* __restrict__ nrm,
                                                                    const double* __restrict__ dden,
                                                                    const long* __restrict__ off, long nves, long N,
                                                                    int seg_tiles, double* __restrict__ part) {
  __shared__ __align__(16) double sm[kTileF64 * 9];
  __shared__ ChunkRange cr;
  chunk_range<NT>(off, nves, N, &cr);
  const int seg = blockIdx.x;
  const long c0 = cr.c0, c1 = cr.c1;
  const long ia = c0 + threadIdx.x, ib = ia + NT;
  const long la = ia < c1 ? ia : c0, lb = ib < c1 ? ib : c0;
  const double ax_ = pos[3 * la], ay_ = pos[3 * la + 1], az_ = pos[3 * la + 2];
  const double bx_ = pos[3 * lb], by_ = pos[3 * lb + 1], bz_ = pos[3 * lb + 2];
  Acc64 A, B;
  const long ntiles = (N + kTileF64 - 1) / kTileF64;
  const long tb = (long)seg * seg_tiles, te = min(tb + seg_tiles, ntiles);
  for (long tile = tb; tile < te; tile++) {
    const long s0 = tile * kTileF64;
    const int ns = (int)min((long)kTileF64, N - s0);
    __syncthreads();
    stage64<9, NT>(sm, pos, nrm, dden, s0, ns);
    __syncthreads();
    int a0, a1, b0, b1;
    split_tile(s0, ns, cr.u0, cr.u1, a0, a1, b0, b1);
    for (int k = a0; k < a1; k++) {
      pair_dl64(sm + 9 * k, ax_, ay_, az_, A);
      pair_dl64(sm + 9 * k, bx_, by_, bz_, B);
    }
    for (int k = b0; k < b1; k++) {
      pair_dl64(sm + 9 * k, ax_, ay_, az_, A);
      pair_dl64(sm + 9 * k, bx_, by_, bz_, B);
    }
  }
  const long g0 = max(cr.u0, tb * kTileF64), g1 = min(cr.u1, min(te * kTileF64, N));
  if (g0 < g1) {
    const long va = vesicle_of(off, nves, la), vb = vesicle_of(off, nves, lb);
    const long ea0 = off[va], ea1 = off[va + 1], eb0 = off[vb], eb1 = off[vb + 1];
    for (long s0 = g0; s0 < g1; s0 += kTileF64) {
      const int ns = (int)min((long)kTileF64, g1 - s0);
      __syncthreads();
      stage64<9, NT>(sm, pos, nrm, dden, s0, ns);
      __syncthreads();
      for (int k = 0; k < ns; k++) {
        const long s = s0 + k;
        if (s < ea0 || s >= ea1) pair_dl64(sm + 9 * k, ax_, ay_, az_, A);
        if (s < eb0 || s >= eb1) pair_dl64(sm + 9 * k, bx_, by_, bz_, B);
      }
    }
  }
  double* P = part + (long)seg * 3 * N;
  if (ia < c1) {
    P[3 * ia] = A.x;
    P[3 * ia + 1] = A.y;
    P[3 * ia + 2] = A.z;
  }
  if (ib < c1) {
    P[3 * ib] = B.x;
    P[3 * ib + 1] = B.y;
    P[3 * ib + 2] = B.z;
  }
}

// ------------------------------------------------------------------------------------
// Mixed (packed FP32 pairs, FP64 accumulation)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// One target's sum over the sources [s0, s1) outside [e0, e1) with coincident pairs
// skipped (|r| = 0 contributes nothing, as in StokesAlltoAll, src/CPUKernels.cc:1030-1040),
// in the pair arithmetic of the mixed kernel (FP32 coordinates relative to the origin
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

// FP32 sources: (x, y, z, dx, dy, dz) relative to the origin cen (shared memory: keeping
// it in registers across the pair loop would cost the loop registers), each broadcast to a
// float2
template <int NT>
__device__ __forceinline__ void stage32(float2* sm, const double* __restrict__ pos, const double* __restrict__ den,
                                        long s0, int ns, const double* cen) {
  const double cx = cen[0], cy = cen[1], cz = cen[2];
#pragma unroll 1
  for (int i = threadIdx.x; i < ns; i += NT) {
    const long s = s0 + i;
    float2* d = sm + 6 * i;
    d[0] = f2((float)(pos[3 * s] - cx));
    d[1] = f2((float)(pos[3 * s + 1] - cy));
    d[2] = f2((float)(pos[3 * s + 2] - cz));
    d[3] = f2((float)den[3 * s]);
    d[4] = f2((float)den[3 * s + 1]);
    d[5] = f2((float)den[3 * s + 2]);
  }
}

// Packed pairs of sources [k0, k1) of the staged tile with the thread's two targets
// (lane x: target a, lane y: target b, negated coordinates), added to u.
__device__ __forceinline__ void pairs_f32(const float2* __restrict__ sm, int k0, int k1, float2 ntx, float2 nty,
                                          float2 ntz, float2& ux, float2& uy, float2& uz) {
#pragma unroll 4
  for (int k = k0; k < k1; k++) {
    const float4* qs = reinterpret_cast<const float4*>(sm + 6 * k);
    const float4 q0 = qs[0], q1 = qs[1], q2 = qs[2];
    const float2 sx = make_float2(q0.x, q0.y), sy = make_float2(q0.z, q0.w);
    const float2 sz = make_float2(q1.x, q1.y), dx_ = make_float2(q1.z, q1.w);
    const float2 dy_ = make_float2(q2.x, q2.y), dz_ = make_float2(q2.z, q2.w);
    // the differences as scalar adds: the packed ops keep one FMA pipe busy (76% of
    // cycles) and the scalar ones can go to the other (measured 1% faster)
    const float2 rx = make_float2(__fadd_rn(sx.x, ntx.x), __fadd_rn(sx.y, ntx.y));
    const float2 ry = make_float2(__fadd_rn(sy.x, nty.x), __fadd_rn(sy.y, nty.y));
    const float2 rz = make_float2(__fadd_rn(sz.x, ntz.x), __fadd_rn(sz.y, ntz.y));
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
    ux = __ffma2_rn(__ffma2_rn(cc, rx, dx_), y, ux);
    uy = __ffma2_rn(__ffma2_rn(cc, ry, dy_), y, uy);
    uz = __ffma2_rn(__ffma2_rn(cc, rz, dz_), y, uz);
  }
}

// Mixed form: coordinates relative to the centroid of the chunk's targets (differences
// taken in FP64, rounded to FP32 once per source per CTA), two targets per thread packed
// in f32x2 lanes, FP32 sums per sub-tile of 120 sources added in FP64. grid (segments,
// target chunks of 2 NT).
template <int NT>
__global__ void __launch_bounds__(NT, 1152 / NT) k_far_f32_flat(const double* __restrict__ pos,
                                                                 const double* __restrict__ den,
                                                                 const long* __restrict__ off, long nves, long N,
                                                                 int seg_tiles, double* __restrict__ part) {
  __shared__ __align__(16) float2 sm[kTileF32 * 6];
  __shared__ ChunkRange cr;
  __shared__ double cen[3];
  __shared__ double red[3][NT / 32];
  chunk_range<NT>(off, nves, N, &cr);
  const int seg = blockIdx.x;
  {  // centroid of the chunk's targets (FP64), the origin of this CTA's FP32 coordinates
    const long c0 = cr.c0, nt = cr.c1 - cr.c0;
    double cx = 0, cy = 0, cz = 0;
#pragma unroll 1
    for (long i = threadIdx.x; i < nt; i += NT) {
      cx += pos[3 * (c0 + i)];
      cy += pos[3 * (c0 + i) + 1];
      cz += pos[3 * (c0 + i) + 2];
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
      for (int i = 0; i < NT / 32; i++) s += red[threadIdx.x][i];
      cen[threadIdx.x] = s / (double)nt;
    }
    __syncthreads();
  }
  float2 ntx, nty, ntz;  // negated targets, packed (lane x = target a, lane y = target b)
  {
    const double cx = cen[0], cy = cen[1], cz = cen[2];
    const long ja = cr.c0 + threadIdx.x, jb = ja + NT;
    const long la = ja < cr.c1 ? ja : cr.c0, lb = jb < cr.c1 ? jb : cr.c0;
    ntx = make_float2((float)(cx - pos[3 * la]), (float)(cx - pos[3 * lb]));
    nty = make_float2((float)(cy - pos[3 * la + 1]), (float)(cy - pos[3 * lb + 1]));
    ntz = make_float2((float)(cz - pos[3 * la + 2]), (float)(cz - pos[3 * lb + 2]));
  }
  double A[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
  const long ntiles = (N + kTileF32 - 1) / kTileF32;
  const long tb = (long)seg * seg_tiles, te = min(tb + seg_tiles, ntiles);
  for (long tile = tb; tile < te; tile++) {
    const long s0 = tile * kTileF32;
    const int ns = (int)min((long)kTileF32, N - s0);
    __syncthreads();
    stage32<NT>(sm, pos, den, s0, ns, cen);
    __syncthreads();
    int r0[2], r1[2];
    split_tile(s0, ns, cr.u0, cr.u1, r0[0], r1[0], r0[1], r1[1]);
    for (int sb = 0; sb < ns; sb += kSubF32) {
      const int se = min(sb + kSubF32, ns);
      float2 ux = f2(0.f), uy = f2(0.f), uz = f2(0.f);
#pragma unroll
      for (int part_i = 0; part_i < 2; part_i++)
        pairs_f32(sm, max(r0[part_i], sb), min(r1[part_i], se), ntx, nty, ntz, ux, uy, uz);
      A[0][0] += ux.x;
      A[0][1] += uy.x;
      A[0][2] += uz.x;
      A[1][0] += ux.y;
      A[1][1] += uy.y;
      A[1][2] += uz.y;
    }
  }
  // the chunk's own vesicles within this segment: each target skips its own vesicle
  const long g0 = max(cr.u0, tb * kTileF32), g1 = min(cr.u1, min(te * kTileF32, N));
  if (g0 < g1) {
    // own-vesicle ranges relative to g0 (int), clamped to the swept range
    const long ja = cr.c0 + threadIdx.x, jb = ja + NT;
    const long va = vesicle_of(off, nves, ja < cr.c1 ? ja : cr.c0), vb = vesicle_of(off, nves, jb < cr.c1 ? jb : cr.c0);
    const int ia0 = (int)max(-1L, off[va] - g0), ia1 = (int)min(g1 - g0, off[va + 1] - g0);
    const int ib0 = (int)max(-1L, off[vb] - g0), ib1 = (int)min(g1 - g0, off[vb + 1] - g0);
    for (long s0 = g0; s0 < g1; s0 += kTileF32) {
      const int ns = (int)min((long)kTileF32, g1 - s0);
      __syncthreads();
      stage32<NT>(sm, pos, den, s0, ns, cen);
      __syncthreads();
      const int so = (int)(s0 - g0);
      for (int sb = 0; sb < ns; sb += kSubF32) {
        const int se = min(sb + kSubF32, ns);
        float2 ux = f2(0.f), uy = f2(0.f), uz = f2(0.f);
        for (int k = sb; k < se; k++) {
          const float2* q6 = sm + 6 * k;
          const float2 rx = make_float2(q6[0].x + ntx.x, q6[0].y + ntx.y);
          const float2 ry = make_float2(q6[1].x + nty.x, q6[1].y + nty.y);
          const float2 rz = make_float2(q6[2].x + ntz.x, q6[2].y + ntz.y);
          float2 r2 = __fmul2_rn(rx, rx);
          r2 = __ffma2_rn(ry, ry, r2);
          r2 = __ffma2_rn(rz, rz, r2);
          float2 y = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
          const int kk = so + k;
          if (kk >= ia0 && kk < ia1) y.x = 0.f;  // a select: the own point's 1/0 is dropped, not multiplied
          if (kk >= ib0 && kk < ib1) y.y = 0.f;
          const float2 y2 = __fmul2_rn(y, y);
          float2 dot = __fmul2_rn(rx, q6[3]);
          dot = __ffma2_rn(ry, q6[4], dot);
          dot = __ffma2_rn(rz, q6[5], dot);
          const float2 cc = __fmul2_rn(dot, y2);
          ux = __ffma2_rn(__ffma2_rn(cc, rx, q6[3]), y, ux);
          uy = __ffma2_rn(__ffma2_rn(cc, ry, q6[4]), y, uy);
          uz = __ffma2_rn(__ffma2_rn(cc, rz, q6[5]), y, uz);
        }
        A[0][0] += ux.x;
        A[0][1] += uy.x;
        A[0][2] += uz.x;
        A[1][0] += ux.y;
        A[1][1] += uy.y;
        A[1][2] += uz.y;
      }
    }
  }
  // A coincident pair of distinct vesicles left a target's sum non-finite: sum the
  // segment again for that target with coincident pairs skipped (non-finite inputs stay
  // non-finite). One test per target and segment; no instruction in the pair loop.
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const long g = cr.c0 + threadIdx.x + (long)j * NT;
    if (g < cr.c1 && !isfinite(A[j][0] + A[j][1] + A[j][2])) {
      // the origin from shared memory again: keeping it in registers across the pair
      // loop would cost the loop registers
      const double gx = cen[0], gy = cen[1], gz = cen[2];
      const long v = vesicle_of(off, nves, g);
      const double3 a = far_f32_guarded(pos, den, (long)blockIdx.x * seg_tiles * kTileF32,
                                        min(((long)blockIdx.x * seg_tiles + seg_tiles) * kTileF32, N), off[v],
                                        off[v + 1], gx, gy, gz, (float)(gx - pos[3 * g]),
                                        (float)(gy - pos[3 * g + 1]), (float)(gz - pos[3 * g + 2]));
      A[j][0] = a.x;
      A[j][1] = a.y;
      A[j][2] = a.z;
    }
  }
  double* P = part + (long)seg * 3 * N;
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const long g = cr.c0 + threadIdx.x + (long)j * NT;
    if (g < cr.c1) {
      P[3 * g] = A[j][0];
      P[3 * g + 1] = A[j][1];
      P[3 * g + 2] = A[j][2];
    }
  }
}

// ---- the far double layer in the mixed form --------------------------------------------
// Pair arithmetic of k_far_dl_f64_flat (u += (t - s) (r.n)(r.g) / |r|^5, r = t - s) in
// packed FP32 pairs: coordinates relative to the centroid of the chunk's targets (FP64
// difference rounded once per source per CTA), the hardware 1/sqrt with one Newton step
// (the kernel takes its fifth power), coincident pairs dropped by a select, FP32 sums per
// sub-tile of kSubDL32 sources added in FP64.
constexpr int kTileDL32 = 640;  // 9 float2 per source: 46 KB staged per barrier pair
constexpr int kSubDL32 = 128;

template <int NT>
__device__ __forceinline__ void stage_dl32(float2* sm, const double* __restrict__ pos, const double* __restrict__ nrm,
                                           const double* __restrict__ dden, long s0, int ns, const double* cen) {
  const double cx = cen[0], cy = cen[1], cz = cen[2];
#pragma unroll 1
  for (int i = threadIdx.x; i < ns; i += NT) {
    const long s = s0 + i;
    float2* d = sm + 9 * i;
    d[0] = f2((float)(pos[3 * s] - cx));
    d[1] = f2((float)(pos[3 * s + 1] - cy));
    d[2] = f2((float)(pos[3 * s + 2] - cz));
    d[3] = f2((float)nrm[3 * s]);
    d[4] = f2((float)nrm[3 * s + 1]);
    d[5] = f2((float)nrm[3 * s + 2]);
    d[6] = f2((float)dden[3 * s]);
    d[7] = f2((float)dden[3 * s + 1]);
    d[8] = f2((float)dden[3 * s + 2]);
  }
}

// One staged source against the thread's two targets (negated, packed); own: the lanes
// whose target belongs to this source's vesicle (their pair is dropped).
__device__ __forceinline__ void pair_dl32(const float2* __restrict__ q, float2 ntx, float2 nty, float2 ntz,
                                          bool own_a, bool own_b, float2& ux, float2& uy, float2& uz) {
  // s - t (the sign of t - s cancels in (r.n)(r.g); the sum takes -(s - t))
  const float2 rx = make_float2(__fadd_rn(q[0].x, ntx.x), __fadd_rn(q[0].y, ntx.y));
  const float2 ry = make_float2(__fadd_rn(q[1].x, nty.x), __fadd_rn(q[1].y, nty.y));
  const float2 rz = make_float2(__fadd_rn(q[2].x, ntz.x), __fadd_rn(q[2].y, ntz.y));
  float2 r2 = __fmul2_rn(rx, rx);
  r2 = __ffma2_rn(ry, ry, r2);
  r2 = __ffma2_rn(rz, rz, r2);
  float2 y = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
  const float2 e = __ffma2_rn(__fmul2_rn(make_float2(-r2.x, -r2.y), y), y, f2(1.f));
  y = __ffma2_rn(__fmul2_rn(f2(0.5f), y), e, y);
  // coincident pairs (|r|^2 below 2^-126) and the target's own vesicle contribute nothing
  y.x = (own_a || !(r2.x >= 1.17549435e-38f)) ? 0.f : y.x;
  y.y = (own_b || !(r2.y >= 1.17549435e-38f)) ? 0.f : y.y;
  float2 rn = __fmul2_rn(rx, q[3]);
  rn = __ffma2_rn(ry, q[4], rn);
  rn = __ffma2_rn(rz, q[5], rn);
  float2 rg = __fmul2_rn(rx, q[6]);
  rg = __ffma2_rn(ry, q[7], rg);
  rg = __ffma2_rn(rz, q[8], rg);
  const float2 y2 = __fmul2_rn(y, y);
  const float2 y5 = __fmul2_rn(__fmul2_rn(y2, y2), y);
  const float2 nq = __fmul2_rn(__fmul2_rn(rn, rg), make_float2(-y5.x, -y5.y));
  ux = __ffma2_rn(rx, nq, ux);
  uy = __ffma2_rn(ry, nq, uy);
  uz = __ffma2_rn(rz, nq, uz);
}

template <int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) k_far_dl_f32_flat(const double* __restrict__ pos,
                                                                    const double* __restrict__ nrm,
                                                                    const double* __restrict__ dden,
                                                                    const long* __restrict__ off, long nves, long N,
                                                                    int seg_tiles, double* __restrict__ part) {
  __shared__ __align__(16) float2 sm[kTileDL32 * 9];
  __shared__ ChunkRange cr;
  __shared__ double cen[3];
  __shared__ double red[3][NT / 32];
  chunk_range<NT>(off, nves, N, &cr);
  const int seg = blockIdx.x;
  {  // centroid of the chunk's targets (FP64), the origin of this CTA's FP32 coordinates
    const long c0 = cr.c0, nt = cr.c1 - cr.c0;
    double cx = 0, cy = 0, cz = 0;
#pragma unroll 1
    for (long i = threadIdx.x; i < nt; i += NT) {
      cx += pos[3 * (c0 + i)];
      cy += pos[3 * (c0 + i) + 1];
      cz += pos[3 * (c0 + i) + 2];
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
      double sum = 0;
      for (int i = 0; i < NT / 32; i++) sum += red[threadIdx.x][i];
      cen[threadIdx.x] = sum / (double)nt;
    }
    __syncthreads();
  }
  const long ja = cr.c0 + threadIdx.x, jb = ja + NT;
  const long la = ja < cr.c1 ? ja : cr.c0, lb = jb < cr.c1 ? jb : cr.c0;
  float2 ntx, nty, ntz;  // negated targets, packed (lane x = target a, lane y = target b)
  {
    const double cx = cen[0], cy = cen[1], cz = cen[2];
    ntx = make_float2((float)(cx - pos[3 * la]), (float)(cx - pos[3 * lb]));
    nty = make_float2((float)(cy - pos[3 * la + 1]), (float)(cy - pos[3 * lb + 1]));
    ntz = make_float2((float)(cz - pos[3 * la + 2]), (float)(cz - pos[3 * lb + 2]));
  }
  double A[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
  auto flush = [&](float2 ux, float2 uy, float2 uz) {
    A[0][0] += ux.x;
    A[0][1] += uy.x;
    A[0][2] += uz.x;
    A[1][0] += ux.y;
    A[1][1] += uy.y;
    A[1][2] += uz.y;
  };
  const long ntiles = (N + kTileDL32 - 1) / kTileDL32;
  const long tb = (long)seg * seg_tiles, te = min(tb + seg_tiles, ntiles);
  for (long tile = tb; tile < te; tile++) {
    const long s0 = tile * kTileDL32;
    const int ns = (int)min((long)kTileDL32, N - s0);
    __syncthreads();
    stage_dl32<NT>(sm, pos, nrm, dden, s0, ns, cen);
    __syncthreads();
    int r0[2], r1[2];
    split_tile(s0, ns, cr.u0, cr.u1, r0[0], r1[0], r0[1], r1[1]);
    for (int sb = 0; sb < ns; sb += kSubDL32) {
      const int se = min(sb + kSubDL32, ns);
      float2 ux = f2(0.f), uy = f2(0.f), uz = f2(0.f);
#pragma unroll
      for (int part_i = 0; part_i < 2; part_i++) {
        const int k1 = min(r1[part_i], se);
#pragma unroll 2
        for (int k = max(r0[part_i], sb); k < k1; k++) pair_dl32(sm + 9 * k, ntx, nty, ntz, false, false, ux, uy, uz);
      }
      flush(ux, uy, uz);
    }
  }
  // the chunk's own vesicles within this segment: each target skips its own vesicle
  const long g0 = max(cr.u0, tb * kTileDL32), g1 = min(cr.u1, min(te * kTileDL32, N));
  if (g0 < g1) {
    const long va = vesicle_of(off, nves, la), vb = vesicle_of(off, nves, lb);
    const long ea0 = off[va], ea1 = off[va + 1], eb0 = off[vb], eb1 = off[vb + 1];
    for (long s0 = g0; s0 < g1; s0 += kTileDL32) {
      const int ns = (int)min((long)kTileDL32, g1 - s0);
      __syncthreads();
      stage_dl32<NT>(sm, pos, nrm, dden, s0, ns, cen);
      __syncthreads();
      for (int sb = 0; sb < ns; sb += kSubDL32) {
        const int se = min(sb + kSubDL32, ns);
        float2 ux = f2(0.f), uy = f2(0.f), uz = f2(0.f);
        for (int k = sb; k < se; k++) {
          const long sg = s0 + k;
          pair_dl32(sm + 9 * k, ntx, nty, ntz, sg >= ea0 && sg < ea1, sg >= eb0 && sg < eb1, ux, uy, uz);
        }
        flush(ux, uy, uz);
      }
    }
  }
  double* P = part + (long)seg * 3 * N;
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const long g = cr.c0 + threadIdx.x + (long)j * NT;
    if (g < cr.c1) {
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
// (segments) and the threads of a CTA (two targets each).
struct FarShape {
  int waves = 8;
  int nthr = 384;
};

// Default shapes, measured at 512 vesicles of p = 16 (one B200): FP64 16 waves of
// 384-thread CTAs (122.5 ms); FP32 16 waves of 256-thread CTAs (384-thread chunks ran 46.3 ms
// with a larger worst-point error, 5.0e-7 against 3.2e-7: their origins lie farther from
// some of their targets, so the FP32 form tunes over 256-thread CTAs only).
static FarShape default_shape(bool mixed) { return mixed ? FarShape{16, 256} : FarShape{16, 384}; }

static int num_sms() {
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return nsm;
}

// Segments of the source tiles for nchunk target chunks: about waves x (resident CTAs) x
// SMs CTAs in all, at most part_cap_segments.
static int far_segments(long nchunk, long N, int tile, int nthr, int waves, long part_cap_segments, int* seg_tiles) {
  const long ntiles = (N + tile - 1) / tile;
  const int per_sm = max(1, 1152 / max(nthr, 32));  // resident CTAs per SM (the kernels' launch bounds)
  const long want = (long)num_sms() * per_sm * waves;
  long nseg = (want + nchunk - 1) / nchunk;
  nseg = std::max(1L, std::min(nseg, std::min(ntiles, part_cap_segments)));
  *seg_tiles = (int)((ntiles + nseg - 1) / nseg);
  return (int)((ntiles + *seg_tiles - 1) / *seg_tiles);
}

int launch_far_reduce(const double* part, int nseg, const long* off, long nves, long N, const double* add, double* out,
                      double* far_out, cudaStream_t st, const double* part2, int nseg2, double scale2) {
  k_far_reduce<<<(unsigned)nves, 256, 0, st>>>(part, nseg, off, N, add, out, far_out, part2, nseg2, scale2);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

// One launch of the single-layer far field (segments only; the partials stay in part).
static int launch_far_shape(const FarShape& sh, bool mixed, const double* pos, const double* den, const long* off,
                            long nves, long N, double* part, long part_cap_segments, cudaStream_t st, int* nseg_out) {
  const long nchunk = (N + 2L * sh.nthr - 1) / (2L * sh.nthr);
  if (nchunk > 65535) {
    set_error("far field: %ld points exceed the launch's %ld target chunks", N, 65535L * 2 * sh.nthr);
    return VES3D_ERR_ARG;
  }
  int seg_tiles = 1;
  const int nseg = far_segments(nchunk, N, mixed ? kTileF32 : kTileF64, sh.nthr, sh.waves, part_cap_segments,
                                &seg_tiles);
  dim3 grid((unsigned)nseg, (unsigned)nchunk);
  if (mixed && sh.nthr == 384)
    k_far_f32_flat<384><<<grid, 384, 0, st>>>(pos, den, off, nves, N, seg_tiles, part);
  else if (mixed)
    k_far_f32_flat<256><<<grid, 256, 0, st>>>(pos, den, off, nves, N, seg_tiles, part);
  else if (sh.nthr == 384)
    k_far_f64_flat<384><<<grid, 384, 0, st>>>(pos, den, off, nves, N, seg_tiles, part);
  else
    k_far_f64_flat<256><<<grid, 256, 0, st>>>(pos, den, off, nves, N, seg_tiles, part);
  VES3D_LAUNCHED();
  *nseg_out = nseg;
  return VES3D_OK;
}

// ---- autotuner of the launch shape ----------------------------------------------------
// On the first launch of a configuration (precision, N, vesicles and their sizes) with
// autotuning on, every candidate shape is launched once and timed with CUDA events on the
// caller's stream; the fastest is cached for the process. Off by default and never during
// stream capture. Candidates differ in how the source range is split and in the chunks of
// targets, i.e. in the grouping of the FP64 partial sums (and, in the FP32 form, in the
// origin of a chunk's coordinates): results agree to rounding. A tuned configuration
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

static FarShape g_forced{0, 0};  // a caller-fixed shape (waves 0 = none)

int set_far_shape(int waves, int nthr, int tpt) {
  if (waves == 0) {
    g_forced = FarShape{0, 0};
    return VES3D_OK;
  }
  if ((waves != 4 && waves != 8 && waves != 16) || (nthr != 256 && nthr != 384) || tpt != 2) {
    set_error("far shape: waves in {4, 8, 16}, threads per CTA in {256, 384}, targets per thread 2");
    return VES3D_ERR_ARG;
  }
  g_forced = FarShape{waves, nthr};
  return VES3D_OK;
}

static int tuned_shape(bool mixed, const double* pos, const double* den, const long* off, long nves, long N,
                       const FarGroup* groups, int ngroups, double* part, long part_cap_segments, cudaStream_t st,
                       FarShape* shape) {
  *shape = default_shape(mixed);
  if (g_forced.waves) {
    *shape = g_forced;
    return VES3D_OK;
  }
  if (!autotune_on()) return VES3D_OK;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  VES3D_CK(cudaStreamIsCapturing(st, &cap));
  const std::string key = tune_key(mixed, nves, N, groups, ngroups);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
      *shape = it->second.shape;
      return VES3D_OK;
    }
  }
  if (cap != cudaStreamCaptureStatusNone) return VES3D_OK;
  cudaEvent_t e0, e1;
  VES3D_CK(cudaEventCreate(&e0));
  VES3D_CK(cudaEventCreate(&e1));
  FarTuneEntry best;
  best.ms = 1e30f;
  int s = VES3D_OK;
  for (int nthr : {256, 384})
    for (int waves : {4, 8, 16}) {
      if (mixed && nthr != 256) continue;
      const FarShape c{waves, nthr};
      cudaEventRecord(e0, st);
      int nseg = 0;
      if ((s = launch_far_shape(c, mixed, pos, den, off, nves, N, part, part_cap_segments, st, &nseg))) break;
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
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned[key] = best;
  *shape = best.shape;
  return VES3D_OK;
}

int launch_far_groups(bool mixed, const double* pos, const double* den, const long* off, long nves, long N,
                      const FarGroup* groups, int ngroups, const double* add, double* out, double* far_out,
                      double* part, long part_cap_segments, cudaStream_t st, int* nseg_out) {
  if (N <= 0) {
    if (nseg_out) *nseg_out = 0;
    return VES3D_OK;
  }
  FarShape shape;
  int s = tuned_shape(mixed, pos, den, off, nves, N, groups, ngroups, part, part_cap_segments, st, &shape);
  if (s) return s;
  int nseg = 0;
  if ((s = launch_far_shape(shape, mixed, pos, den, off, nves, N, part, part_cap_segments, st, &nseg))) return s;
  if (nseg_out) {
    *nseg_out = nseg;
    return VES3D_OK;
  }
  return launch_far_reduce(part, nseg, off, nves, N, add, out, far_out, st);
}

int set_autotune(int on) {
  g_autotune.store(on ? 1 : 0);
  return VES3D_OK;
}

// "key waves threads ms" per tuned configuration, one per line
std::string autotune_report() {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  std::string r;
  for (const auto& kv : g_tuned)
    r += kv.first + " waves=" + std::to_string(kv.second.shape.waves) + " threads=" +
         std::to_string(kv.second.shape.nthr) + " ms=" + std::to_string(kv.second.ms) + "\n";
  return r;
}

// The far double layer over every point, one launch whatever the vesicle sizes: FP64, or
// packed FP32 pairs with FP64 sub-tile sums in the mixed form.
int launch_far_dl_groups(bool mixed, const double* pos, const double* nrm, const double* dden, const long* off,
                         long nves, long N, const FarGroup* groups, int ngroups, double* part, long part_cap_segments,
                         cudaStream_t st, int* nseg_out) {
  (void)groups;
  (void)ngroups;
  *nseg_out = 0;
  if (N <= 0 || nves <= 0) return VES3D_OK;
  if (mixed) {
    constexpr int NT = 256;
    const long nchunk = (N + 2L * NT - 1) / (2L * NT);
    if (nchunk > 65535) {
      set_error("far double layer: %ld points exceed the launch's %ld target chunks", N, 65535L * 2 * NT);
      return VES3D_ERR_ARG;
    }
    int seg_tiles = 1;
    const int nseg = far_segments(nchunk, N, kTileDL32, NT, 16, part_cap_segments, &seg_tiles);
    k_far_dl_f32_flat<NT><<<dim3((unsigned)nseg, (unsigned)nchunk), NT, 0, st>>>(pos, nrm, dden, off, nves, N,
                                                                                 seg_tiles, part);
    VES3D_LAUNCHED();
    *nseg_out = nseg;
    return VES3D_OK;
  }
  constexpr int NT = 384;
  const long nchunk = (N + 2L * NT - 1) / (2L * NT);
  if (nchunk > 65535) {
    set_error("far double layer: %ld points exceed the launch's %ld target chunks", N, 65535L * 2 * NT);
    return VES3D_ERR_ARG;
  }
  int seg_tiles = 1;
  const int nseg = far_segments(nchunk, N, kTileF64, NT, 8, part_cap_segments, &seg_tiles);
  k_far_dl_f64_flat<NT><<<dim3((unsigned)nseg, (unsigned)nchunk), NT, 0, st>>>(pos, nrm, dden, off, nves, N,
                                                                               seg_tiles, part);
  VES3D_LAUNCHED();
  *nseg_out = nseg;
  return VES3D_OK;
}

int launch_far_dl(bool mixed, const double* pos, const double* nrm, const double* dden, const long* off, long nves,
                  long N, int max_nt, double* part, long part_cap_segments, cudaStream_t st, int* nseg_out) {
  FarGroup g{0, nves, max_nt};
  return launch_far_dl_groups(mixed, pos, nrm, dden, off, nves, N, &g, 1, part, part_cap_segments, st, nseg_out);
}

int launch_far(bool mixed, const double* pos, const double* den, const long* off, long nves, long N, int max_nt,
               const double* add, double* out, double* far_out, double* part, long part_cap_segments,
               cudaStream_t st, int* nseg_out) {
  FarGroup g{0, nves, max_nt};
  return launch_far_groups(mixed, pos, den, off, nves, N, &g, 1, add, out, far_out, part, part_cap_segments, st,
                           nseg_out);
}

}  // namespace ves3d
