// Near-singular correction of the velocity at off-surface targets (FP64): the
// interpolation scheme of NearSingular<Real_t>::operator() (src/NearSingular.cc:1356-1555)
// as StokesVelocity<Real>::operator() composes it for SetTrgCoord targets
// (src/StokesVelocity.cc:475-500).
//
//   every target: the smooth quadrature of every vesicle at the far upsampling order
//   p_up (the reference's far field over its upsampled sources, :476-489);
//   a target closer than r_near = r_ves 2 / sqrt(p_up) to a vesicle (r_ves the largest
//   distance of a surface point from its vesicle's centroid, src/NearSingular.cc:119-160):
//   that vesicle's smooth contribution (SubtractDirect, :1144-1212) is replaced by the
//   Lagrange interpolation (InterPoints / InterPoly, :1356-1374) of 8 values along the line
//   from the target's projection P on the surface through the target: at x = 0 the
//   vesicle's own singular-quadrature velocity at P (plus, with a double layer, g(P)/2
//   outside and -g(P)/2 inside: the jump, :1474-1481), at x_l = 1 + (l - 1)/6, l = 1..7,
//   the smooth quadrature at P + r_near x_l d; evaluated at x = |T - P| / r_near.
//
// The reference finds near pairs with a pvfmm octree and projects on quadratic patches of
// 3 x 3 grid points; here a target's near vesicles come from a bounding-sphere test and
// its distance to the vesicle's upsampled points (up to kNearMax per target, ascending
// vesicle order), and the projection is Gauss-Newton on the spherical-harmonic surface
// itself from the nearest upsampled point: one warp per (target, vesicle) pair, lane m
// carrying the order-m Legendre recurrence. The on-surface velocity and density at P come
// from their coefficients the same way. Each pair's correction is written to its own slot
// and the slots are added in order (deterministic).
#include "common.cuh"
#include "kernels.h"

namespace ves3d {

namespace {

constexpr int kInterpDeg = 8;
constexpr double kSqrt2Pi = 2.5066282746310002;

__device__ __forceinline__ double inter_point(int i) { return i ? 1.0 + (i - 1.0) / (kInterpDeg - 2) : 0.0; }

__device__ double inter_poly(double x, int j) {
  double y = 1.0;
  const double x0 = inter_point(j);
  for (int k = 0; k < kInterpDeg; k++)
    if (k != j) y *= (x - inter_point(k)) / (x0 - inter_point(k));
  return y;
}

// Per vesicle: centroid of its order-p points, the largest distance of a point from it
// (cen_r[v] = (cx, cy, cz, R)), and the global maximum R as an ordered integer.
__global__ void k_centroid_radius(const double* __restrict__ X, int ng, double* __restrict__ cen_r,
                                  unsigned long long* __restrict__ rmax_bits) {
  __shared__ double red[3][256];
  const long v = blockIdx.x;
  const double* x = X + v * 3 * ng;
  double s[3] = {0, 0, 0};
  for (int i = threadIdx.x; i < ng; i += blockDim.x)
    for (int d = 0; d < 3; d++) s[d] += x[d * ng + i];
  for (int d = 0; d < 3; d++) red[d][threadIdx.x] = s[d];
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
      for (int d = 0; d < 3; d++) red[d][threadIdx.x] += red[d][threadIdx.x + h];
    __syncthreads();
  }
  const double c0 = red[0][0] / ng, c1 = red[1][0] / ng, c2 = red[2][0] / ng;
  __syncthreads();
  double m = 0.0;
  for (int i = threadIdx.x; i < ng; i += blockDim.x) {
    const double dx = x[i] - c0, dy = x[ng + i] - c1, dz = x[2 * ng + i] - c2;
    m = fmax(m, dx * dx + dy * dy + dz * dz);
  }
  red[0][threadIdx.x] = m;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[0][threadIdx.x] = fmax(red[0][threadIdx.x], red[0][threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double R = sqrt(red[0][0]);
    cen_r[4 * v] = c0;
    cen_r[4 * v + 1] = c1;
    cen_r[4 * v + 2] = c2;
    cen_r[4 * v + 3] = R;
    atomicMax(rmax_bits, (unsigned long long)__double_as_longlong(R));  // R >= 0: bits order as values
  }
}

// Near vesicles of each target: up to kNearMax in ascending vesicle order, with the index
// of the nearest upsampled point; count[t] = their number, or kNearMax + 1 when more.
__global__ void k_near_find(const double* __restrict__ trg, long M, const double* __restrict__ cen_r, long nv,
                            const double* __restrict__ pos_up, int ng1, double r_near, int* __restrict__ count,
                            int* __restrict__ near_v, int* __restrict__ near_k) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M) return;
  const double tx = trg[3 * t], ty = trg[3 * t + 1], tz = trg[3 * t + 2];
  const double rn2 = r_near * r_near;
  int cnt = 0;
  for (long v = 0; v < nv; v++) {
    const double dx = tx - cen_r[4 * v], dy = ty - cen_r[4 * v + 1], dz = tz - cen_r[4 * v + 2];
    // upsampled points lie within about R of the centroid; a generous bound
    const double reach = 1.25 * cen_r[4 * v + 3] + r_near;
    if (dx * dx + dy * dy + dz * dz > reach * reach) continue;
    const double* P = pos_up + 3 * v * (long)ng1;
    double best = rn2;
    int kb = -1;
    for (int k = 0; k < ng1; k++) {
      const double ex = P[3 * k] - tx, ey = P[3 * k + 1] - ty, ez = P[3 * k + 2] - tz;
      const double d2 = ex * ex + ey * ey + ez * ez;
      if (d2 < best) {
        best = d2;
        kb = k;
      }
    }
    if (kb < 0) continue;
    if (cnt < kNearMax) {
      near_v[t * kNearMax + cnt] = (int)v;
      near_k[t * kNearMax + cnt] = kb;
    }
    cnt++;
  }
  count[t] = cnt <= kNearMax ? cnt : kNearMax + 1;
}

// Sums over lane m of the order-m blocks of the coefficients: value, d/dtheta, d/dphi of
// the 3 functions S[3][nc] at (x = cos theta, phi), reduced over the warp (all lanes get
// them). Lane m < p + 1 runs the normalised associated Legendre recurrence of order m
// (the reference's LegPoly / LegPolyDeriv, src/SphericalHarmonics.cc:889-950; P(m + 1, n)
// for the derivative comes from lane m + 1).
__device__ void sh_point(const double* __restrict__ S, int p, const int* __restrict__ blk_off, double x, double phi,
                         bool grads, double* val) {
  const int lane = threadIdx.x & 31;
  const int m = lane;
  const int nc = p * (p + 2);
  const double s = sqrt(fmax(1.0 - x * x, 0.0));
  double acc[9];
#pragma unroll
  for (int i = 0; i < 9; i++) acc[i] = 0.0;
  // diagonal P(m, m)
  double pmm = 0.28209479177387814;  // 1/sqrt(4 pi)
  for (int i = 1; i <= m && i <= p; i++) pmm = -pmm * s * sqrt((2.0 * i + 1.0) / (2.0 * i));
  double cm = 1.0, sm = 0.0, dcm = 0.0, dsm = 0.0;
  if (m <= p) {
    sincos(m * phi, &sm, &cm);
    dcm = -m * sm;
    dsm = m * cm;
  }
  const int jc = m == 0 ? 0 : (m == p ? 2 * p - 1 : 2 * m - 1);  // cos block of order m
  const int js = (m >= 1 && m < p) ? 2 * m : -1;                  // sin block
  const int oc = m <= p ? blk_off[jc] : 0, os = js >= 0 ? blk_off[js] : 0;
  double pm2 = 0.0, pm1 = pmm;
  for (int n = 0; n <= p; n++) {
    double pn = 0.0;
    if (m <= p && n >= m) {
      if (n == m) {
        pn = pmm;
      } else {
        const double a = sqrt(((2.0 * n - 1) * (2.0 * n + 1)) / ((double)(n - m) * (n + m)));
        const double b = n > 1 ? sqrt(((2.0 * n + 1) * (n + m - 1) * (n - m - 1)) / ((double)(n - m) * (n + m) * (2 * n - 3)))
                               : 0.0;
        pn = x * a * pm1 - b * pm2;
        pm2 = pm1;
        pm1 = pn;
      }
    }
    // P(m + 1, n) from the next lane (0 beyond the diagonal) for the theta derivative
    const double pnext = __shfl_down_sync(0xffffffffu, pn, 1);
    if (m <= p && n >= m) {
      const double c2 = m + 1 <= n ? sqrt(n + m + 1.0) * sqrt((double)(n - m)) : 0.0;
      // -(legpoly_deriv) = d/dtheta of P(m, n)(cos theta)
      const double dpn = s > 0.0 ? (m * x * pn + c2 * s * (m + 1 <= n ? pnext : 0.0)) / s : 0.0;
      const int ic = oc + (n - m);
      for (int d = 0; d < 3; d++) {
        const double a = S[(long)d * nc + ic];
        acc[d] += a * pn * cm;
        if (grads) {
          acc[3 + d] += a * dpn * cm;
          acc[6 + d] += a * pn * dcm;
        }
      }
      if (js >= 0) {
        const int is = os + (n - m);
        for (int d = 0; d < 3; d++) {
          const double a = S[(long)d * nc + is];
          acc[d] += a * pn * sm;
          if (grads) {
            acc[3 + d] += a * dpn * sm;
            acc[6 + d] += a * pn * dsm;
          }
        }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 9; i++) {
    double v = acc[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    val[i] = kSqrt2Pi * v;
  }
}

struct NearArgs {
  const double* trg;
  const int* count;
  const int* near_v;
  const int* near_k;
  const double* Sx;      // [nv][3][nc] position coefficients
  const double* Vc;      // [nv][3][nc] self-velocity coefficients (single + double layer)
  const double* Gc;      // [nv][3][nc] double-layer density coefficients, or null
  const double* pos_up;  // [nv ng1][3]
  const double* den_up;
  const double* nrm_up;  // null without a double layer
  const double* dden_up;
  const double* theta_up;  // [p_up + 1] latitudes of the upsampled grid
  const int* blk_off;
  int p, p_up;
  double r_near;
  double* corr;  // [M][kNearMax][3]
};

// One CTA of 128 threads per (target, slot): warp 0 projects the target on the vesicle
// and evaluates the on-surface values at the projection; then all threads sum the smooth
// quadrature at the 7 line points and at the target; thread 0 writes the correction.
__global__ void __launch_bounds__(128) k_near_correct(NearArgs A) {
  const long t = blockIdx.x / kNearMax;
  const int slot = blockIdx.x - (int)(t * kNearMax);
  const int cnt = A.count[t];
  if (slot >= cnt || cnt > kNearMax) return;
  __shared__ double sh[8 * 3];   // line points (7) and the target
  __shared__ double s_y0[3];     // on-surface value at the projection
  __shared__ double s_x;         // |T - P| / r_near
  __shared__ double red[4][8 * 3];
  const int v = A.near_v[t * kNearMax + slot], k0 = A.near_k[t * kNearMax + slot];
  const int p = A.p, nc = p * (p + 2), ng1 = 2 * A.p_up * (A.p_up + 1);
  const double tx = A.trg[3 * t], ty = A.trg[3 * t + 1], tz = A.trg[3 * t + 2];
  if (threadIdx.x < 32) {
    const double* S = A.Sx + (long)v * 3 * nc;
    double th = A.theta_up[k0 / (2 * A.p_up)], ph = M_PI * (k0 % (2 * A.p_up)) / A.p_up;
    double val[9];
    for (int itn = 0; itn < 40; itn++) {  // Gauss-Newton on |X(theta, phi) - T|^2
      sh_point(S, p, A.blk_off, cos(th), ph, true, val);
      const double rx = val[0] - tx, ry = val[1] - ty, rz = val[2] - tz;
      const double a11 = val[3] * val[3] + val[4] * val[4] + val[5] * val[5];
      const double a12 = val[3] * val[6] + val[4] * val[7] + val[5] * val[8];
      const double a22 = val[6] * val[6] + val[7] * val[7] + val[8] * val[8];
      const double g1 = val[3] * rx + val[4] * ry + val[5] * rz, g2 = val[6] * rx + val[7] * ry + val[8] * rz;
      const double reg = 1e-14 * (a11 + a22);
      const double b11 = a11 + reg, b22 = a22 + reg, det = b11 * b22 - a12 * a12;
      const double d1 = -(b22 * g1 - a12 * g2) / det, d2 = -(b11 * g2 - a12 * g1) / det;
      th += d1;
      ph += d2;
      if (fmax(fabs(d1), fabs(d2)) < 1e-15) break;
    }
    sh_point(S, p, A.blk_off, cos(th), ph, true, val);
    const double px = val[0], py = val[1], pz = val[2];
    // outward normal X_theta x X_phi (the orientation of the library's unit normals)
    double nx = val[4] * val[8] - val[5] * val[7], ny = val[5] * val[6] - val[3] * val[8],
           nz = val[3] * val[7] - val[4] * val[6];
    const double nn = sqrt(nx * nx + ny * ny + nz * nz);
    nx /= nn;
    ny /= nn;
    nz /= nn;
    const double dx = tx - px, dy = ty - py, dz = tz - pz;
    const double dist = sqrt(dx * dx + dy * dy + dz * dz);
    const bool exterior = dx * nx + dy * ny + dz * nz >= 0.0;
    double ux = nx, uy = ny, uz = nz;
    if (dist > 0.0) {
      ux = dx / dist;
      uy = dy / dist;
      uz = dz / dist;
    }
    double vs[9];
    sh_point(A.Vc + (long)v * 3 * nc, p, A.blk_off, cos(th), ph, false, vs);
    double y0[3] = {vs[0], vs[1], vs[2]};
    if (A.Gc) {
      double gs[9];
      sh_point(A.Gc + (long)v * 3 * nc, p, A.blk_off, cos(th), ph, false, gs);
      const double jump = exterior ? 0.5 : -0.5;
      for (int d = 0; d < 3; d++) y0[d] += jump * gs[d];
    }
    if (threadIdx.x == 0) {
      for (int l = 1; l < kInterpDeg; l++) {
        const double r = A.r_near * inter_point(l);
        sh[3 * (l - 1)] = px + r * ux;
        sh[3 * (l - 1) + 1] = py + r * uy;
        sh[3 * (l - 1) + 2] = pz + r * uz;
      }
      sh[21] = tx;
      sh[22] = ty;
      sh[23] = tz;
      for (int d = 0; d < 3; d++) s_y0[d] = y0[d];
      s_x = dist / A.r_near;
    }
  }
  __syncthreads();
  // smooth upsampled quadrature of vesicle v at the 8 points
  double acc[24];
#pragma unroll
  for (int i = 0; i < 24; i++) acc[i] = 0.0;
  const double* P = A.pos_up + 3 * (long)v * ng1;
  const double* D = A.den_up + 3 * (long)v * ng1;
  const double* Nn = A.nrm_up ? A.nrm_up + 3 * (long)v * ng1 : nullptr;
  const double* G = A.dden_up ? A.dden_up + 3 * (long)v * ng1 : nullptr;
  for (int s = threadIdx.x; s < ng1; s += blockDim.x) {
    const double sx = P[3 * s], sy = P[3 * s + 1], sz = P[3 * s + 2];
    const double fx = D[3 * s], fy = D[3 * s + 1], fz = D[3 * s + 2];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      // single layer: r = source - point (src/CPUKernels.cc:1011-1057)
      const double rx = sx - sh[3 * q], ry = sy - sh[3 * q + 1], rz = sz - sh[3 * q + 2];
      const double r2 = rx * rx + ry * ry + rz * rz;
      const double ri = r2 > 0.0 ? rsqrt_f64(r2) : 0.0;
      const double c = (rx * fx + ry * fy + rz * fz) * ri * ri;
      acc[3 * q] += (fx + c * rx) * ri * kInv8Pi;
      acc[3 * q + 1] += (fy + c * ry) * ri * kInv8Pi;
      acc[3 * q + 2] += (fz + c * rz) * ri * kInv8Pi;
      if (Nn) {  // double layer: r = point - source, 3/(4 pi) (r.n)(r.g) r / |r|^5
        const double rn = -(rx * Nn[3 * s] + ry * Nn[3 * s + 1] + rz * Nn[3 * s + 2]);
        const double rg = -(rx * G[3 * s] + ry * G[3 * s + 1] + rz * G[3 * s + 2]);
        const double w = kDl * rn * rg * ri * ri * ri * ri * ri;
        acc[3 * q] -= w * rx;
        acc[3 * q + 1] -= w * ry;
        acc[3 * q + 2] -= w * rz;
      }
    }
  }
  // fixed-order reduction: warp shuffles, then the 4 warps in order
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < 24; i++) {
    double a = acc[i];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) red[warp][i] = a;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int d = threadIdx.x;
    double y[kInterpDeg];
    y[0] = s_y0[d];
    for (int l = 1; l < kInterpDeg; l++)
      y[l] = ((red[0][3 * (l - 1) + d] + red[1][3 * (l - 1) + d]) + (red[2][3 * (l - 1) + d] + red[3][3 * (l - 1) + d]));
    const double direct = (red[0][21 + d] + red[1][21 + d]) + (red[2][21 + d] + red[3][21 + d]);
    double interp = 0.0;
    for (int l = 0; l < kInterpDeg; l++) interp += y[l] * inter_poly(s_x, l);
    A.corr[(t * kNearMax + slot) * 3 + d] = interp - direct;
  }
}

// vel[t] += the corrections of its near vesicles, in slot order
__global__ void k_near_add(const int* __restrict__ count, const double* __restrict__ corr, long M,
                           double* __restrict__ vel) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M) return;
  const int cnt = count[t];
  for (int s = 0; s < cnt && s < kNearMax; s++)
    for (int d = 0; d < 3; d++) vel[3 * t + d] += corr[(t * kNearMax + s) * 3 + d];
}

}  // namespace

int launch_centroid_radius(const double* X, long nv, int p, double* cen_r, unsigned long long* rmax_bits,
                           cudaStream_t st) {
  if (nv <= 0) return VES3D_OK;
  VES3D_CK(cudaMemsetAsync(rmax_bits, 0, sizeof(unsigned long long), st));
  k_centroid_radius<<<(unsigned)nv, 256, 0, st>>>(X, ngrid_(p), cen_r, rmax_bits);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

int launch_near_find(const double* trg, long M, const double* cen_r, long nv, const double* pos_up, int p_up,
                     double r_near, int* count, int* near_v, int* near_k, cudaStream_t st) {
  if (M <= 0) return VES3D_OK;
  k_near_find<<<(unsigned)((M + 127) / 128), 128, 0, st>>>(trg, M, cen_r, nv, pos_up, ngrid_(p_up), r_near, count,
                                                          near_v, near_k);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

int launch_near_correct(const double* trg, long M, const int* count, const int* near_v, const int* near_k,
                        const double* Sx, const double* Vc, const double* Gc, const double* pos_up,
                        const double* den_up, const double* nrm_up, const double* dden_up, const double* theta_up,
                        const int* blk_off, int p, int p_up, double r_near, double* corr, double* vel,
                        cudaStream_t st) {
  if (M <= 0) return VES3D_OK;
  if (p + 1 > 32) {
    set_error("near-singular correction: orders up to 31");
    return VES3D_ERR_ARG;
  }
  NearArgs a{trg, count, near_v, near_k, Sx, Vc, Gc, pos_up, den_up, nrm_up, dden_up, theta_up, blk_off,
             p, p_up, r_near, corr};
  k_near_correct<<<(unsigned)(M * kNearMax), 128, 0, st>>>(a);
  VES3D_LAUNCHED();
  k_near_add<<<(unsigned)((M + 127) / 128), 128, 0, st>>>(count, corr, M, vel);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

}  // namespace ves3d
