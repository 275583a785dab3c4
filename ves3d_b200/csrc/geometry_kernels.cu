// Surface geometry and interfacial forces on the device (FP64), pointwise parts.
// The derivative fields come from the synthesis kernels (sht_kernels.cu); here they are
// combined per point exactly as the reference does:
//   first forms, normal, div/grad vectors     Surface::updateFirstForms  src/Surface.cc:212-262
//   mean / Gaussian curvature                 Surface::updateAll          src/Surface.cc:264-323
//   gradient, divergence                      Surface::grad / div         src/Surface.cc:325-379
//   linearised mean curvature                 Surface::linearizedMeanCurv src/Surface.cc:530-569
//   bending and tension tractions             InterfacialForce            src/InterfacialForce.cc:21-125
// u is the latitude (Legendre-derivative) direction and v the longitude (Fourier) one.
// Fields are AxisMajor per vesicle, [nv][comp][ng]; the geometry record has kGeoComps
// components per point (see kernels.h).
#include "common.cuh"
#include "kernels.h"

namespace ves3d {

#define FOR_POINTS(N)                                                 \
  const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;        \
  if (g >= (N)) return;                                               \
  const long v = g / ng, k = g - v * ng;

// Fields may hold several copies of the suspension (batched operator applications):
// field vesicle v uses the geometry of vesicle v % geo_nv.
#define GEO_OF(v) (geo + ((v) % geo_nv) * kGeoComps * (long)ng + k)

__global__ void k_geometry(const double* __restrict__ xu, const double* __restrict__ xv,
                           const double* __restrict__ xuu, const double* __restrict__ xuv,
                           const double* __restrict__ xvv, long N, int ng, double* __restrict__ geo) {
  FOR_POINTS(N)
  const long b = v * 3 * ng + k;
  double au[3], av[3], auu[3], auv[3], avv[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    au[c] = xu[b + c * ng];
    av[c] = xv[b + c * ng];
    auu[c] = xuu[b + c * ng];
    auv[c] = xuv[b + c * ng];
    avv[c] = xvv[b + c * ng];
  }
  const double E = au[0] * au[0] + au[1] * au[1] + au[2] * au[2];
  const double F = au[0] * av[0] + au[1] * av[1] + au[2] * av[2];
  const double G = av[0] * av[0] + av[1] * av[1] + av[2] * av[2];
  const double W2 = E * G - F * F;
  const double W = sqrt(W2);
  const double En = E / W2, Fn = F / W2, Gn = G / W2;
  // the reference's normal x_theta x x_phi / W (outward); u here is -d/dtheta
  double n[3] = {(au[2] * av[1] - au[1] * av[2]) / W, (au[0] * av[2] - au[2] * av[0]) / W,
                 (au[1] * av[0] - au[0] * av[1]) / W};
  double L = 0, M = 0, Nn = 0;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    L += auu[c] * n[c];
    M += auv[c] * n[c];
    Nn += avv[c] * n[c];
  }
  const double H = 0.5 * (Gn * L + En * Nn) - Fn * M;
  const double K = (L * Nn - M * M) / W2;
  double* o = geo + v * kGeoComps * (long)ng + k;
  o[0 * ng] = En;
  o[1 * ng] = Fn;
  o[2 * ng] = Gn;
  o[3 * ng] = W;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    o[(4 + c) * ng] = n[c];
    o[(7 + c) * ng] = Gn * au[c] - Fn * av[c];   // cu
    o[(10 + c) * ng] = En * av[c] - Fn * au[c];  // cv
  }
  o[13 * ng] = H;
  o[14 * ng] = K;
}

// grad: out[v][c][k] = fu cu[c] + fv cv[c]   (fu, fv scalar fields [nv][ng])
__global__ void k_grad_combine(const double* __restrict__ fu, const double* __restrict__ fv,
                               const double* __restrict__ geo, long N, int ng, double* __restrict__ out, long geo_nv) {
  FOR_POINTS(N)
  const double* o = GEO_OF(v);
  const double a = fu[g], b = fv[g];
#pragma unroll
  for (int c = 0; c < 3; c++) out[v * 3 * ng + c * ng + k] = a * o[(7 + c) * ng] + b * o[(10 + c) * ng];
}

// div: out[g] = sum_c Fu[c] cu[c] + Fv[c] cv[c]   (Fu, Fv vector fields)
__global__ void k_div_combine(const double* __restrict__ Fu, const double* __restrict__ Fv,
                              const double* __restrict__ geo, long N, int ng, double scale,
                              double* __restrict__ out, long geo_nv) {
  FOR_POINTS(N)
  const double* o = GEO_OF(v);
  const long b = v * 3 * ng + k;
  double s = 0.0, t = 0.0;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    s += Fu[b + c * ng] * o[(7 + c) * ng];
    t += Fv[b + c * ng] * o[(10 + c) * ng];
  }
  out[g] = scale * (s + t);
}

// linearised mean curvature: 0.5 (G (x_uu.n) - 2 F (x_uv.n) + E (x_vv.n))
__global__ void k_linH_combine(const double* __restrict__ duu, const double* __restrict__ duv,
                               const double* __restrict__ dvv, const double* __restrict__ geo, long N, int ng,
                               double* __restrict__ out, long geo_nv) {
  FOR_POINTS(N)
  const double* o = GEO_OF(v);
  const long b = v * 3 * ng + k;
  double a = 0, m = 0, c2 = 0;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const double nc = o[(4 + c) * ng];
    a += duu[b + c * ng] * nc;
    m += duv[b + c * ng] * nc;
    c2 += dvv[b + c * ng] * nc;
  }
  out[g] = 0.5 * (o[2 * ng] * a - 2.0 * o[1 * ng] * m + o[0 * ng] * c2);
}

// bending traction from h and its Laplace-Beltrami lap: -kappa (lap + 2 h (H^2 - K)) n
// (InterfacialForce::bendingForce scaled by bending_coeff = -bending_modulus,
// src/VesicleProps.cc:39-41; restoring with the outward normal), written to out
// (AxisMajor vector) with out = add + that if add is given; kappa is the bending modulus.
__global__ void k_bend_combine(const double* __restrict__ h, const double* __restrict__ lap,
                               const double* __restrict__ geo, long N, int ng, double kappa,
                               const double* __restrict__ add, double* __restrict__ out, long geo_nv) {
  FOR_POINTS(N)
  const double* o = GEO_OF(v);
  const double H = o[13 * ng], K = o[14 * ng];
  const double s = -kappa * (lap[g] + 2.0 * h[g] * (H * H - K));
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const long i = v * 3 * ng + c * ng + k;
    out[i] = (add ? add[i] : 0.0) + s * o[(4 + c) * ng];
  }
}

// tension traction: 2 sigma H n + grad sigma (grad given as a vector field), added to add
__global__ void k_tension_combine(const double* __restrict__ sigma, const double* __restrict__ gsig,
                                  const double* __restrict__ geo, long N, int ng, const double* __restrict__ add,
                                  double* __restrict__ out, long geo_nv) {
  FOR_POINTS(N)
  const double* o = GEO_OF(v);
  const double s = 2.0 * sigma[g] * o[13 * ng];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const long i = v * 3 * ng + c * ng + k;
    out[i] = (add ? add[i] : 0.0) + s * o[(4 + c) * ng] + gsig[i];
  }
}

// gravity traction: excess_density (g . x) n for a vector field x, added to add
// (InterfacialForce::gravityForce, src/InterfacialForce.cc:127-160)
__global__ void k_gravity_combine(const double* __restrict__ x, const double* __restrict__ geo, long N, int ng,
                                  double drho, double gx, double gy, double gz, const double* __restrict__ add,
                                  double* __restrict__ out, long geo_nv) {
  FOR_POINTS(N)
  const double* o = GEO_OF(v);
  const long b = v * 3 * ng + k;
  const double s = drho * (gx * x[b] + gy * x[b + ng] + gz * x[b + 2 * ng]);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const long i = b + c * ng;
    out[i] = (add ? add[i] : 0.0) + s * o[(4 + c) * ng];
  }
}

// u = (rate * y, 0, 0) on AxisMajor positions
__global__ void k_shear(const double* __restrict__ X, long N, int ng, double rate, double* __restrict__ out) {
  FOR_POINTS(N)
  const long b = v * 3 * ng + k;
  out[b] = rate * X[b + ng];
  out[b + ng] = 0.0;
  out[b + 2 * ng] = 0.0;
}

#undef FOR_POINTS

// Per vesicle (one CTA each): area = sum W q, volume = sum (x.n)/3 W q, centre =
// sum (|x|^2/2) n W q / volume, with W n = x_u x x_v and the Gauss-Legendre surface
// weights q (Surface::area / volume / getCenters, src/Surface.cc:378-440;
// GaussLegendreIntegrator, src/GLIntegrator.cc:33-80). out[v] = {area, volume, cx, cy, cz}.
// Fixed-order block reduction: the result is bitwise reproducible.
__global__ void __launch_bounds__(256) k_integrals(const double* __restrict__ X, const double* __restrict__ Xu,
                                                   const double* __restrict__ Xv, const double* __restrict__ w,
                                                   int p, double* __restrict__ out) {
  __shared__ double red[5][8];
  const int ng = 2 * p * (p + 1);
  const long v = blockIdx.x;
  const long b = v * 3 * ng;
  double acc[5] = {0, 0, 0, 0, 0};
  for (int k = threadIdx.x; k < ng; k += blockDim.x) {
    double x[3], a[3], c[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      x[d] = X[b + d * ng + k];
      a[d] = Xu[b + d * ng + k];
      c[d] = Xv[b + d * ng + k];
    }
    // W n with the outward normal of Surface::updateFirstForms (u here is -d/dtheta)
    const double nx = a[2] * c[1] - a[1] * c[2], ny = a[0] * c[2] - a[2] * c[0], nz = a[1] * c[0] - a[0] * c[1];
    const double q = w[k / (2 * p)];
    const double W = sqrt(nx * nx + ny * ny + nz * nz);
    const double h = 0.5 * (x[0] * x[0] + x[1] * x[1] + x[2] * x[2]) * q;
    acc[0] += W * q;
    acc[1] += (x[0] * nx + x[1] * ny + x[2] * nz) * (q / 3.0);
    acc[2] += h * nx;
    acc[3] += h * ny;
    acc[4] += h * nz;
  }
#pragma unroll
  for (int i = 0; i < 5; i++) {
    double t = acc[i];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) red[i][threadIdx.x >> 5] = t;
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    double t = 0;
    for (int w8 = 0; w8 < (int)(blockDim.x >> 5); w8++) t += red[threadIdx.x][w8];
    red[threadIdx.x][0] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double vol = red[1][0];
    out[v * 5] = red[0][0];
    out[v * 5 + 1] = vol;
    out[v * 5 + 2] = red[2][0] / vol;
    out[v * 5 + 3] = red[3][0] / vol;
    out[v * 5 + 4] = red[4][0] / vol;
  }
}

static inline unsigned nblk(long n) { return (unsigned)((n + 255) / 256); }

int launch_geometry(const double* xu, const double* xv, const double* xuu, const double* xuv, const double* xvv,
                    long nv, int ng, double* geo, cudaStream_t st) {
  const long N = nv * ng;
  if (N <= 0) return VES3D_OK;
  k_geometry<<<nblk(N), 256, 0, st>>>(xu, xv, xuu, xuv, xvv, N, ng, geo);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

int launch_grad_combine(const double* fu, const double* fv, const double* geo, long nv, int ng, double* out,
                        cudaStream_t st, long geo_nv) {
  const long N = nv * ng;
  if (N <= 0) return VES3D_OK;
  k_grad_combine<<<nblk(N), 256, 0, st>>>(fu, fv, geo, N, ng, out, geo_nv > 0 ? geo_nv : nv);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

int launch_div_combine(const double* Fu, const double* Fv, const double* geo, long nv, int ng, double scale,
                       double* out, cudaStream_t st, long geo_nv) {
  const long N = nv * ng;
  if (N <= 0) return VES3D_OK;
  k_div_combine<<<nblk(N), 256, 0, st>>>(Fu, Fv, geo, N, ng, scale, out, geo_nv > 0 ? geo_nv : nv);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

int launch_linH_combine(const double* duu, const double* duv, const double* dvv, const double* geo, long nv, int ng,
                        double* out, cudaStream_t st, long geo_nv) {
  const long N = nv * ng;
  if (N <= 0) return VES3D_OK;
  k_linH_combine<<<nblk(N), 256, 0, st>>>(duu, duv, dvv, geo, N, ng, out, geo_nv > 0 ? geo_nv : nv);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

int launch_bend_combine(const double* h, const double* lap, const double* geo, long nv, int ng, double kappa,
                        const double* add, double* out, cudaStream_t st, long geo_nv) {
  const long N = nv * ng;
  if (N <= 0) return VES3D_OK;
  k_bend_combine<<<nblk(N), 256, 0, st>>>(h, lap, geo, N, ng, kappa, add, out, geo_nv > 0 ? geo_nv : nv);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

int launch_tension_combine(const double* sigma, const double* gsig, const double* geo, long nv, int ng,
                           const double* add, double* out, cudaStream_t st, long geo_nv) {
  const long N = nv * ng;
  if (N <= 0) return VES3D_OK;
  k_tension_combine<<<nblk(N), 256, 0, st>>>(sigma, gsig, geo, N, ng, add, out, geo_nv > 0 ? geo_nv : nv);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

int launch_integrals(const double* X, const double* Xu, const double* Xv, const double* w, long nv, int p,
                     double* out, cudaStream_t st) {
  if (nv <= 0) return VES3D_OK;
  k_integrals<<<(unsigned)nv, 256, 0, st>>>(X, Xu, Xv, w, p, out);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

int launch_gravity_combine(const double* x, const double* geo, long nv, int ng, double drho, const double* g,
                           const double* add, double* out, cudaStream_t st, long geo_nv) {
  const long N = nv * ng;
  if (N <= 0) return VES3D_OK;
  k_gravity_combine<<<nblk(N), 256, 0, st>>>(x, geo, N, ng, drho, g[0], g[1], g[2], add, out,
                                             geo_nv > 0 ? geo_nv : nv);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

int launch_shear(const double* X, long nv, int ng, double rate, double* out, cudaStream_t st) {
  const long N = nv * ng;
  if (N <= 0) return VES3D_OK;
  k_shear<<<nblk(N), 256, 0, st>>>(X, N, ng, rate, out);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

}  // namespace ves3d
