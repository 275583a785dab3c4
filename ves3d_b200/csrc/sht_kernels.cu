// FP64 spherical-harmonic transform kernels (plain form).
//
// Analysis-like map (Grid2SHC, src/SphericalHarmonics.cc:152-235, and
// SHC2GridTranspose, :238-322): for each function on an (nlat x nlon) grid
//     F[lat][k]  = sum_j  X[lat][j] * four[j][k]          (length-nlon DFT as a GEMM)
//     S[c]       = sum_lat F[lat][jf(c)] * leg[c][lat]     (per-frequency Legendre GEMMs)
// Synthesis map (SHC2Grid, :4-149): for each coefficient vector
//     B[lat][jf] = sum_{c in block jf} S[c] * leg[c][lat]
//     X[lat][j]  = sum_jf B[lat][jf] * four[jf][j]   (X_theta with dfour, X_phi from dleg)
// One CTA transforms FPB functions with every intermediate in shared memory; the
// tables are small and read through the read-only cache.
#include "common.cuh"
#include "kernels.h"

namespace ves3d {

__global__ void __launch_bounds__(256) k_analysis(const double* __restrict__ in, long nfun, int nlat, int nlon,
                                                  int nfo, const double* __restrict__ four,
                                                  const double* __restrict__ leg, const int* __restrict__ jf,
                                                  int nco, int fpb, double* __restrict__ out) {
  extern __shared__ double sm[];
  double* sx = sm;
  double* sf = sm + (size_t)fpb * nlat * nlon;
  const long f0 = (long)blockIdx.x * fpb;
  const int nf = (int)min((long)fpb, nfun - f0);
  const int tot = nf * nlat * nlon;
  const double* src = in + f0 * nlat * nlon;
  for (int i = threadIdx.x; i < tot; i += blockDim.x) sx[i] = src[i];
  __syncthreads();
  const int totF = nf * nlat * nfo;
  for (int i = threadIdx.x; i < totF; i += blockDim.x) {
    const int k = i % nfo;
    const double* xr = sx + (i / nfo) * nlon;
    double s = 0.0;
#pragma unroll 4
    for (int j = 0; j < nlon; j++) s = fma(xr[j], __ldg(four + j * nfo + k), s);
    sf[i] = s;
  }
  __syncthreads();
  const int totC = nf * nco;
  for (int i = threadIdx.x; i < totC; i += blockDim.x) {
    const int c = i % nco, f = i / nco;
    const double* fr = sf + (size_t)f * nlat * nfo + __ldg(jf + c);
    const double* lr = leg + (size_t)c * nlat;
    double s = 0.0;
    for (int lat = 0; lat < nlat; lat++) s = fma(fr[lat * nfo], __ldg(lr + lat), s);
    out[(f0 + f) * nco + c] = s;
  }
}

__global__ void __launch_bounds__(256) k_synthesis(const double* __restrict__ S, long nfun, int nci, int nfi,
                                                   int nlat, int nlon, const double* __restrict__ leg,
                                                   const double* __restrict__ dleg,
                                                   const double* __restrict__ four,
                                                   const double* __restrict__ dfour,
                                                   const int* __restrict__ blk_off, int fpb,
                                                   double* __restrict__ X, double* __restrict__ Xt,
                                                   double* __restrict__ Xp) {
  extern __shared__ double sm[];
  double* ss = sm;                                  // fpb * nci
  double* sb = ss + (size_t)fpb * nci;              // fpb * nlat * nfi
  double* sd = sb + (size_t)fpb * nlat * nfi;       // fpb * nlat * nfi (if Xp)
  const long f0 = (long)blockIdx.x * fpb;
  const int nf = (int)min((long)fpb, nfun - f0);
  for (int i = threadIdx.x; i < nf * nci; i += blockDim.x) ss[i] = S[f0 * nci + i];
  __syncthreads();
  const int totB = nf * nlat * nfi;
  for (int i = threadIdx.x; i < totB; i += blockDim.x) {
    const int k = i % nfi, lat = (i / nfi) % nlat, f = i / (nfi * nlat);
    const int c0 = __ldg(blk_off + k), c1 = __ldg(blk_off + k + 1);
    const double* sr = ss + (size_t)f * nci;
    double s = 0.0, d = 0.0;
    for (int c = c0; c < c1; c++) {
      s = fma(sr[c], __ldg(leg + (size_t)c * nlat + lat), s);
      if (Xp) d = fma(sr[c], __ldg(dleg + (size_t)c * nlat + lat), d);
    }
    sb[i] = s;
    if (Xp) sd[i] = d;
  }
  __syncthreads();
  const int totX = nf * nlat * nlon;
  for (int i = threadIdx.x; i < totX; i += blockDim.x) {
    const int j = i % nlon, r = i / nlon;  // r = f*nlat + lat
    const double* br = sb + (size_t)r * nfi;
    double x = 0.0, xt = 0.0;
#pragma unroll 4
    for (int k = 0; k < nfi; k++) {
      x = fma(br[k], __ldg(four + k * nlon + j), x);
      if (Xt) xt = fma(br[k], __ldg(dfour + k * nlon + j), xt);
    }
    X[f0 * nlat * nlon + i] = x;
    if (Xt) Xt[f0 * nlat * nlon + i] = xt;
    if (Xp) {
      const double* dr = sd + (size_t)r * nfi;
      double xp = 0.0;
#pragma unroll 4
      for (int k = 0; k < nfi; k++) xp = fma(dr[k], __ldg(four + k * nlon + j), xp);
      Xp[f0 * nlat * nlon + i] = xp;
    }
  }
}

static int pick_fpb(size_t per_fun_doubles, long nfun) {
  size_t budget = 96 * 1024 / sizeof(double);
  int fpb = (int)(budget / per_fun_doubles);
  if (fpb < 1) fpb = 1;
  if (fpb > 8) fpb = 8;
  if (fpb > nfun) fpb = (int)nfun;
  return fpb;
}

int launch_analysis(const double* in, long nfun, int pin, int pout, const double* four, const double* leg,
                    const int* jf, double* out, cudaStream_t st) {
  if (nfun <= 0) return VES3D_OK;
  const int nlat = pin + 1, nlon = 2 * pin, nfo = 2 * pout, nco = ncoef_(pout);
  const int fpb = pick_fpb((size_t)nlat * (nlon + nfo), nfun);
  size_t smem = (size_t)fpb * nlat * (nlon + nfo) * sizeof(double);
  if (smem > 48 * 1024) VES3D_CK(cudaFuncSetAttribute(k_analysis, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  long nblk = (nfun + fpb - 1) / fpb;
  k_analysis<<<(unsigned)nblk, 256, smem, st>>>(in, nfun, nlat, nlon, nfo, four, leg, jf, nco, fpb, out);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

int launch_synthesis(const double* S, long nfun, int p0, int q, const double* leg, const double* dleg,
                     const double* four, const double* dfour, const int* blk_off, double* X, double* Xt,
                     double* Xp, cudaStream_t st) {
  if (nfun <= 0) return VES3D_OK;
  const int nci = ncoef_(p0), nfi = 2 * p0, nlat = q + 1, nlon = 2 * q;
  const size_t per = (size_t)nci + (size_t)nlat * nfi * (Xp ? 2 : 1);
  const int fpb = pick_fpb(per, nfun);
  size_t smem = (size_t)fpb * per * sizeof(double);
  if (smem > 48 * 1024) VES3D_CK(cudaFuncSetAttribute(k_synthesis, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  long nblk = (nfun + fpb - 1) / fpb;
  k_synthesis<<<(unsigned)nblk, 256, smem, st>>>(S, nfun, nci, nfi, nlat, nlon, leg, dleg, four, dfour, blk_off,
                                                  fpb, X, Xt, Xp);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

}  // namespace ves3d
