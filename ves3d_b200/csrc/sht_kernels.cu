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
#include <cstdlib>

#include <algorithm>

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

// Functions per CTA: as many as 96 KB of shared memory holds (at most 8), but no more
// than keeps two CTAs per SM busy -- small batches (one vesicle's worth of functions in
// an operator assembly) are otherwise latency-bound on a handful of CTAs.
static int pick_fpb(size_t per_fun_doubles, long nfun) {
  size_t budget = 96 * 1024 / sizeof(double);
  int fpb = (int)(budget / per_fun_doubles);
  if (fpb < 1) fpb = 1;
  if (fpb > 8) fpb = 8;
  const long fill = nfun / (2 * 148);
  if (fill < fpb) fpb = (int)(fill < 1 ? 1 : fill);
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

namespace ves3d {

__device__ __forceinline__ void dmma_a(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

constexpr int pad4m16(int n) { return ((n + 11) / 16) * 16 + 4; }

// Grid2SHC(p, p) on FP64 tensor cores: 4 functions per CTA. The length-2p DFT of every
// (function, latitude) row is one GEMM [rows x 2p] . MatFourierInv(p, p) with
// mma.sync m8n8k4 (fragments as in build_kernels.cu); the per-frequency Legendre sums
// run on the CUDA cores from shared memory. Needs 2p % 8 == 0.
template <int P>
struct AnaTcCfg {
  static constexpr int FB = 4;
  static constexpr int NLAT = P + 1, NLON = 2 * P, NC = P * (P + 2);
  static constexpr int ROWS = ((FB * NLAT + 7) / 8) * 8;
  static constexpr int LD = pad4m16(NLON);
  static constexpr int OFF_A = 0, OFF_F = ROWS * LD, OFF_M = 2 * ROWS * LD, OFF_L = OFF_M + NLON * LD;
  static constexpr int OFF_JF = OFF_L + NC * NLAT;  // jf [NC] (int)
  static constexpr int TOTAL = OFF_JF + (NC + 1) / 2;
  static constexpr size_t SMEM = (size_t)TOTAL * sizeof(double);
};

// Persistent CTAs: the DFT and Legendre tables are staged once per CTA, which then walks
// groups of FB functions (grid-stride). Per group: rows (function, latitude) x 2p DFT on
// the tensor cores, then per-frequency Legendre sums on the CUDA cores.
template <int P, typename InT>
__global__ void __launch_bounds__(256, 2) k_analysis_tc(const InT* __restrict__ in, long nfun,
                                                        const double* __restrict__ four, const double* __restrict__ leg,
                                                        const int* __restrict__ jf, double* __restrict__ out) {
  using G = AnaTcCfg<P>;
  extern __shared__ __align__(16) double sm[];
  double* sA = sm + G::OFF_A;
  double* sF = sm + G::OFF_F;
  double* sM = sm + G::OFF_M;
  double* sL = sm + G::OFF_L;
  int* sJf = reinterpret_cast<int*>(sm + G::OFF_JF);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < G::NLON * G::NLON; i += 256) {
    const int r = i / G::NLON, j = i - r * G::NLON;
    sM[r * G::LD + j] = __ldg(four + i);
  }
  for (int i = tid; i < G::NC * G::NLAT; i += 256) sL[i] = __ldg(leg + i);
  for (int i = tid; i < G::NC; i += 256) sJf[i] = __ldg(jf + i);
  const int grow = lane >> 2, gcol = lane & 3;
  constexpr int MT = G::ROWS / 8, NT = G::NLON / 8;
  const long ngroups = (nfun + G::FB - 1) / G::FB;
  // software pipeline: the next group's grid values are loaded into registers while the
  // current group goes through the DFT and Legendre phases (the kernel was bound by the
  // latency of these loads: shared memory allows two CTAs per SM)
  constexpr int U = (G::ROWS * G::NLON + 255) / 256;
  double pre[U];
  auto load_group = [&](long g) {
    const long f0 = g * G::FB;
    const int nf = g < ngroups ? (int)min((long)G::FB, nfun - f0) : 0;
    const InT* src = in + (nf ? f0 : 0) * G::NLAT * G::NLON;  // no loads past the last group
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int i = tid + u * 256;
      pre[u] = (i < G::ROWS * G::NLON && i / G::NLON < nf * G::NLAT) ? (double)src[i] : 0.0;
    }
  };
  load_group(blockIdx.x);
  for (long grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    const long f0 = grp * G::FB;
    const int nf = (int)min((long)G::FB, nfun - f0);
    __syncthreads();  // the previous group's sA / sF reads are done
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int i = tid + u * 256;
      if (i < G::ROWS * G::NLON) {
        const int r = i / G::NLON, j = i - r * G::NLON;
        sA[r * G::LD + j] = pre[u];
      }
    }
    __syncthreads();
    load_group(grp + gridDim.x);
    for (int it = warp; it < MT * NT; it += 8) {
      const int nt = it % NT, mt = it / NT;
      const double* a = sA + (mt * 8 + grow) * G::LD + gcol;
      const double* b = sM + gcol * G::LD + nt * 8 + grow;  // B[k][n] = four[k][n]
      double c0 = 0, c1 = 0, d0 = 0, d1 = 0;
#pragma unroll
      for (int ks = 0; ks < G::NLON / 4; ks += 2) {
        dmma_a(c0, c1, a[ks * 4], b[ks * 4 * G::LD]);
        if (ks + 1 < G::NLON / 4) dmma_a(d0, d1, a[ks * 4 + 4], b[(ks * 4 + 4) * G::LD]);
      }
      double* o = sF + (mt * 8 + grow) * G::LD + nt * 8 + 2 * gcol;
      o[0] = c0 + d0;
      o[1] = c1 + d1;
    }
    __syncthreads();
    for (int i = tid; i < nf * G::NC; i += 256) {
      const int f = i / G::NC, c = i - f * G::NC;
      const int k = sJf[c];
      const double* fr = sF + (f * G::NLAT) * G::LD + k;
      const double* lr = sL + c * G::NLAT;
      double s = 0.0;
#pragma unroll
      for (int lat = 0; lat < G::NLAT; lat++) s = fma(fr[lat * G::LD], lr[lat], s);
      out[(f0 + f) * G::NC + c] = s;
    }
  }
}

// shc_out[f][c] = shc_in[f][c] scale[c] (in place allowed): SHTrans::ScaleFreq on
// function-major coefficient arrays
__global__ void k_scale_freq(const double* in, long n, int nc, const double* __restrict__ scale, double* out) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = in[i] * __ldg(scale + i % nc);
}

int launch_scale_freq(const double* in, long nfun, int nc, const double* scale, double* out, cudaStream_t st) {
  const long n = nfun * nc;
  if (n <= 0) return VES3D_OK;
  const long b = std::min((n + 255) / 256, 4096L);
  k_scale_freq<<<(unsigned)b, 256, 0, st>>>(in, n, nc, scale, out);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

// SHC2Pole (src/SphericalHarmonics.cc:325-360): the values of every function at x = -1
// and x = +1 from its m = 0 block, P[2f + t] = sum_n S[f][n] qp[t][n], summed in degree order
// like the reference. One thread per function; the data is n_fun (p0 + 1) doubles, so the
// strided reads cost nothing next to the transforms around it.
__global__ void k_shc2pole(const double* __restrict__ S, long nfun, int nc, int p0, const double* __restrict__ qp,
                           double* __restrict__ P) {
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < nfun; f += (long)gridDim.x * blockDim.x) {
    const double* s = S + f * nc;
    double a = 0.0, b = 0.0;
    for (int n = 0; n <= p0; n++) {
      const double c = s[n];
      a += c * qp[n];
      b += c * qp[p0 + 1 + n];
    }
    P[2 * f] = a;
    P[2 * f + 1] = b;
  }
}

int launch_shc2pole(const double* S, long nfun, int p0, const double* qp, double* P, cudaStream_t st) {
  if (nfun <= 0) return VES3D_OK;
  const long b = std::min((nfun + 255) / 256, 4096L);
  k_shc2pole<<<(unsigned)b, 256, 0, st>>>(S, nfun, p0 * (p0 + 2), p0, qp, P);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

static int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// Grid2SHC(p, p) of FP32 grid values in FP32 on the CUDA cores (the mixed form's
// self-matrix grid, whose values carry FP32 precision): persistent CTAs of NC = p (p + 2)
// threads stage the DFT table (FP32) once, each thread keeps the Legendre row of its
// coefficient in registers, and the CTA walks groups of FB functions. Per group the
// length-2p DFT of every (function, latitude) row, one thread per 4 rows x 4 frequencies
// (16 accumulators: row values broadcast across a warp's frequency quads, conflict-free
// table rows; one pass: RQ x KQ <= NC), then the Legendre sums of every function of the
// group at the thread's coefficient (the DFT rows of its Fourier block, broadcast to the
// block's coefficients); the next group's grid values are loaded into registers meanwhile.
// Output FP64 like the FP64 forms'.
template <int P>
struct AnaF32Cfg {
  static constexpr int FB = 8;
  static constexpr int NLAT = P + 1, NLON = 2 * P, NC = P * (P + 2), NT = (NC + 31) / 32 * 32;
  static constexpr int MINB = P == 16 ? 3 : 1;  // CTAs per SM the registers are sized for
  static constexpr int ROWS = FB * NLAT, RQ = (ROWS + 3) / 4, KQ = NLON / 4;
  static constexpr int LDG = NLON + 1;  // grid rows (odd: a warp's 4 row quads on distinct banks)
  static constexpr int LDF = NLON + 1;  // DFT result rows
  static constexpr int SZ_G = RQ * 4 * LDG, SZ_F = ROWS * LDF;
  static constexpr int OFF_G = 0, OFF_F = OFF_G + SZ_G, OFF_M = OFF_F + SZ_F;
  static constexpr size_t SMEM = (size_t)(OFF_M + NLON * NLON) * sizeof(float);
  static constexpr int U = (ROWS * NLON + NT - 1) / NT;  // grid values per thread per group
  static_assert(NLON % 4 == 0 && NT % 32 == 0 && RQ * KQ <= NT, "frequency quads; whole warps; one DFT pass");
};

template <int P>
__global__ void __launch_bounds__(AnaF32Cfg<P>::NT, AnaF32Cfg<P>::MINB) k_analysis_f32(const float* __restrict__ in, long nfun,
                                                                       const double* __restrict__ four,
                                                                       const double* __restrict__ leg,
                                                                       const int* __restrict__ jf,
                                                                       double* __restrict__ out) {
  using G = AnaF32Cfg<P>;
  constexpr int NT = G::NT;
  extern __shared__ __align__(16) float smf[];
  float* sG = smf + G::OFF_G;
  float* sF = smf + G::OFF_F;
  float* sM = smf + G::OFF_M;  // four [j][k], row stride NLON (float4 reads of 4 frequencies)
  const int tid = threadIdx.x;
  for (int i = tid; i < G::NLON * G::NLON; i += NT) sM[i] = (float)__ldg(four + i);
  // rows past the group's last function stay zero (their outputs are never written)
  for (int i = tid; i < G::SZ_G; i += NT) sG[i] = 0.f;
  // this thread's coefficient c = tid (threads past NC have none): its Fourier block and
  // Legendre row
  const bool has_c = tid < G::NC;
  const int jfc = has_c ? __ldg(jf + tid) : 0;
  float lr[G::NLAT];
#pragma unroll
  for (int lat = 0; lat < G::NLAT; lat++) lr[lat] = has_c ? (float)__ldg(leg + tid * G::NLAT + lat) : 0.f;
  const long ngroups = (nfun + G::FB - 1) / G::FB;
  float pre[G::U];
  auto load_group = [&](long g) {
    const long f0 = g * G::FB;
    const int nf = g < ngroups ? (int)min((long)G::FB, nfun - f0) : 0;
    const float* src = in + (nf ? f0 : 0) * G::NLAT * G::NLON;
#pragma unroll
    for (int u = 0; u < G::U; u++) {
      const int i = tid + u * NT;
      pre[u] = (i < nf * G::NLAT * G::NLON) ? src[i] : 0.f;
    }
  };
  load_group(blockIdx.x);
  for (long grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    const long f0 = grp * G::FB;
    const int nf = (int)min((long)G::FB, nfun - f0);
    __syncthreads();  // the previous group's sG / sF reads are done
#pragma unroll
    for (int u = 0; u < G::U; u++) {
      const int i = tid + u * NT;
      if (i < G::ROWS * G::NLON) {
        const int r = i / G::NLON, j = i - r * G::NLON;
        sG[r * G::LDG + j] = pre[u];
      }
    }
    __syncthreads();
    load_group(grp + gridDim.x);
    // DFT: F[r][k] = sum_j G[r][j] four[j][k]
    if (tid < G::RQ * G::KQ) {
      const int kq = tid % G::KQ, rq = tid / G::KQ;
      const float* g = sG + rq * 4 * G::LDG;
      const float4* m = reinterpret_cast<const float4*>(sM) + kq;
      float acc[4][4] = {};
#pragma unroll 8
      for (int j = 0; j < G::NLON; j++) {
        const float4 b = m[j * G::KQ];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const float a = g[q * G::LDG + j];
          acc[q][0] = fmaf(a, b.x, acc[q][0]);
          acc[q][1] = fmaf(a, b.y, acc[q][1]);
          acc[q][2] = fmaf(a, b.z, acc[q][2]);
          acc[q][3] = fmaf(a, b.w, acc[q][3]);
        }
      }
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int r = rq * 4 + q;
        if (r < G::ROWS) {
          float* o = sF + r * G::LDF + kq * 4;
          o[0] = acc[q][0];
          o[1] = acc[q][1];
          o[2] = acc[q][2];
          o[3] = acc[q][3];
        }
      }
    }
    __syncthreads();
    // Legendre: out[f][c] = sum_lat F[f][lat][jf(c)] leg[c][lat], c = tid
    for (int f = 0; f < (has_c ? nf : 0); f++) {
      const float* fr = sF + (f * G::NLAT) * G::LDF + jfc;
      float s = 0.f;
#pragma unroll
      for (int lat = 0; lat < G::NLAT; lat++) s = fmaf(fr[lat * G::LDF], lr[lat], s);
      out[(f0 + f) * G::NC + tid] = (double)s;
    }
  }
}

template <int P>
static int launch_ana_f32(const float* in, long nfun, const double* four, const double* leg, const int* jf,
                          double* out, cudaStream_t st) {
  using G = AnaF32Cfg<P>;
  VES3D_CK(cudaFuncSetAttribute(k_analysis_f32<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM));
  int per_sm = 0;
  VES3D_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_analysis_f32<P>, G::NT, G::SMEM));
  const long ngroups = (nfun + G::FB - 1) / G::FB;
  const long grid = std::min(ngroups, (long)std::max(per_sm, 1) * sm_count());
  k_analysis_f32<P><<<(unsigned)grid, G::NT, G::SMEM, st>>>(in, nfun, four, leg, jf, out);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

template <int P, typename InT>
static int launch_ana_tc(const InT* in, long nfun, const double* four, const double* leg, const int* jf,
                         double* out, cudaStream_t st) {
  using G = AnaTcCfg<P>;
  VES3D_CK(cudaFuncSetAttribute(k_analysis_tc<P, InT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM));
  const long ngroups = (nfun + G::FB - 1) / G::FB;
  const long grid = std::min(ngroups, 2L * sm_count());
  k_analysis_tc<P, InT><<<(unsigned)grid, 256, G::SMEM, st>>>(in, nfun, four, leg, jf, out);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

// Grid2SHC(p, p) with the tensor-core kernel where it is instantiated, else the generic one.
int launch_grid2shc(const double* in, long nfun, int p, const double* four, const double* leg, const int* jf,
                    double* out, cudaStream_t st) {
  if (nfun <= 0) return VES3D_OK;
  const char* env = getenv("VES3D_TC_ANALYSIS");
  const bool tc = !(env && env[0] == '0');
  if (tc) {
    switch (p) {
      case 4: return launch_ana_tc<4>(in, nfun, four, leg, jf, out, st);
      case 8: return launch_ana_tc<8>(in, nfun, four, leg, jf, out, st);
      case 12: return launch_ana_tc<12>(in, nfun, four, leg, jf, out, st);
      case 16: return launch_ana_tc<16>(in, nfun, four, leg, jf, out, st);
      default: break;
    }
  }
  return launch_analysis(in, nfun, p, p, four, leg, jf, out, st);
}

// Grid2SHC(p, p) of FP32 grid values, p in {4, 8, 12, 16}: FP32 arithmetic on the CUDA
// cores at p = 16 (the mixed self-matrix grid), FP64 DMMA from the FP32 values otherwise;
// FP64 output.
int launch_grid2shc_f32(const float* in, long nfun, int p, const double* four, const double* leg, const int* jf,
                        double* out, cudaStream_t st) {
  if (nfun <= 0) return VES3D_OK;
  switch (p) {
    case 4: return launch_ana_tc<4>(in, nfun, four, leg, jf, out, st);
    case 8: return launch_ana_tc<8>(in, nfun, four, leg, jf, out, st);
    case 12: return launch_ana_f32<12>(in, nfun, four, leg, jf, out, st);
    case 16: return launch_ana_f32<16>(in, nfun, four, leg, jf, out, st);
    case 24: return launch_ana_f32<24>(in, nfun, four, leg, jf, out, st);
    default: break;
  }
  set_error("Grid2SHC of FP32 values is instantiated for p in {4, 8, 12, 16, 24}, not %d", p);
  return VES3D_ERR_ARG;
}

}  // namespace ves3d
