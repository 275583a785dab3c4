// Fused singular-quadrature kernel of the self-matrix build (FP64), one CTA per rotated
// surface (vesicle v, rotation (t, j)):
//
//   R (rotated coefficients, 3 x Nc)
//     -> Legendre synthesis at the p1 = 2 p0 nodes, values and theta-derivatives
//     -> DFT synthesis: X, X_theta, X_phi on the upsampled grid          [GEMM, K = 2p0]
//     -> pole targets and the singular Stokes kernel, 2 poles x 6 components
//     -> transposed DFT                                                  [GEMM, K = 2p1]
//     -> transposed Legendre sums, accumulated over latitude groups
//     -> C (2 x 6 x Nc): the kernel contracted back to order-p0 coefficients.
//
// This is SHC2Grid(p0 -> p1, grads) + the kernel loop + SHC2GridTranspose(p1 -> p0) of
// SphericalHarmonics<Real>::StokesSingularInteg_ (src/SphericalHarmonics.cc:963-1082)
// with every intermediate in shared memory (the unfused form writes 150 KB of upsampled
// surface and 200 KB of kernel values per rotation to HBM and reads them back).
//
// Both DFT GEMMs run on the FP64 tensor cores with mma.sync m8n8k4 (sm_100 has no FP64
// kind in tcgen05). Fragment layout (PTX ISA, m8n8k4 .f64): A: a0 = A[lane/4][lane%4];
// B: b0 = B[lane%4][lane/4]; C: {c0, c1} = C[lane/4][2(lane%4) + {0, 1}]. Shared-memory
// row strides are padded to 4 mod 16 doubles so those loads are bank-conflict free.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

#include "common.cuh"
#include "kernels.h"

namespace ves3d {

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// Row stride >= n with stride = 4 (mod 16) doubles.
__host__ __device__ constexpr int pad16_4(int n) { return ((n + 11) / 16) * 16 + 4; }

// Number of 8-wide n-tiles over the Fourier blocks of the order-p0 coefficient vector
// (block lengths p0+1, then p0+1-m twice for m = 1..p0-1, then 1).
__host__ __device__ constexpr int legt_ntiles(int p0) {
  int t = (p0 + 1 + 7) / 8 + 1;
  for (int m = 1; m < p0; m++) t += 2 * ((p0 + 1 - m + 7) / 8);
  return t;
}

template <int P0>
struct RingCfg {
  static constexpr int P1 = 2 * P0;
  static constexpr int NC = P0 * (P0 + 2);
  static constexpr int L1 = P1 + 1;           // latitudes of the upsampled grid
  static constexpr int F0 = 2 * P0;           // Fourier coefficients at order p0
  static constexpr int N1 = 2 * P1;           // longitudes of the upsampled grid
  static constexpr int LG = 4;                // latitudes per group (= K of one m8n8k4 step)
  static constexpr int NGRP = (L1 + LG - 1) / LG;
  static constexpr int ROWS1 = ((3 * LG + 7) / 8) * 8;   // (lat, d) rows of a group, m-tile padded
  static constexpr int LDA = pad16_4(F0);
  static constexpr int LDM = pad16_4(N1);
  static constexpr int LDX = pad16_4(N1);
  static constexpr int LDK = pad16_4(N1);
  // C rows (lat, component) read down a column by the transposed-Legendre MMAs: an odd
  // stride of F0 + 5 makes those fragment reads conflict-free
  static constexpr int LDC = F0 + 5;
  // coefficient rows (R, Legendre slices) padded to 4 mod 16 for the MMA fragments, with
  // room for the K padding of the last Fourier block
  static constexpr int LDR = pad16_4(NC + 3);
  static constexpr int NTT = legt_ntiles(P0);             // n-tiles of the transposed Legendre
  static constexpr int QMAX = (2 * NTT + 7) / 8;          // its accumulator tiles per warp
  // Shared memory, with buffers of disjoint lifetimes aliased:
  //   region Q: A/dA (Legendre synthesis -> G1)  then  K (kernel -> G2)
  //   region P: X/X_theta/X_phi (G1 -> kernel)   then  C (G2 -> Legendre sums)
  static constexpr int SZ_A = 2 * ROWS1 * LDA;
  static constexpr int SZ_K = (LG * 12) * LDK;
  static constexpr int SZ_X = 3 * ROWS1 * LDX;
  static constexpr int SZ_C = (LG * 12) * LDC;
  static constexpr int OFF_R = 0;
  static constexpr int OFF_MF = OFF_R + 3 * LDR;
  static constexpr int OFF_DMF = OFF_MF + F0 * LDM;
  static constexpr int OFF_LEG = OFF_DMF + F0 * LDM;       // [LG][LDR] slice of the latitude group
  static constexpr int OFF_DLEG = OFF_LEG + LG * LDR;
  static constexpr int OFF_Q = OFF_DLEG + LG * LDR;
  static constexpr int OFF_P = OFF_Q + (SZ_A > SZ_K ? SZ_A : SZ_K);
  static constexpr int OFF_TRG = OFF_P + (SZ_X > SZ_C ? SZ_X : SZ_C);
  // small index/weight tables read in every latitude group, kept on chip
  static constexpr int OFF_SW = OFF_TRG + 8;                    // sing_w [L1]
  static constexpr int OFF_BO = OFF_SW + L1;                    // blk_off [F0 + 1] (int)
  static constexpr int OFF_TL = OFF_BO + (F0 + 2) / 2;          // n-tile list: (block, tile) [NTT] (uchar2)
  static constexpr int TOTAL = OFF_TL + (NTT + 3) / 4;
  static constexpr size_t SMEM = (size_t)TOTAL * sizeof(double);
  static constexpr int NOUT = 12 * NC;
};

// Persistent: each CTA stages the DFT tables and the small index tables once, then walks
// rotations blockIdx.x, blockIdx.x + gridDim.x, ...
// Two CTAs per SM up to p = 16; at p = 24 the tables and stage buffers take ~208 KB of
// shared memory and one CTA fills the SM.
template <int P0>
__global__ void __launch_bounds__(256, (P0 <= 16 ? 2 : 1)) k_build_ring(const double* __restrict__ R, DevTables T,
                                                       double* __restrict__ C, long nrot) {
  using G = RingCfg<P0>;
  extern __shared__ __align__(16) double sm[];
  double* sR = sm + G::OFF_R;
  double* sMf = sm + G::OFF_MF;
  double* sdMf = sm + G::OFF_DMF;
  double* sLeg = sm + G::OFF_LEG;
  double* sdLeg = sm + G::OFF_DLEG;
  double* sA = sm + G::OFF_Q;
  double* sdA = sA + G::ROWS1 * G::LDA;
  double* sK = sm + G::OFF_Q;
  double* sX = sm + G::OFF_P;
  double* sC = sm + G::OFF_P;
  double* trg = sm + G::OFF_TRG;
  double* sSw = sm + G::OFF_SW;
  int* sBo = reinterpret_cast<int*>(sm + G::OFF_BO);
  uchar2* sTl = reinterpret_cast<uchar2*>(sm + G::OFF_TL);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < G::L1; i += 256) sSw[i] = __ldg(T.sing_w + i);
  for (int i = tid; i <= G::F0; i += 256) sBo[i] = __ldg(T.blk_off + i);
  if (tid == 0) {
    // n-tiles of the transposed Legendre: (Fourier block, 8-wide tile within it)
    int j = 0;
    for (int k = 0; k < G::F0; k++) {
      const int len = __ldg(T.blk_off + k + 1) - __ldg(T.blk_off + k);
      for (int nt = 0; nt * 8 < len && j < G::NTT; nt++) sTl[j++] = make_uchar2((unsigned char)k, (unsigned char)nt);
    }
  }

  // ---- DFT tables (once per CTA) ----------------------------------------------------------
  for (int i = tid; i < G::F0 * G::N1; i += 256) {
    const int k = i / G::N1, j = i - k * G::N1;
    sMf[k * G::LDM + j] = __ldg(T.syn1_four + i);
    sdMf[k * G::LDM + j] = __ldg(T.syn1_dfour + i);
  }
  for (long rot = blockIdx.x; rot < nrot; rot += gridDim.x) {
  // ---- rotated coefficients, pole targets ------------------------------------------------
  // rotated coefficients, rows padded to LDR (zeros beyond NC: K padding of the last block);
  // the previous rotation's last reads of sR ended at its final barrier
  for (int i = tid; i < 3 * G::LDR; i += 256) {
    const int d = i / G::LDR, c = i - d * G::LDR;
    sR[i] = c < G::NC ? R[rot * 3 * G::NC + d * G::NC + c] : 0.0;
  }
  __syncthreads();
  if (tid < 6) {
    const int c = tid >> 1, t = tid & 1;
    double s = 0.0;
    for (int n = 0; n <= P0; n++) s += sR[c * G::LDR + n] * __ldg(T.qp + t * (P0 + 1) + n);
    trg[c * 2 + t] = s;
  }
  // transposed-Legendre accumulators: tile warp + 8 q = (m-tile of components, n-tile)
  double acc[G::QMAX][2];
#pragma unroll
  for (int q = 0; q < G::QMAX; q++) acc[q][0] = acc[q][1] = 0.0;

  const int grow = lane >> 2, gcol = lane & 3;
  for (int g = 0; g < G::NGRP; g++) {
    const int lat0 = g * G::LG;
    const int nlat = min(G::LG, G::L1 - lat0);
    // ---- the group's slice of the Legendre tables -------------------------------------
    {
      constexpr int U = (G::LDR * G::LG + 255) / 256;  // loads in flight per thread
      double a[U], b[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = tid + u * 256;
        const int l = i / G::LDR, c = i - l * G::LDR;
        const bool ok = i < G::LDR * G::LG && l < nlat && c < G::NC;
        a[u] = ok ? __ldg(T.syn1_leg_t + (lat0 + l) * G::NC + c) : 0.0;
        b[u] = ok ? __ldg(T.syn1_dleg_t + (lat0 + l) * G::NC + c) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = tid + u * 256;
        if (i < G::LDR * G::LG) {
          sLeg[i] = a[u];
          sdLeg[i] = b[u];
        }
      }
    }
    __syncthreads();
    // ---- Legendre synthesis of the group's latitudes on tensor cores ------------------
    // per Fourier block k: A[(l, d)][k] = sum_{c in block k} Leg[l][c] R[d][c] (and dA with
    // the derivative table) is one m8n8k4 GEMM [lat x c] . [c x d], K = the block length;
    // K padding reads the next block's (finite) Legendre values against zeros in B
    for (int i = tid; i < (G::ROWS1 - 3 * nlat) * G::F0; i += 256) {
      const int row = 3 * nlat + i / G::F0, k = i % G::F0;
      sA[row * G::LDA + k] = 0.0;
      sdA[row * G::LDA + k] = 0.0;
    }
    for (int it = warp; it < 2 * G::F0; it += 8) {
      const int k = it >> 1, which = it & 1;
      const int c0 = sBo[k], c1 = sBo[k + 1];
      const double* L = (which ? sdLeg : sLeg) + grow * G::LDR + c0 + gcol;
      const double* Rr = sR + grow * G::LDR + c0 + gcol;
      double e0 = 0.0, e1 = 0.0;
      for (int ks = 0; 4 * ks < c1 - c0; ks++) {
        const int c = c0 + 4 * ks + gcol;
        const double a = grow < nlat ? L[4 * ks] : 0.0;
        const double b = (grow < 3 && c < c1) ? Rr[4 * ks] : 0.0;
        dmma(e0, e1, a, b);
      }
      // C[l = grow][d = 2 gcol + {0, 1}]
      double* out = which ? sdA : sA;
      const int d0 = 2 * gcol;
      if (grow < nlat) {
        if (d0 < 3) out[(grow * 3 + d0) * G::LDA + k] = e0;
        if (d0 + 1 < 3) out[(grow * 3 + d0 + 1) * G::LDA + k] = e1;
      }
    }
    __syncthreads();
    // ---- DFT synthesis on tensor cores: X, X_theta (from A), X_phi (from dA) ------------
    {
      const int mt_n = (3 * nlat + 7) / 8;
      const int nitems = mt_n * 3 * (G::N1 / 16);    // (m-tile, variant, pair of n-tiles)
      for (int it = warp; it < nitems; it += 8) {
        const int np2 = it % (G::N1 / 16);
        const int var = (it / (G::N1 / 16)) % 3;
        const int mt = it / (3 * (G::N1 / 16));
        const double* Asrc = (var == 2 ? sdA : sA) + (mt * 8 + grow) * G::LDA + gcol;
        const double* Bsrc = (var == 1 ? sdMf : sMf) + gcol * G::LDM + np2 * 16 + grow;
        double c00 = 0, c01 = 0, c10 = 0, c11 = 0;
#pragma unroll
        for (int ks = 0; ks < G::F0 / 4; ks++) {
          const double a = Asrc[ks * 4];
          dmma(c00, c01, a, Bsrc[ks * 4 * G::LDM]);
          dmma(c10, c11, a, Bsrc[ks * 4 * G::LDM + 8]);
        }
        double* out = sX + var * G::ROWS1 * G::LDX + (mt * 8 + grow) * G::LDX + np2 * 16 + 2 * gcol;
        out[0] = c00;
        out[1] = c01;
        out[8] = c10;
        out[9] = c11;
      }
    }
    __syncthreads();
    // ---- singular kernel at the group's upsampled points (K aliases A/dA) ---------------
    for (int pnt = tid; pnt < nlat * G::N1; pnt += 256) {
      const int l = pnt / G::N1, j = pnt - l * G::N1;
      const int lat = lat0 + l;
      const double* x = sX + (l * 3) * G::LDX + j;
      const double* xt = x + G::ROWS1 * G::LDX;
      const double* xp = xt + G::ROWS1 * G::LDX;
      const double px = x[0], py = x[G::LDX], pz = x[2 * G::LDX];
      const double ax = xt[0], ay = xt[G::LDX], az = xt[2 * G::LDX];
      const double bx = xp[0], by = xp[G::LDX], bz = xp[2 * G::LDX];
      const double nx = ay * bz - az * by, ny = az * bx - ax * bz, nz = ax * by - ay * bx;
      const double n2 = nx * nx + ny * ny + nz * nz;
      const double area = n2 * rsqrt_f64_int_seed(n2);  // |X_theta x X_phi| > 0 on the upsampled grid
#pragma unroll
      for (int t = 0; t < 2; t++) {
        const double dx = trg[t] - px, dy = trg[2 + t] - py, dz = trg[4 + t] - pz;
        const double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_f64_int_seed(r2);  // (r2 below 2^-126 is cut off here too)
        if (r2 <= 2.220446049250313e-16) rinv = 0.0;
        const double a1 = kInv8Pi * sSw[t ? lat : G::P1 - lat] * area * rinv;
        const double a2 = a1 * rinv * rinv;
        double* k = sK + (l * 12 + t * 6) * G::LDK + j;
        k[0] = a1 + dx * dx * a2;
        k[G::LDK] = dx * dy * a2;
        k[2 * G::LDK] = dx * dz * a2;
        k[3 * G::LDK] = a1 + dy * dy * a2;
        k[4 * G::LDK] = dy * dz * a2;
        k[5 * G::LDK] = a1 + dz * dz * a2;
      }
    }
    __syncthreads();
    // ---- transposed DFT on tensor cores: Cg[(l,q)][jf] = sum_j K[(l,q)][j] Mf[jf][j] -----
    {
      const int mt_n = (12 * nlat + 7) / 8;
      const int nitems = mt_n * (G::F0 / 8);
      for (int it = warp; it < nitems; it += 8) {
        const int nt = it % (G::F0 / 8), mt = it / (G::F0 / 8);
        const double* Asrc = sK + (mt * 8 + grow) * G::LDK + gcol;
        const double* Bsrc = sMf + (nt * 8 + grow) * G::LDM + gcol;  // B[j][jf] = Mf[jf][j]
        double c0 = 0, c1 = 0, d0 = 0, d1 = 0;
#pragma unroll
        for (int ks = 0; ks < G::N1 / 4; ks += 2) {
          dmma(c0, c1, Asrc[ks * 4], Bsrc[ks * 4]);
          dmma(d0, d1, Asrc[ks * 4 + 4], Bsrc[ks * 4 + 4]);
        }
        double* out = sC + (mt * 8 + grow) * G::LDC + nt * 8 + 2 * gcol;
        out[0] = c0 + d0;
        out[1] = c1 + d1;
      }
    }
    __syncthreads();
    // ---- transposed Legendre sums on tensor cores, accumulated over the groups ---------
    // Cout[comp][c] += sum_{l < LG} C[(l, comp)][k(c)] Leg[l][c]: per (m-tile of the 12
    // components, n-tile of a Fourier block) one m8n8k4 step with K = the LG latitudes
#pragma unroll
    for (int q = 0; q < G::QMAX; q++) {
      const int tile = warp + 8 * q;
      if (tile < 2 * G::NTT) {
        const int mt = tile / G::NTT;
        const uchar2 kt = sTl[tile - mt * G::NTT];
        const int k = kt.x, c0 = sBo[k], c1 = sBo[k + 1];
        const int comp = mt * 8 + grow, l = gcol, c = c0 + kt.y * 8 + grow;
        const double a = (comp < 12 && l < nlat) ? sC[(l * 12 + comp) * G::LDC + k] : 0.0;
        const double b = (l < nlat && c < c1) ? sLeg[l * G::LDR + c] : 0.0;
        dmma(acc[q][0], acc[q][1], a, b);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < G::QMAX; q++) {
    const int tile = warp + 8 * q;
    if (tile < 2 * G::NTT) {
      const int mt = tile / G::NTT;
      const uchar2 kt = sTl[tile - mt * G::NTT];
      const int c0 = sBo[kt.x], c1 = sBo[kt.x + 1];
      const int comp = mt * 8 + grow, c = c0 + kt.y * 8 + 2 * gcol;
      if (comp < 12) {
        if (c < c1) C[rot * G::NOUT + comp * G::NC + c] = acc[q][0];
        if (c + 1 < c1) C[rot * G::NOUT + comp * G::NC + c + 1] = acc[q][1];
      }
    }
  }
  }  // rotations
}

// Persistent CTAs per SM: 2 fill the shared memory (the default: 52.1 ms per build at 512
// vesicles, p = 16); 1 leaves room beside each for two far-field CTAs when the far field
// runs concurrently (VES3D_RING_CTAS=1 with VES3D_FAR_OVERLAP=1: 97.6 ms per evaluation
// step against 100.9 serial)
static int ring_ctas_per_sm() {
  static int n = 0;
  if (!n) {
    const char* e = getenv("VES3D_RING_CTAS");
    n = (e && (e[0] == '1' || e[0] == '2') && !e[1]) ? e[0] - '0' : 2;
  }
  return n;
}

template <int P0>
static int launch_ring(const double* R, long nrot, const DevTables& T, double* C, cudaStream_t st) {
  using G = RingCfg<P0>;
  VES3D_CK(cudaFuncSetAttribute(k_build_ring<P0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM));
  int dev = 0, nsm = 148;
  VES3D_CK(cudaGetDevice(&dev));
  VES3D_CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const long grid = std::min(nrot, (long)nsm * (P0 <= 16 ? ring_ctas_per_sm() : 1));
  k_build_ring<P0><<<(unsigned)grid, 256, G::SMEM, st>>>(R, T, C, nrot);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

// ======================================================================================
// Mixed form of the fused build on the fifth-generation tensor cores (tcgen05).
//
// The two DFT GEMMs of a rotation -- the synthesis of X, X_theta, X_phi on the upsampled
// grid (K = 2 p0 Fourier coefficients) and the transposed DFT of the 12 kernel components
// (K = 2 p1 longitudes) -- are 89% of the ring's multiply-adds. Here they run as
// tcgen05.mma kind::f16 products with BF16 operands split three ways and FP32
// accumulation in tensor memory (TMEM):
//     a = a0 + a1 + a2 (a0 = bf16(a), a1 = bf16(a - a0), a2 = bf16(a - a0 - a1)),
//     A.B ~ sum over i + j <= 2 of Ai.Bj   (six products, smallest first),
// which represents each operand to ~2^-24 relative. Three products (i + j <= 1, the
// "3xBF16" form) leave ~2^-16 and measured 2.5e-6 relative error on the self velocity;
// six measure below 1e-7 (numpy emulation of this kernel's arithmetic on the
// 512-vesicle p = 16 suspension).
//
// Positions are synthesised relative to the pole target of their hemisphere (the m = 0
// Fourier column is shifted by the target before the split, X = D + c added back in
// FP64), so that r = target - source near the pole -- where the singular kernel
// amplifies relative errors of the positions by |X| / |r| -- carries the GEMM's relative
// error of |r|, not of |X| (which includes the vesicle's centre). Kept in FP64: the m = 0
// block of the Legendre synthesis (it carries the position), the pole targets, the
// singular kernel and its quadrature weights; the other Legendre sums run in FP32 on the
// CUDA cores (their per-block shapes fill an m8n8k4 tile to a fifth). Emulated in numpy
// on the 512-vesicle suspension this arithmetic gives 1.1e-7 relative error on the self
// velocity against the FP64 oracle.
//
// One CTA of 16 warps per SM, persistent over rotations, with the Legendre tables resident
// in shared memory (the m = 0 block in FP64: it carries the vesicle's position; the other
// blocks in FP32: they multiply shape-sized coefficients) and the DFT tables as split BF16
// operands. Per rotation:
//   R (FP64, bulk-copied by TMA, the next rotation's prefetched)
//   -> Legendre synthesis (FP64 for the m = 0 block, FP32 for the others) -> A, dA split
//      to BF16 in shared memory
//      (UMMA K-major layout, no swizzle)
//   -> GEMM 1: [X | X_theta] = A [Mf | dMf], X_phi = dA Mf         (TMEM cols 0..191)
//   -> per chunk of 16 longitudes: TMEM -> shared, FP64 kernel at 33 x 16 points,
//      12 components split to BF16 -> GEMM 2 accumulating C = K Mf^T   (TMEM 192..287),
//      overlapping the next chunk's TMEM reads
//   -> TMEM -> shared (FP32), transposed Legendre sums (FP32 FMA) -> C [12][Nc].
// The last upsampled latitude (p1 + 1 = 33 rows do not fit the 32 lanes of a warp
// quarter) takes its kernel and transposed DFT in FP64 on the CUDA cores.
//
// Every wait is bounded (about a second of %globaltimer); a wait that runs out sets
// g_tc_build_error, the CTA stops, waits (bounded) for its copies and MMAs, frees its
// TMEM and returns, and the host reports the error.
// ======================================================================================
__device__ int g_tc_build_error = 0;

namespace tc {

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

constexpr uint64_t kWaitNs = 1000000000ull;  // a second: MMAs and copies here take microseconds

// Bounded wait for the phase of the given parity; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_test(bar, parity)) return true;
  const uint64_t t0 = gtimer();
  while (!mbar_test(bar, parity))
    if (gtimer() - t0 > kWaitNs) return false;
  return true;
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}

// 1-D bulk copy global -> shared through the TMA engine, completing on an mbarrier
// (addresses 16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   saddr(dst)),
               "l"(src), "r"(bytes), "r"(saddr(bar))
               : "memory");
}

// 1-D bulk copy shared -> global through the TMA engine (bulk-group completion, tracked
// per issuing thread; addresses 16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(saddr(src)), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// this thread's bulk stores have read their shared-memory sources / are complete
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor of a K-major operand without swizzle: core matrices of
// 8 rows x 16 bytes, lbo = byte distance between K-adjacent core matrices, sbo = between
// 8-row groups; bit 46 = descriptor version of sm_100.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: kind::f16, A and B BF16, D FP32, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
               : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (32x32b shape).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// The same for three column ranges, one wait for the three loads.
__device__ __forceinline__ void tmem_ld16x3(uint32_t ta, uint32_t tb, uint32_t tc_, float* a, float* b, float* c) {
  uint32_t r[48];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%48];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%49];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47}, [%50];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]),
        "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]),
        "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47])
      : "r"(ta), "r"(tb), "r"(tc_)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) {
    a[i] = __uint_as_float(r[i]);
    b[i] = __uint_as_float(r[16 + i]);
    c[i] = __uint_as_float(r[32 + i]);
  }
}

// Byte offset of element (row, k) of a K-major no-swizzle operand with kcols columns
// (core matrices K-adjacent at 128 B, 8-row groups at kcols * 16 B).
__host__ __device__ constexpr uint32_t umma_off(int row, int k, int kcols) {
  return (uint32_t)((row >> 3) * (kcols * 16) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Three-way BF16 split of a value rounded to FP32 (its 24-bit significand is covered
// exactly: v = h0 + h1 + h2 with each residual exact in FP32), stored at byte offset off
// of three operand buffers stride bytes apart.
__device__ __forceinline__ void store_split3(unsigned char* base, uint32_t stride, uint32_t off, float v) {
  const __nv_bfloat16 h0 = __float2bfloat16_rn(v);
  const float r1 = v - __bfloat162float(h0);
  const __nv_bfloat16 h1 = __float2bfloat16_rn(r1);
  const __nv_bfloat16 h2 = __float2bfloat16_rn(r1 - __bfloat162float(h1));
  *reinterpret_cast<__nv_bfloat16*>(base + off) = h0;
  *reinterpret_cast<__nv_bfloat16*>(base + stride + off) = h1;
  *reinterpret_cast<__nv_bfloat16*>(base + 2 * stride + off) = h2;
}

// The same split for two values of adjacent K columns (one 32-bit word per split).
__device__ __forceinline__ void store_split3x2(unsigned char* base, uint32_t stride, uint32_t off, float lo, float hi) {
  const __nv_bfloat162 h0 = __floats2bfloat162_rn(lo, hi);
  const float2 f0 = __bfloat1622float2(h0);
  const float rlo = lo - f0.x, rhi = hi - f0.y;
  const __nv_bfloat162 h1 = __floats2bfloat162_rn(rlo, rhi);
  const float2 f1 = __bfloat1622float2(h1);
  const __nv_bfloat162 h2 = __floats2bfloat162_rn(rlo - f1.x, rhi - f1.y);
  *reinterpret_cast<__nv_bfloat162*>(base + off) = h0;
  *reinterpret_cast<__nv_bfloat162*>(base + stride + off) = h1;
  *reinterpret_cast<__nv_bfloat162*>(base + 2 * stride + off) = h2;
}

// Split products (i, j), i + j <= 2, smallest first (compile-time in the unrolled issue loops).
__host__ __device__ constexpr int split_i(int pr) { return pr == 0 ? 2 : (pr == 1 || pr == 3) ? 1 : 0; }
__host__ __device__ constexpr int split_j(int pr) { return pr == 2 ? 2 : (pr == 1 || pr == 4) ? 1 : 0; }

// Descriptor of an operand at a byte offset from the one described by d: the start address
// field holds address >> 4 in 14 bits, so a 16-byte multiple is added there directly (no
// carry out of the field below 256 KB of shared memory).
__device__ __forceinline__ uint64_t desc_at(uint64_t d, uint32_t byte_off) { return d + (byte_off >> 4); }

}  // namespace tc

template <int P0>
struct RingTcCfg {
  using G = RingCfg<P0>;
  static constexpr int P1 = 2 * P0, L1 = P1 + 1, F0 = 2 * P0, N1 = 2 * P1, NC = P0 * (P0 + 2);
  static_assert(P0 == 16, "the tensor-core ring is laid out for p = 16 (33 upsampled latitudes)");
  static constexpr int NTHR = 512, NWARP = NTHR / 32;
  static constexpr int LDR = G::LDR;     // FP64 coefficient rows of R
  static constexpr int M0 = P0 + 1;      // the m = 0 Fourier block: coefficients 0..P0
  static constexpr int LD0 = M0;         // FP64 m = 0 table rows (odd: conflict-free columns)
  static constexpr int LDF = NC + 1;     // FP32 table rows (odd)
  static constexpr int LDCL = F0 * 12 + 4;  // FP32 transposed-DFT result: latitude stride of [lat][jf][comp]
  static constexpr int JC = 16;          // longitudes per kernel chunk (K of one GEMM-2 step)
  static constexpr int NCH = N1 / JC;    // chunks per rotation
  static constexpr int KROWS = 12 * 32;  // GEMM-2 rows (component, latitude < 32): 3 M-tiles
  // Row of (component, latitude) in the GEMM-2 operand, hence TMEM lane of its result: tile
  // comp / 4; lane quarter lat / 8; within the quarter, lane bits (lat & 3, comp bit 1) low and
  // (lat bit 2, comp bit 0) high. A quarter then holds 8 latitudes x 4 components, whose FP32
  // stores into C (latitude stride LDCL = 4 mod 32 words) fall on 32 distinct banks; the
  // chunk operand's stores stay two-way.
  __host__ __device__ static constexpr int krow(int comp, int lat) {
    return (comp >> 2) * 128 + (lat >> 3) * 32 + (((lat >> 2) & 1) * 2 + (comp & 1)) * 8 + (lat & 3) * 2 + ((comp >> 1) & 1);
  }
  static_assert(32 * JC == NTHR, "one chunk point per thread");
  // operand sizes (bytes, one split)
  static constexpr int SZ_A = 128 * F0 * 2;       // A or dA: 128 rows x K = F0
  static constexpr int SZ_B12 = 128 * F0 * 2;     // [Mf | dMf]^T: N = 2 N1 = 128 rows x K = F0
  static constexpr int SZ_BT = F0 * N1 * 2;       // Mf: N = F0 rows x K = N1
  static constexpr int SZ_K = KROWS * JC * 2;     // one chunk of kernel values
  // FP32 surface values [9][32 lat][SXS_LD]: rows of 80 bytes take the TMEM rows as
  // conflict-free float4 stores, and 8 latitudes x 4 longitudes of a warp read distinct banks
  static constexpr int SXS_LD = 20;
  static constexpr int SZ_XS = 9 * 32 * SXS_LD * 4;
  static constexpr int SZ_C = L1 * LDCL * 4;      // FP32 transposed-DFT result [lat][jf][comp]
  // byte offsets; the union region U holds A/dA (pass 1 -> GEMM 1), then two chunk buffers
  // (chunk ch in buffer ch % 2: GEMM 2 of one chunk runs while the next is formed) and the
  // chunk's surface values (-> GEMM 2), then C (-> pass 2)
  static constexpr int OFF_B12 = 0;
  static constexpr int OFF_BT = OFF_B12 + 3 * SZ_B12;
  static constexpr int OFF_U = OFF_BT + 3 * SZ_BT;
  static constexpr int OFF_A = OFF_U;
  static constexpr int OFF_K = OFF_U;
  static constexpr int OFF_XS = OFF_K + 6 * SZ_K;
  static constexpr int U_SZ = std::max(std::max(6 * SZ_A, 6 * SZ_K + SZ_XS), SZ_C);
  // a rotation's output C [12][NC] FP32, staged in U by pass 2 beside the C tile and above
  // A/dA, stored by a bulk copy during the next rotation's pass 1 (before the chunk buffers
  // reuse it)
  static constexpr int SZ_CST = 12 * NC * 4;
  static constexpr int OFF_CST = OFF_U + (std::max(SZ_C, 6 * SZ_A) + 15) / 16 * 16;
  static_assert(OFF_CST + SZ_CST <= OFF_U + U_SZ && SZ_CST % 16 == 0, "output staging inside U");
  // every region starts on a 16-byte boundary (float4 and bulk-copy destinations need it)
  static constexpr int al16(int x) { return (x + 15) / 16 * 16; }
  static constexpr int OFF_R = (OFF_U + U_SZ + 127) / 128 * 128;      // 2 x [3][LDR] FP64
  // Legendre tables of latitudes 0..LH - 1 only: the Gauss nodes are symmetric and
  // P_n^m(-x) = (-1)^(n+m) P_n^m(x), so latitude 32 - l follows from latitude l
  static constexpr int LH = P1 / 2 + 1;
  static constexpr int OFF_T0 = al16(OFF_R + 2 * 3 * LDR * 8);        // FP64 m = 0 tables: leg, dleg [LH][LD0]
  static constexpr int OFF_TF = al16(OFF_T0 + 2 * LH * LD0 * 8);      // FP32 tables: leg, dleg [LH][LDF]
  static constexpr int OFF_X32 = al16(OFF_TF + 2 * LH * LDF * 4);     // last latitude: [9][N1] FP32
  static constexpr int OFF_K32 = al16(OFF_X32 + 9 * N1 * 4);          // its kernel values [12][N1] FP32
  static constexpr int OFF_R4 = al16(OFF_K32 + 12 * N1 * 4);          // R as float4 (x, y, z, 0) [NC]
  static constexpr int OFF_MFT = al16(OFF_R4 + NC * 16);              // Mf^T [N1][F0] FP32 (the last latitude's DFT)
  static constexpr int OFF_C32 = al16(OFF_MFT + N1 * F0 * 4);         // row 32 of C [F0][12], outside U
  static constexpr int OFF_TRG = al16(OFF_C32 + F0 * 12 * 4);
  static constexpr int OFF_CQ = OFF_TRG + 6 * 8;  // the pole targets over the m = 0 Fourier row
  static constexpr int OFF_DF = OFF_CQ + 6 * 8;   // target t - centre h as FP32 pairs: hi [2][2][3], lo [2][2][3]
  static constexpr int OFF_SWF = OFF_DF + 24 * 4;  // singular weights x 1/(8 pi), FP32
  static constexpr int OFF_BO = OFF_SWF + (L1 * 4 + 7) / 8 * 8;
  static constexpr int OFF_JF = OFF_BO + ((F0 + 1) * 4 + 7) / 8 * 8;   // Fourier block of each coefficient
  static constexpr int OFF_BAR = OFF_JF + (NC + 7) / 8 * 8;
  static_assert(OFF_U % 16 == 0 && OFF_XS % 16 == 0 && OFF_R % 16 == 0 && OFF_T0 % 16 == 0 && OFF_TF % 16 == 0 && OFF_X32 % 16 == 0 &&
                    OFF_K32 % 16 == 0 && OFF_R4 % 16 == 0 && OFF_BAR % 8 == 0 && (LDCL * 4) % 16 == 0,
                "alignment of the shared-memory regions");
  static constexpr int NBAR = 5;  // GEMM 1, GEMM 2 of chunk buffers 0 and 1, R buffers 0 and 1
  static constexpr int OFF_TMEM = OFF_BAR + NBAR * 8;
  static constexpr int SMEM = OFF_TMEM + 16;
  static constexpr uint32_t TMEM_COLS = 512;
  // GEMM 2 accumulates per M tile and per split j of Mf: columns COL_T + (tile * 3 + j) * F0
  static constexpr int COL_X = 0, COL_XT = N1, COL_XP = 2 * N1, COL_T = 3 * N1;
  static_assert(COL_T + 9 * F0 <= (int)TMEM_COLS, "TMEM columns");
  static_assert(SZ_BT == (F0 / 8) * (N1 * 16), "the three Mf splits continue one K-major operand of N = 3 F0");
  static_assert(SMEM <= 227 * 1024, "shared memory");
};

// The singular kernel (FP64) of one pole target t at one upsampled point: positions D
// relative to the centre of the point's hemisphere h, the tangents, the latitude's
// singular weight; out[6] the weighted single-layer tensor (src/SphericalHarmonics.cc:989-1068).
__device__ __forceinline__ void ring_kernel_sl(double px, double py, double pz, double area, const double* trg,
                                               const double* cen, int h, int t, double w, double* out) {
  // r = target_t - (centre_h + D) with target_t - centre_h exact (0 when t == h)
  const double dx = (trg[t] - cen[h * 3]) - px, dy = (trg[2 + t] - cen[h * 3 + 1]) - py,
               dz = (trg[4 + t] - cen[h * 3 + 2]) - pz;
  const double r2 = dx * dx + dy * dy + dz * dz;
  double rinv = rsqrt_f64_int_seed(r2);  // (r2 below 2^-126 is cut off here too)
  if (r2 <= 2.220446049250313e-16) rinv = 0.0;
  const double a1 = kInv8Pi * w * area * rinv;
  const double a2 = a1 * rinv * rinv;
  out[0] = a1 + dx * dx * a2;
  out[1] = dx * dy * a2;
  out[2] = dx * dz * a2;
  out[3] = a1 + dy * dy * a2;
  out[4] = dy * dz * a2;
  out[5] = a1 + dz * dz * a2;
}

__device__ __forceinline__ double area_of(double ax, double ay, double az, double bx, double by, double bz) {
  const double nx = ay * bz - az * by, ny = az * bx - ax * bz, nz = ax * by - ay * bx;
  const double n2 = nx * nx + ny * ny + nz * nz;
  return n2 * rsqrt_f64_int_seed(n2);  // |X_theta x X_phi| > 0 on the upsampled grid
}

// 1/sqrt(x) in FP32: the hardware estimate and one Newton step (about one ulp).
__device__ __forceinline__ float rsqrt_f32_nr(float x) {
  const float y = rsqrt_ftz(x);
  const float e = fmaf(-x * y, y, 1.f);
  return fmaf(0.5f * y, e, y);
}

// FP32 forms of the two above for the tensor-core build, whose surface values are FP32
// and whose kernel values are rounded to FP32 for the split. The offset of the pole target
// t from the point's hemisphere centre h arrives as an FP32 pair (hi + lo: the FP64
// difference to FP32 rounding); it is 0 for t == h, so the near-pole differences, where
// the kernel is large, are exact, and for t != h the point is a vesicle size away. w holds
// the latitude's singular weight times 1/(8 pi).
__device__ __forceinline__ float area_of_f32(float ax, float ay, float az, float bx, float by, float bz) {
  const float nx = fmaf(ay, bz, -az * by), ny = fmaf(az, bx, -ax * bz), nz = fmaf(ax, by, -ay * bx);
  const float n2 = fmaf(nx, nx, fmaf(ny, ny, nz * nz));
  return n2 * rsqrt_f32_nr(n2);
}

__device__ __forceinline__ void ring_kernel_sl_f32(float px, float py, float pz, float area, const float* dhi,
                                                   const float* dlo, float w, float* out) {
  const float dx = (dhi[0] - px) + dlo[0], dy = (dhi[1] - py) + dlo[1], dz = (dhi[2] - pz) + dlo[2];
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  const float rinv = r2 > 2.220446049250313e-16f ? rsqrt_f32_nr(r2) : 0.f;
  const float a1 = w * area * rinv;
  const float a2 = a1 * rinv * rinv;
  out[0] = fmaf(dx * dx, a2, a1);
  out[1] = dx * dy * a2;
  out[2] = dx * dz * a2;
  out[3] = fmaf(dy * dy, a2, a1);
  out[4] = dy * dz * a2;
  out[5] = fmaf(dz * dz, a2, a1);
}

template <int P0>
__global__ void __launch_bounds__(512, 1) k_build_ring_tc(const double* __restrict__ R, DevTables T,
                                                          float* __restrict__ C, long nrot) {
  using G = RingCfg<P0>;
  using H = RingTcCfg<P0>;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* sB12 = smem + H::OFF_B12;
  unsigned char* sBT = smem + H::OFF_BT;
  unsigned char* sA = smem + H::OFF_A;                 // splits at sA + i * SZ_A
  unsigned char* sdA = smem + H::OFF_A + 3 * H::SZ_A;  // splits at sdA + i * SZ_A
  unsigned char* sK = smem + H::OFF_K;                 // splits at sK + i * SZ_K
  float* sXs = reinterpret_cast<float*>(smem + H::OFF_XS);
  float* sC = reinterpret_cast<float*>(smem + H::OFF_U);
  double* sRb = reinterpret_cast<double*>(smem + H::OFF_R);
  double* sT0 = reinterpret_cast<double*>(smem + H::OFF_T0);  // leg, then dleg: [LH][LD0]
  float* sTF = reinterpret_cast<float*>(smem + H::OFF_TF);    // leg, then dleg: [LH][LDF]
  float* sX32 = reinterpret_cast<float*>(smem + H::OFF_X32);
  float* sK32 = reinterpret_cast<float*>(smem + H::OFF_K32);
  float4* sR4 = reinterpret_cast<float4*>(smem + H::OFF_R4);
  float* sMfT = reinterpret_cast<float*>(smem + H::OFF_MFT);
  float* sC32 = reinterpret_cast<float*>(smem + H::OFF_C32);
  double* trg = reinterpret_cast<double*>(smem + H::OFF_TRG);
  double* cq = reinterpret_cast<double*>(smem + H::OFF_CQ);
  float* sSwf = reinterpret_cast<float*>(smem + H::OFF_SWF);
  float* sDf = reinterpret_cast<float*>(smem + H::OFF_DF);  // hi at [(h * 2 + t) * 3 + d], lo 12 on
  int* sBo = reinterpret_cast<int*>(smem + H::OFF_BO);
  unsigned char* sJf = smem + H::OFF_JF;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + H::OFF_BAR);
  uint64_t* bar_mma1 = bars;     // GEMM 1 done
  uint64_t* bar_k = bars + 1;    // [2] GEMM 2 of the chunk in buffer 0 / 1 done (the buffer is free)
  uint64_t* bar_r = bars + 3;    // [2] R buffers loaded
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + H::OFF_TMEM);
  int* s_abort = reinterpret_cast<int*>(smem + H::OFF_TMEM + 4);

  constexpr int NTHR = H::NTHR;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NC = H::NC, LDR = H::LDR, F0 = H::F0, N1 = H::N1, L1 = H::L1, M0 = H::M0;
  constexpr int LD0 = H::LD0, LDF = H::LDF, LDCL = H::LDCL, LH = H::LH;

  // ---- set-up: TMEM, barriers, constant operands and tables ---------------------------
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::saddr(s_tmem)),
                 "r"(H::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < H::NBAR; i++) tc::mbar_init(bars + i);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // [Mf | dMf]^T and Mf as split BF16 operands: B12 row n < N1 is Mf[.][n], n >= N1 dMf[.][n - N1]
  for (int i = tid; i < 2 * N1 * F0; i += NTHR) {
    const int n = i / F0, k = i - n * F0;
    const double v = n < N1 ? __ldg(T.syn1_four + k * N1 + n) : __ldg(T.syn1_dfour + k * N1 + n - N1);
    tc::store_split3(sB12, H::SZ_B12, tc::umma_off(n, k, F0), (float)v);
  }
  for (int i = tid; i < F0 * N1; i += NTHR) {
    const int n = i / N1, k = i - n * N1;  // BT[jf][j] = Mf[jf][j]
    const float v = (float)__ldg(T.syn1_four + i);
    tc::store_split3(sBT, H::SZ_BT, tc::umma_off(n, k, N1), v);
    sMfT[k * F0 + n] = v;  // the same FP32 values (the split covers them exactly), transposed
  }
  // Legendre tables resident for the CTA's life: the m = 0 block in FP64 (it carries the
  // vesicle's position), the other blocks in FP32 (their values multiply shape-sized
  // coefficients; no change in the self velocity's error measured)
  for (int i = tid; i < 2 * LH * LD0; i += NTHR) {
    const int tb = i / (LH * LD0), r = i - tb * LH * LD0, lat = r / LD0, c = r - lat * LD0;
    sT0[i] = __ldg((tb ? T.syn1_dleg_t : T.syn1_leg_t) + (long)lat * NC + c);
  }
  for (int i = tid; i < 2 * LH * LDF; i += NTHR) {
    const int tb = i / (LH * LDF), r = i - tb * LH * LDF, lat = r / LDF, c = r - lat * LDF;
    sTF[i] = c < NC ? (float)__ldg((tb ? T.syn1_dleg_t : T.syn1_leg_t) + (long)lat * NC + c) : 0.f;
  }
  for (int i = tid; i < L1; i += NTHR) sSwf[i] = (float)(kInv8Pi * __ldg(T.sing_w + i));
  for (int i = tid; i <= F0; i += NTHR) sBo[i] = __ldg(T.blk_off + i);
  for (int i = tid; i < NC; i += NTHR) sJf[i] = (unsigned char)__ldg(T.jf_of_coef + i);
  tc::fence_async_smem();
  tc::tc_before_sync();
  __syncthreads();
  tc::tc_after_sync();
  const uint32_t tmem = *s_tmem;
  const double mf00 = __ldg(T.syn1_four);  // the constant m = 0 Fourier row
  // operand descriptors of split 0 (K-major, no swizzle; LBO 128 B, SBO one 8-row group)
  const uint64_t dA = tc::umma_desc(tc::saddr(sA), 128, F0 * 16), ddA = tc::umma_desc(tc::saddr(sdA), 128, F0 * 16);
  const uint64_t dB12 = tc::umma_desc(tc::saddr(sB12), 128, F0 * 16);
  const uint64_t dBT = tc::umma_desc(tc::saddr(sBT), 128, N1 * 16);
  const uint64_t dK0 = tc::umma_desc(tc::saddr(sK), 128, H::JC * 16);
  const uint64_t dK1 = tc::umma_desc(tc::saddr(sK + 3 * H::SZ_K), 128, H::JC * 16);

  auto issue_r = [&](long rot, int b) {
    double* dst = sRb + b * 3 * LDR;
    tc::mbar_expect_tx(bar_r + b, 3 * NC * 8);
    for (int d = 0; d < 3; d++) tc::bulk_g2s(dst + d * LDR, R + (rot * 3 + d) * NC, NC * 8, bar_r + b);
  };
  // phases waited for per barrier and issued (uniform over the CTA: every issue decision
  // depends only on loop indices)
  uint32_t n_r[2] = {0, 0}, n_k[2] = {0, 0}, n_mma1 = 0;
  uint32_t i_r[2] = {0, 0}, i_k[2] = {0, 0}, i_mma1 = 0;
  bool ok = true;
  auto wait = [&](uint64_t* bar, uint32_t& cnt) {
    if (!tc::mbar_wait(bar, cnt & 1)) {
      atomicExch(&g_tc_build_error, 1);
      *s_abort = 1;
    }
    cnt++;
  };
  auto sync_ok = [&]() {
    __syncthreads();
    return *s_abort == 0;
  };
  // Per-rotation values from R, formed by the 224 threads i = 0..223 of seven whole warps
  // (named barrier 1) before the rotation begins: the pole targets (trg), their values over
  // the m = 0 Fourier row (cq), target t - centre h as FP32 pairs (sDf), R as float4 (sR4).
  // Inside the loop the warps idle in pass 2 (threads NC..511) form the next rotation's.
  static_assert(NTHR - NC == 224 && NC >= 224, "seven warps idle in pass 2");
  auto prep = [&](const double* sRn, int i) {
    for (int c = i; c < NC; c += 224) sR4[c] = make_float4((float)sRn[c], (float)sRn[LDR + c], (float)sRn[2 * LDR + c], 0.f);
    if (i < 6) {
      const int c = i >> 1, t = i & 1;
      double s = 0.0;
      for (int n = 0; n <= P0; n++) s += sRn[c * LDR + n] * __ldg(T.qp + t * (P0 + 1) + n);
      trg[c * 2 + t] = s;
    }
    asm volatile("bar.sync 1, 224;" ::: "memory");
    if (i < 6) {  // cq[h * 3 + d]: the target of hemisphere h (its centre) over the m = 0 row
      cq[i] = trg[(i % 3) * 2 + i / 3] / mf00;
    } else if (i < 18) {  // target t - centre h (the target of hemisphere h) as FP32 pairs
      const int j = i - 6, h = j / 6, t = (j / 3) & 1, d = j % 3;
      const double dd = trg[d * 2 + t] - trg[d * 2 + h];
      const float hi = (float)dd;
      sDf[j] = hi;
      sDf[12 + j] = (float)(dd - (double)hi);
    }
  };
  if (blockIdx.x < nrot) {
    if (tid == 0) issue_r(blockIdx.x, 0);
    i_r[0]++;
    wait(bar_r, n_r[0]);
    if (tid < 224) prep(sRb, tid);
    ok = sync_ok();
  }
  float* sCst = reinterpret_cast<float*>(smem + H::OFF_CST);
  constexpr int kIssuer = 12 * 32;  // a thread of a warp idle in pass 1: bulk copies in and out
  long it = 0, staged = -1;         // staged: the rotation whose C waits in sCst
  for (long rot = blockIdx.x; rot < nrot && ok; rot += gridDim.x, it++) {
    const int rb = (int)(it & 1);
    const double* sR = sRb + rb * 3 * LDR;
    const bool has_next = rot + gridDim.x < nrot;
    // ---- pass 1: Legendre synthesis -> split BF16 A, dA -----------------------------------
    // the m = 0 block in FP64 (it carries the vesicle's position, shifted by the pole target
    // here), the others in FP32 (shape-sized terms; their sums are rounded to FP32 for the
    // split anyway)
    // Sums over Fourier block k at latitude pair l, split by the parity of n + m: latitude l
    // is even + odd, its mirror 32 - l even - odd (the theta derivative odd - even), from
    // one pass over the coefficients (P_n^m(-x) = (-1)^(n+m) P_n^m(x) on the symmetric Gauss
    // nodes); l = 16 is the equator. The m = 0 block in FP64, centred on the pole targets
    // (its values carry the vesicle's position), the others in FP32.
    auto block_sums = [&](int k, int l, float* ev, float* od, float* dev, float* dod) {
      if (k == 0) {
        const double* L = sT0 + l * LD0;
        const double* dL = sT0 + (LH + l) * LD0;
        double e0 = 0, e1 = 0, e2 = 0, f0 = 0, f1 = 0, f2 = 0;  // n even
        double o0 = 0, o1 = 0, o2 = 0, g0 = 0, g1 = 0, g2 = 0;  // n odd
#pragma unroll
        for (int c = 0; c < M0; c += 2) {
          const double lv = L[c], dl = dL[c], r0 = sR[c], r1 = sR[LDR + c], r2 = sR[2 * LDR + c];
          e0 = fma(lv, r0, e0); e1 = fma(lv, r1, e1); e2 = fma(lv, r2, e2);
          f0 = fma(dl, r0, f0); f1 = fma(dl, r1, f1); f2 = fma(dl, r2, f2);
          if (c + 1 < M0) {
            const double lw = L[c + 1], dw = dL[c + 1], q0 = sR[c + 1], q1 = sR[LDR + c + 1], q2 = sR[2 * LDR + c + 1];
            o0 = fma(lw, q0, o0); o1 = fma(lw, q1, o1); o2 = fma(lw, q2, o2);
            g0 = fma(dw, q0, g0); g1 = fma(dw, q1, g1); g2 = fma(dw, q2, g2);
          }
        }
        ev[0] = (float)(e0 + o0 - cq[0]); ev[1] = (float)(e1 + o1 - cq[1]); ev[2] = (float)(e2 + o2 - cq[2]);
        od[0] = (float)(e0 - o0 - cq[3]); od[1] = (float)(e1 - o1 - cq[4]); od[2] = (float)(e2 - o2 - cq[5]);
        dev[0] = (float)(f0 + g0); dev[1] = (float)(f1 + g1); dev[2] = (float)(f2 + g2);
        dod[0] = (float)(g0 - f0); dod[1] = (float)(g1 - f1); dod[2] = (float)(g2 - f2);
      } else {
        const float* L = sTF + l * LDF;
        const float* dL = sTF + (LH + l) * LDF;
        const int c0 = sBo[k], c1 = sBo[k + 1];
        float ge[6] = {}, go[6] = {};
        int c = c0;
        for (; c + 1 < c1; c += 2) {  // n - m = c - c0: even, then odd
          const float l0 = L[c], d0 = dL[c], l1 = L[c + 1], d1 = dL[c + 1];
          const float4 r = sR4[c], q = sR4[c + 1];
          ge[0] = fmaf(l0, r.x, ge[0]); ge[1] = fmaf(l0, r.y, ge[1]); ge[2] = fmaf(l0, r.z, ge[2]);
          ge[3] = fmaf(d0, r.x, ge[3]); ge[4] = fmaf(d0, r.y, ge[4]); ge[5] = fmaf(d0, r.z, ge[5]);
          go[0] = fmaf(l1, q.x, go[0]); go[1] = fmaf(l1, q.y, go[1]); go[2] = fmaf(l1, q.z, go[2]);
          go[3] = fmaf(d1, q.x, go[3]); go[4] = fmaf(d1, q.y, go[4]); go[5] = fmaf(d1, q.z, go[5]);
        }
        if (c < c1) {
          const float l0 = L[c], d0 = dL[c];
          const float4 r = sR4[c];
          ge[0] = fmaf(l0, r.x, ge[0]); ge[1] = fmaf(l0, r.y, ge[1]); ge[2] = fmaf(l0, r.z, ge[2]);
          ge[3] = fmaf(d0, r.x, ge[3]); ge[4] = fmaf(d0, r.y, ge[4]); ge[5] = fmaf(d0, r.z, ge[5]);
        }
#pragma unroll
        for (int d = 0; d < 3; d++) {
          ev[d] = ge[d] + go[d];
          od[d] = ge[d] - go[d];
          dev[d] = ge[3 + d] + go[3 + d];
          dod[d] = go[3 + d] - ge[3 + d];
        }
      }
    };
    // rows of latitude l (hemisphere 0: l + 32 d) and of its mirror (hemisphere 1: 32 - l +
    // 32 d, or 96 + d for latitude 32)
    auto row_of = [&](int lat, int d) { return lat < 32 ? lat + 32 * d : 96 + d; };
    // Items (pair of blocks kp = (2 kp, 2 kp + 1) >= 1, latitude pair l): a warp holds 8
    // latitude pairs x 4 block pairs, so each of its bf16x2 stores fills whole core matrices
    // of the K-major operands (conflict-free); warps 0-7 take l < 16, warp 8 the equator.
    // The pair of blocks 0 and 1 goes to warps 9 (block 0, FP64) and 10 (block 1), one lane
    // per latitude pair with 16-bit stores, so that the FP64 sums run beside the others
    // instead of after them (they were the pass's critical path).
    static_assert(H::P1 == 32 && LH == 17 && F0 == 32 && NTHR >= 11 * 32, "latitude and block pairs");
    if (warp < 9) {
      const int l = warp < 8 ? 8 * (warp & 1) + (lane >> 2) : 16;
      const int kp = warp < 8 ? 4 * (warp >> 1) + (lane & 3) : lane;
      if (kp > 0 && (warp < 8 || lane < 16)) {
        const int lb = H::P1 - l;
        float ev[2][3], od[2][3], dev[2][3], dod[2][3];  // [block][coordinate]
        block_sums(2 * kp, l, ev[0], od[0], dev[0], dod[0]);
        block_sums(2 * kp + 1, l, ev[1], od[1], dev[1], dod[1]);
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const uint32_t o = tc::umma_off(row_of(l, d), 2 * kp, F0);
          tc::store_split3x2(sA, H::SZ_A, o, ev[0][d], ev[1][d]);
          tc::store_split3x2(sdA, H::SZ_A, o, dev[0][d], dev[1][d]);
        }
        if (l < 16) {
#pragma unroll
          for (int d = 0; d < 3; d++) {
            const uint32_t o = tc::umma_off(row_of(lb, d), 2 * kp, F0);
            tc::store_split3x2(sA, H::SZ_A, o, od[0][d], od[1][d]);
            tc::store_split3x2(sdA, H::SZ_A, o, dod[0][d], dod[1][d]);
          }
        }
      }
    } else if (tid == kIssuer) {
      // the previous rotation's C out, the next rotation's R in (buffer rb ^ 1 held the R of
      // rotation it - 1, whose readers are done)
      if (staged >= 0) tc::bulk_s2g(C + staged * G::NOUT, sCst, H::SZ_CST);
      if (has_next) issue_r(rot + gridDim.x, rb ^ 1);
    } else if (warp < 11 && lane < LH) {
      const int k = warp - 9, l = lane, lb = H::P1 - l;
      float ev[3], od[3], dev[3], dod[3];
      block_sums(k, l, ev, od, dev, dod);
#pragma unroll
      for (int d = 0; d < 3; d++) {
        tc::store_split3(sA, H::SZ_A, tc::umma_off(row_of(l, d), k, F0), ev[d]);
        tc::store_split3(sdA, H::SZ_A, tc::umma_off(row_of(l, d), k, F0), dev[d]);
        if (l < 16) {
          tc::store_split3(sA, H::SZ_A, tc::umma_off(row_of(lb, d), k, F0), od[d]);
          tc::store_split3(sdA, H::SZ_A, tc::umma_off(row_of(lb, d), k, F0), dod[d]);
        }
      }
    }
    if (has_next) i_r[rb ^ 1]++;
    if (tid == kIssuer && staged >= 0) tc::bulk_wait_read();  // sCst free for the chunk buffers
    staged = -1;
    // ---- GEMM 1 on the tensor cores ------------------------------------------------------
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::tc_after_sync();
      constexpr uint32_t id128 = tc::idesc_bf16(128, 2 * N1), id64 = tc::idesc_bf16(128, N1);
#pragma unroll
      for (int pr = 0; pr < 6; pr++) {
#pragma unroll
        for (int s = 0; s < F0 / 16; s++) {
          const uint64_t db = tc::desc_at(dB12, tc::split_j(pr) * H::SZ_B12 + s * 256);
          tc::mma_bf16(tmem + H::COL_X, tc::desc_at(dA, tc::split_i(pr) * H::SZ_A + s * 256), db, id128,
                       (pr | s) ? 1u : 0u);
          tc::mma_bf16(tmem + H::COL_XP, tc::desc_at(ddA, tc::split_i(pr) * H::SZ_A + s * 256), db, id64,
                       (pr | s) ? 1u : 0u);
        }
      }
      tc::mma_commit(bar_mma1);
    }
    i_mma1++;
    wait(bar_mma1, n_mma1);
    if (!(ok = sync_ok())) break;
    tc::tc_after_sync();
    // ---- per chunk of longitudes: kernel values and GEMM 2 ------------------------------
    for (int ch = 0; ch < H::NCH && ok; ch++) {
      // (a) surfaces of the chunk: TMEM -> shared; warp w reads lane quarter w % 4 of the
      // variable w / 4 (X, X_theta, X_phi); quarter 3 holds the last latitude (lanes 0..2)
      if (warp < 12) {
        const int q = warp & 3, var = warp >> 2;
        float v[16];
        const int col = (var == 0 ? H::COL_X : var == 1 ? H::COL_XT : H::COL_XP) + ch * H::JC;
        tc::tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + col, v);
        if (q < 3) {
          float4* o = reinterpret_cast<float4*>(sXs + ((var * 3 + q) * 32 + lane) * H::SXS_LD);
#pragma unroll
          for (int jj = 0; jj < H::JC / 4; jj++)
            o[jj] = make_float4(v[4 * jj], v[4 * jj + 1], v[4 * jj + 2], v[4 * jj + 3]);
        } else if (lane < 3) {
          float* o = sX32 + (var * 3 + lane) * N1 + ch * H::JC;
#pragma unroll
          for (int jj = 0; jj < H::JC; jj++) o[jj] = v[jj];
        }
      }
      tc::tc_before_sync();
      const int kb = ch & 1;
      unsigned char* sKb = sK + kb * 3 * H::SZ_K;
      if (ch >= 2) wait(bar_k + kb, n_k[kb]);  // GEMM 2 of chunk ch - 2 has read this buffer
      if (!(ok = sync_ok())) break;
      // (b) singular kernel (FP64) at the chunk's 32 x 16 points (one per thread) -> split
      // BF16 chunk operand; a warp takes 8 latitudes x 4 longitudes (its split stores then
      // fall on 16 banks twice, against four times for 2 latitudes x 16 longitudes)
      {
        const int lat = (warp >> 2) * 8 + (lane >> 2), jj = (warp & 3) * 4 + (lane & 3);
        const int h = 2 * lat > H::P1 ? 1 : 0;
        const float* xs = sXs + lat * H::SXS_LD + jj;
        constexpr int VS = 32 * H::SXS_LD;
        const float area = area_of_f32(xs[3 * VS], xs[4 * VS], xs[5 * VS], xs[6 * VS], xs[7 * VS], xs[8 * VS]);
        const float px = xs[0], py = xs[VS], pz = xs[2 * VS];
        float kv[12];
#pragma unroll
        for (int t = 0; t < 2; t++)
          ring_kernel_sl_f32(px, py, pz, area, sDf + (h * 2 + t) * 3, sDf + 12 + (h * 2 + t) * 3,
                             sSwf[t ? lat : H::P1 - lat], kv + t * 6);
        // lanes 2i, 2i + 1 hold longitudes jj, jj + 1 of one latitude: the even lane splits
        // components 0..5 of both, the odd lane 6..11, as BF16 pairs (one 32-bit word per
        // split and component)
        const bool odd = lane & 1;
        const uint32_t off = tc::umma_off(0, jj & ~1, H::JC);  // the row is added below
#pragma unroll
        for (int c = 0; c < 6; c++) {
          const float send = odd ? kv[c] : kv[6 + c];
          const float recv = __shfl_xor_sync(0xffffffffu, send, 1);
          const float lo = odd ? recv : kv[c], hi = odd ? kv[6 + c] : recv;
          const int comp = odd ? 6 + c : c;
          tc::store_split3x2(sKb, H::SZ_K, off + tc::umma_off(H::krow(comp, lat), 0, H::JC), lo, hi);
        }
      }
      tc::fence_async_smem();
      __syncthreads();
      // GEMM 2 issued by warp 12, which has no surface values to move: warps 0-11 start the
      // next chunk's TMEM reads meanwhile
      if (tid == 12 * 32) {
        tc::tc_after_sync();
        // split i of the kernel values against the Mf splits j <= 2 - i stacked along N (the
        // three split buffers continue one operand): one MMA of N = (3 - i) F0 per M tile puts
        // K_i Mf_j^T into column block j; nine MMAs per chunk instead of eighteen of N = F0.
        // Split 0 comes first: it writes all three blocks (the first chunk's initial values).
        const uint64_t dBc = tc::desc_at(dBT, ch * (H::JC / 8) * 128), dKc = kb ? dK1 : dK0;
#pragma unroll
        for (int i = 0; i < 3; i++) {
          const uint32_t idn = tc::idesc_bf16(128, (3 - i) * F0);
#pragma unroll
          for (int tt = 0; tt < 3; tt++)
            tc::mma_bf16(tmem + H::COL_T + tt * 3 * F0, tc::desc_at(dKc, i * H::SZ_K + tt * 128 * H::JC * 2), dBc, idn,
                         (ch | i) ? 1u : 0u);
        }
        tc::mma_commit(bar_k + kb);
      }
      i_k[kb]++;
    }
    if (!ok) break;
    // ---- the last latitude's kernel (warps 8-11, one (point, target) each) and its
    // transposed DFT (its row of C, into a buffer outside U) by warps 0-11 while warp 12
    // issues the last GEMM 2 and the GEMMs run (named barrier 2: warp 12 is not waited for);
    // then the transposed-DFT result -> shared (FP32) ----------------------------------
    if (warp >= 8 && warp < 12) {
      const int item = tid - 256, j = item >> 1, t = item & 1;
      const float* xs = sX32 + j;
      const float area = area_of_f32(xs[3 * N1], xs[4 * N1], xs[5 * N1], xs[6 * N1], xs[7 * N1], xs[8 * N1]);
      float kv[6];
      ring_kernel_sl_f32(xs[0], xs[N1], xs[2 * N1], area, sDf + (2 + t) * 3, sDf + 12 + (2 + t) * 3,
                         sSwf[t ? 32 : H::P1 - 32], kv);
#pragma unroll
      for (int c = 0; c < 6; c++) sK32[(t * 6 + c) * N1 + j] = kv[c];
    }
    static_assert(12 * F0 == 384 && 2 * N1 == 128, "warps 0-11: the DFT; warps 8-11: the 128 kernel items");
    if (warp < 12) asm volatile("bar.sync 2, 384;" ::: "memory");
    // FP32 like the BF16-split GEMM of the other rows (the same FP32 values of Mf): a warp
    // takes one component, its lanes the 32 Fourier columns (broadcast kernel values,
    // conflict-free Mf^T rows). It read Mf from global memory in FP64 before, 32 cache lines
    // per load: 42% of a rotation's time.
    if (tid < 12 * F0) {
      const int comp = tid / F0, jf = tid - comp * F0;
      const float* kr = sK32 + comp * N1;
      const float* mf = sMfT + jf;
      float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll 4
      for (int j = 0; j < N1; j += 4) {
        s0 = fmaf(kr[j], mf[j * F0], s0);
        s1 = fmaf(kr[j + 1], mf[(j + 1) * F0], s1);
        s2 = fmaf(kr[j + 2], mf[(j + 2) * F0], s2);
        s3 = fmaf(kr[j + 3], mf[(j + 3) * F0], s3);
      }
      sC32[jf * 12 + comp] = (s0 + s1) + (s2 + s3);
    }
    // the last two chunks' GEMMs 2 before TMEM is read and U reused
    wait(bar_k + 0, n_k[0]);
    wait(bar_k + 1, n_k[1]);
    if (!(ok = sync_ok())) break;
    tc::tc_after_sync();
    if (warp < 12) {
      const int q = warp & 3, tt = warp >> 2;
      // TMEM lane 32 q + lane of tile tt holds row krow(comp, lat)
      const int lat = 8 * q + ((lane >> 4) & 1) * 4 + ((lane >> 1) & 3);
      const int comp = 4 * tt + (((lane & 1) << 1) | ((lane >> 3) & 1));
      float v[16], w1[16], w2[16];
#pragma unroll
      for (int half = 0; half < 2; half++) {  // the split blocks summed smallest first
        const uint32_t ta = tmem + ((uint32_t)(32 * q) << 16) + H::COL_T + tt * 3 * F0 + half * 16;
        tc::tmem_ld16x3(ta, ta + F0, ta + 2 * F0, v, w1, w2);
        float* o = sC + lat * LDCL + half * 16 * 12 + comp;
#pragma unroll
        for (int x = 0; x < 16; x++) o[x * 12] = v[x] + (w1[x] + w2[x]);
      }
    }
    tc::tc_before_sync();
    __syncthreads();
    // ---- pass 2: transposed Legendre sums (FP32 FMA), one output coefficient and its 12
    // components per thread; measured 1.1e-7 on the self velocity (emulation against the
    // FP64 oracle). Latitude pairs first: row l <- C[l] + C[32 - l], row 32 - l <- C[l] -
    // C[32 - l] (l < 16), so that a coefficient of parity n + m sums 17 rows with the
    // tables of latitudes 0..16 (P_n^m at latitude 32 - l is (-1)^(n+m) that at l). -------
    {
      constexpr int RQ = F0 * 12 / 4;  // float4 per row of C
      for (int i = tid; i < (H::P1 / 2) * RQ; i += NTHR) {
        const int l = i / RQ, f = i - l * RQ;
        float4* pa = reinterpret_cast<float4*>(sC + l * LDCL) + f;
        float4* pb = reinterpret_cast<float4*>(l ? sC + (H::P1 - l) * LDCL : sC32) + f;  // row 32 in sC32
        const float4 x = *pa, y = *pb;
        *pa = make_float4(x.x + y.x, x.y + y.y, x.z + y.z, x.w + y.w);
        *pb = make_float4(x.x - y.x, x.y - y.y, x.z - y.z, x.w - y.w);
      }
    }
    __syncthreads();
    if (has_next) {  // the next rotation's R (issued during pass 1)
      if (tid >= NC)
        wait(bar_r + (rb ^ 1), n_r[rb ^ 1]);
      else
        n_r[rb ^ 1]++;
    }
    if (tid >= NC) {
      if (has_next) prep(sRb + (rb ^ 1) * 3 * LDR, tid - NC);
    } else {
      const int c = tid, jf = sJf[c];
      const bool odd = (c - sBo[jf]) & 1;  // parity of n + m
      const float4* a = reinterpret_cast<const float4*>(sC + jf * 12);
      const float* b = sTF + c;
      float acc[12];
#pragma unroll
      for (int q = 0; q < 12; q++) acc[q] = 0.f;
#pragma unroll 4
      for (int l = 0; l < LH; l++) {
        const float w = b[l * LDF];
        const int row = (odd && l < H::P1 / 2) ? H::P1 - l : l;  // C- for odd parity; the equator alone
        const float4* al = row == H::P1 ? reinterpret_cast<const float4*>(sC32 + jf * 12) : a + row * (LDCL / 4);
        const float4 a0 = al[0], a1 = al[1], a2 = al[2];
        acc[0] = fmaf(a0.x, w, acc[0]); acc[1] = fmaf(a0.y, w, acc[1]);
        acc[2] = fmaf(a0.z, w, acc[2]); acc[3] = fmaf(a0.w, w, acc[3]);
        acc[4] = fmaf(a1.x, w, acc[4]); acc[5] = fmaf(a1.y, w, acc[5]);
        acc[6] = fmaf(a1.z, w, acc[6]); acc[7] = fmaf(a1.w, w, acc[7]);
        acc[8] = fmaf(a2.x, w, acc[8]); acc[9] = fmaf(a2.y, w, acc[9]);
        acc[10] = fmaf(a2.z, w, acc[10]); acc[11] = fmaf(a2.w, w, acc[11]);
      }
#pragma unroll
      for (int q = 0; q < 12; q++) sCst[q * NC + c] = acc[q];  // conflict-free: consecutive c
    }
    staged = rot;
    tc::fence_async_smem();  // the staged C is read by the bulk copy (async proxy)
    // pass 2's reads of C before the next rotation's pass 1 overwrites it
    if (!(ok = sync_ok())) break;
  }
  if (tid == kIssuer) {  // the last rotation's C, then every bulk store complete
    if (ok && staged >= 0) tc::bulk_s2g(C + staged * G::NOUT, sCst, H::SZ_CST);
    tc::bulk_wait_all();
  }
  // ---- drain: copies and MMAs issued but not waited for (after an abort, whatever was in
  // flight), each wait bounded; then TMEM is freed -------------------------------------
  {
    bool drained = true;
    auto drain = [&](uint64_t* bar, uint32_t& waited, uint32_t issued) {
      while (drained && waited < issued) {
        if (!tc::mbar_wait(bar, waited & 1)) {
          atomicExch(&g_tc_build_error, 1);
          drained = false;
        }
        waited++;
      }
    };
    for (int b = 0; b < 2; b++) drain(bar_r + b, n_r[b], i_r[b]);
    for (int b = 0; b < 2; b++) drain(bar_k + b, n_k[b], i_k[b]);
    drain(bar_mma1, n_mma1, i_mma1);
  }
  tc::tc_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::tc_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(H::TMEM_COLS) : "memory");
  }
}

bool tc_build_supported(int p0, int p1) { return p0 == 16 && p1 == 32; }

int launch_build_ring_tc(const double* R, long nrot, const DevTables& T, float* C, cudaStream_t st) {
  if (nrot <= 0) return VES3D_OK;
  if (!tc_build_supported(T.p0, T.p1)) {
    set_error("tensor-core build not laid out for p = %d, p_up = %d", T.p0, T.p1);
    return VES3D_ERR_ARG;
  }
  if (((uintptr_t)R | (uintptr_t)C) & 15) {  // the bulk copies in and out need 16-byte alignment
    set_error("internal: tensor-core build buffers not 16-byte aligned");
    return VES3D_ERR_ARG;
  }
  using H = RingTcCfg<16>;
  VES3D_CK(cudaFuncSetAttribute(k_build_ring_tc<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, H::SMEM));
  int dev = 0, nsm = 148;
  VES3D_CK(cudaGetDevice(&dev));
  VES3D_CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const long grid = std::min(nrot, (long)nsm);
  k_build_ring_tc<16><<<(unsigned)grid, H::NTHR, H::SMEM, st>>>(R, T, C, nrot);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

int tc_build_error(bool reset) {
  int v = 0;
  VES3D_CK(cudaMemcpyFromSymbol(&v, g_tc_build_error, sizeof(int)));
  if (v && reset) {
    const int zero = 0;
    VES3D_CK(cudaMemcpyToSymbol(g_tc_build_error, &zero, sizeof(int)));
  }
  return v;
}

bool fused_build_supported(int p0, int p1) {
  if (p1 != 2 * p0) return false;
  // the tensor-core tiling needs 2 p0 % 8 == 0 and 4 p0 % 16 == 0
  switch (p0) {
    case 4: case 8: case 12: case 16: case 24: return true;
    default: return false;
  }
}

int launch_build_ring(const double* R, long nrot, const DevTables& T, double* C, cudaStream_t st) {
  if (nrot <= 0) return VES3D_OK;
  switch (T.p0) {
    case 4: return launch_ring<4>(R, nrot, T, C, st);
    case 8: return launch_ring<8>(R, nrot, T, C, st);
    case 12: return launch_ring<12>(R, nrot, T, C, st);
    case 16: return launch_ring<16>(R, nrot, T, C, st);
    case 24: return launch_ring<24>(R, nrot, T, C, st);
    default:
      set_error("fused build not instantiated for p = %d", T.p0);
      return VES3D_ERR_ARG;
  }
}

}  // namespace ves3d
