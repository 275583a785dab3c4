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
template <int P0>
__global__ void __launch_bounds__(256, 2) k_build_ring(const double* __restrict__ R, DevTables T,
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
      const double area = n2 * rsqrt_f64(n2);  // |X_theta x X_phi| > 0 on the upsampled grid
#pragma unroll
      for (int t = 0; t < 2; t++) {
        const double dx = trg[t] - px, dy = trg[2 + t] - py, dz = trg[4 + t] - pz;
        const double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_f64(r2);
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
  const long grid = std::min(nrot, (long)nsm * ring_ctas_per_sm());
  k_build_ring<P0><<<(unsigned)grid, 256, G::SMEM, st>>>(R, T, C, nrot);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

bool fused_build_supported(int p0, int p1) {
  if (p1 != 2 * p0) return false;
  // the tensor-core tiling needs 2 p0 % 8 == 0 and 4 p0 % 16 == 0
  switch (p0) {
    case 4: case 8: case 12: case 16: return true;
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
    default:
      set_error("fused build not instantiated for p = %d", T.p0);
      return VES3D_ERR_ARG;
  }
}

}  // namespace ves3d
