// FP64 kernels of the singular self-interaction build (plain form): coefficient
// rotation to every target, the pole-singular Stokes kernel, and the adjoint rotation
// that scatters the result into the per-vesicle self-matrix layout.
// Math: SphericalHarmonics<Real>::RotateAll / StokesSingularInteg_ / RotateTranspose
// (src/SphericalHarmonics.cc:363-541, 954-1180).
#include <cstdlib>

#include "common.cuh"
#include "kernels.h"

namespace ves3d {

// One CTA per (vesicle v, latitude rotation t); loops over the p0 longitude phases j, JB
// of them at a time (4, or fewer where the staging would not fit: p = 24).
// out[c'] = sum_b (P_j s)[perm_n[b]] * Mr[t][n][b][pos(c')],   n = degree(c').
// The blocks Mr[t][.] (mr_per_t doubles, contiguous for one t) are staged in shared memory.
// Outputs are formed in degree-major order (a warp's lanes share a degree: one loop length,
// broadcast inputs, consecutive block columns) and each thread forms its coefficient for
// JB longitudes at once, reusing every block element.
template <int JB>
__global__ void __launch_bounds__(256) k_rotate_all(const double* __restrict__ S, int p0, int mr_per_t, DevTables T,
                                                    double* __restrict__ R) {
  constexpr int kRaJ = JB;
  extern __shared__ double sm[];
  const int nc = p0 * (p0 + 2);
  double* sS = sm;
  double* sB = sm + 3 * nc;                                        // [kRaJ][3 nc]
  double* sM = sB + kRaJ * 3 * nc;
  double* sCs = sM + mr_per_t;                                     // cos_tab [2 p0]
  double* sSn = sCs + 2 * p0;                                      // sin_tab [2 p0]
  int* sMo = reinterpret_cast<int*>(sSn + 2 * p0);                 // mr_off of (t, n) - base [p0 + 1]
  int* sPo = sMo + (p0 + 1);                                       // perm_off [p0 + 2]
  short* sPc = reinterpret_cast<short*>(sPo + (p0 + 2));           // partner [nc]
  unsigned short* sPerm = reinterpret_cast<unsigned short*>(sPc + nc);  // perm [nc]
  unsigned char* sMs = reinterpret_cast<unsigned char*>(sPerm + nc);    // m | (is_sin << 7) [nc]
  unsigned char* sNd = sMs + nc;                                   // degree of degree-major position [nc]
  const int t = blockIdx.x;
  const long v = blockIdx.y;
  const int mbase = __ldg(T.mr_off + t * (p0 + 1));
  for (int i = threadIdx.x; i < 3 * nc; i += blockDim.x) sS[i] = S[v * 3 * nc + i];
  for (int i = threadIdx.x; i < mr_per_t; i += blockDim.x) sM[i] = __ldg(T.mr + mbase + i);
  for (int i = threadIdx.x; i < 2 * p0; i += blockDim.x) {
    sCs[i] = __ldg(T.cos_tab + i);
    sSn[i] = __ldg(T.sin_tab + i);
  }
  for (int i = threadIdx.x; i <= p0; i += blockDim.x) sMo[i] = __ldg(T.mr_off + t * (p0 + 1) + i) - mbase;
  for (int i = threadIdx.x; i <= p0 + 1; i += blockDim.x) sPo[i] = __ldg(T.perm_off + i);
  for (int c = threadIdx.x; c < nc; c += blockDim.x) {
    sPc[c] = (short)__ldg(T.partner + c);
    sPerm[c] = (unsigned short)__ldg(T.perm + c);
    sMs[c] = (unsigned char)(__ldg(T.m_of_coef + c) | (__ldg(T.is_sin + c) ? 0x80 : 0));
    const int n = __ldg(T.n_of_coef + c);
    sNd[__ldg(T.perm_off + n) + __ldg(T.pos_in_block + c)] = (unsigned char)n;
  }
  __syncthreads();
  for (int j0 = 0; j0 < p0; j0 += kRaJ) {
    const int nj = min(kRaJ, p0 - j0);
    for (int i = threadIdx.x; i < nj * 3 * nc; i += blockDim.x) {
      const int jj = i / (3 * nc), r = i - jj * 3 * nc;
      const int d = r / nc, c = r - d * nc;
      const int pc = sPc[c];
      double val;
      if (pc < 0) {
        val = sS[r];
      } else {
        const int ms = sMs[c];
        const int q = ((ms & 0x7f) * (j0 + jj)) % (2 * p0);
        const double cs = sCs[q], sn = sSn[q];
        val = (ms & 0x80) ? -sS[d * nc + pc] * sn + sS[r] * cs : sS[r] * cs + sS[d * nc + pc] * sn;
      }
      sB[jj * 3 * nc + r] = val;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * nc; i += blockDim.x) {
      const int d = i / nc, e = i - d * nc;  // e: degree-major position of the output
      const int n = sNd[e];
      const int po = sPo[n], bn = sPo[n + 1] - po, bp = e - po;
      const double* M = sM + sMo[n] + bp;
      const double* b = sB + d * nc;
      double acc[kRaJ];
#pragma unroll
      for (int q = 0; q < kRaJ; q++) acc[q] = 0.0;
      for (int k = 0; k < bn; k++) {
        const double m = M[k * bn];
        const int src = sPerm[po + k];
#pragma unroll
        for (int q = 0; q < kRaJ; q++) acc[q] = fma(b[q * 3 * nc + src], m, acc[q]);
      }
      const int c = sPerm[e];
#pragma unroll
      for (int q = 0; q < kRaJ; q++)
        if (q < nj) R[(((v * (p0 + 1) + t) * p0 + j0 + q) * 3 + d) * (long)nc + c] = acc[q];
    }
    __syncthreads();
  }
}

static int mr_per_t(const DevTables& T) { return T.mr_total / (T.p0 + 1); }

// One rotation of n_fun coefficient vectors: the grid point (latitude t, longitude j) of
// order p0 moved to the x = -1 pole, j in [0, 2 p0) (the step of RotateAll for one (t, j),
// src/SphericalHarmonics.cc:363-449: longitude phase P_j, then the per-degree blocks of
// MatRotate for latitude t). One CTA per function.
__global__ void __launch_bounds__(256) k_rotate_one(const double* __restrict__ S, int p0, int t, int j, DevTables T,
                                                    double* __restrict__ R) {
  extern __shared__ double sB[];  // phase-shifted coefficients [nc]
  const int nc = p0 * (p0 + 2);
  const long f = blockIdx.x;
  const double* s = S + f * nc;
  for (int c = threadIdx.x; c < nc; c += blockDim.x) {
    const int pc = __ldg(T.partner + c);
    if (pc < 0) {
      sB[c] = s[c];
    } else {
      const int q = (__ldg(T.m_of_coef + c) * j) % (2 * p0);
      const double cs = __ldg(T.cos_tab + q), sn = __ldg(T.sin_tab + q);
      sB[c] = __ldg(T.is_sin + c) ? -s[pc] * sn + s[c] * cs : s[c] * cs + s[pc] * sn;
    }
  }
  __syncthreads();
  for (int c = threadIdx.x; c < nc; c += blockDim.x) {
    const int n = __ldg(T.n_of_coef + c), bp = __ldg(T.pos_in_block + c);
    const int po = __ldg(T.perm_off + n), bn = __ldg(T.perm_off + n + 1) - po;
    const double* M = T.mr + __ldg(T.mr_off + t * (p0 + 1) + n);
    double acc = 0.0;
    for (int k = 0; k < bn; k++) acc = fma(sB[__ldg(T.perm + po + k)], __ldg(M + k * bn + bp), acc);
    R[f * nc + c] = acc;
  }
}

int launch_rotate_one(const double* S, long n_fun, int t, int j, const DevTables& T, double* R, cudaStream_t st) {
  if (n_fun <= 0) return VES3D_OK;
  const int nc = ncoef_(T.p0);
  k_rotate_one<<<(unsigned)n_fun, 256, nc * sizeof(double), st>>>(S, T.p0, t, j, T, R);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

int launch_rotate_all(const double* S, long nv, const DevTables& T, double* R, cudaStream_t st) {
  if (nv <= 0) return VES3D_OK;
  const int p0 = T.p0;
  const int mpt = mr_per_t(T);
  const size_t nc = ncoef_(p0);
  if (p0 > 127) {  // the on-chip tables hold orders and block positions in one byte
    set_error("rotation kernels support SH orders up to 127");
    return VES3D_ERR_ARG;
  }
  auto smem_of = [&](int jb) {
    return (((3 + 3 * (size_t)jb) * nc + mpt + 4 * p0) * sizeof(double) + (2 * p0 + 3) * sizeof(int) + nc * 4 + nc * 2 +
            15) / 16 * 16;
  };
  dim3 grid(p0 + 1, (unsigned)nv);
  const size_t cap = 227 * 1024;
  if (smem_of(4) <= cap) {
    VES3D_CK(cudaFuncSetAttribute(k_rotate_all<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_of(4)));
    k_rotate_all<4><<<grid, 256, smem_of(4), st>>>(S, p0, mpt, T, R);
  } else if (smem_of(2) <= cap) {
    VES3D_CK(cudaFuncSetAttribute(k_rotate_all<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_of(2)));
    k_rotate_all<2><<<grid, 256, smem_of(2), st>>>(S, p0, mpt, T, R);
  } else if (smem_of(1) <= cap) {
    VES3D_CK(cudaFuncSetAttribute(k_rotate_all<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_of(1)));
    k_rotate_all<1><<<grid, 256, smem_of(1), st>>>(S, p0, mpt, T, R);
  } else {
    set_error("RotateAll: the rotation blocks of p = %d do not fit in shared memory", p0);
    return VES3D_ERR_ARG;
  }
  VES3D_LAUNCHED();
  return VES3D_OK;
}

// One CTA per rotated surface. Pole targets from the m = 0 block (SHC2Pole, :325-360),
// then for every upsampled source point s (latitude j0) and pole t, with r = target - source,
// n = X_theta x X_phi (area-weighted outward normal), qs = SingularWeights(p1)[t ? j0 : p1 - j0]
// and |r|^-1 := 0 when |r|^2 <= 2^-52 (src/SphericalHarmonics.cc:989-1068):
//   single layer  a1 + r_a r_b a2 with a1 = qs |n| / (8 pi |r|), a2 = a1 / |r|^2
//   double layer  r_a r_b q      with q  = 3 qs (n . r) / (4 pi |r|^5)
template <bool DL>
__global__ void __launch_bounds__(256) k_singular(const double* __restrict__ X, const double* __restrict__ Xt,
                                                  const double* __restrict__ Xp, const double* __restrict__ R,
                                                  int p0, int p1, const double* __restrict__ qp,
                                                  const double* __restrict__ sw, double* __restrict__ K) {
  __shared__ double trg[6];
  const long rot = blockIdx.x;
  const int nc = p0 * (p0 + 2), M1 = 2 * p1 * (p1 + 1);
  if (threadIdx.x < 6) {
    const int c = threadIdx.x >> 1, t = threadIdx.x & 1;
    const double* r = R + (rot * 3 + c) * nc;
    double s = 0.0;
    for (int n = 0; n <= p0; n++) s += r[n] * __ldg(qp + t * (p0 + 1) + n);
    trg[c * 2 + t] = s;
  }
  __syncthreads();
  const double eps = 2.220446049250313e-16;
  const double* x = X + rot * 3 * M1;
  const double* xt = Xt + rot * 3 * M1;
  const double* xp = Xp + rot * 3 * M1;
  double* k = K + rot * 12 * (long)M1;
  for (int s = threadIdx.x; s < M1; s += blockDim.x) {
    const int j0 = s / (2 * p1);
    const double px = x[s], py = x[M1 + s], pz = x[2 * M1 + s];
    const double ax = xt[s], ay = xt[M1 + s], az = xt[2 * M1 + s];
    const double bx = xp[s], by = xp[M1 + s], bz = xp[2 * M1 + s];
    const double nx = ay * bz - az * by, ny = az * bx - ax * bz, nz = ax * by - ay * bx;
    const double area = DL ? 0.0 : sqrt(nx * nx + ny * ny + nz * nz);
#pragma unroll
    for (int t = 0; t < 2; t++) {
      const double dx = trg[t] - px, dy = trg[2 + t] - py, dz = trg[4 + t] - pz;
      const double r2 = dx * dx + dy * dy + dz * dz;
      double rinv = 1.0 / sqrt(r2);
      if (r2 <= eps) rinv = 0.0;
      const double rinv2 = rinv * rinv;
      double* kt = k + (long)t * 6 * M1;
      if (DL) {
        const double q = kDl * __ldg(sw + (t ? j0 : p1 - j0)) * (nx * dx + ny * dy + nz * dz) * (rinv2 * rinv2 * rinv);
        kt[s] = dx * dx * q;
        kt[M1 + s] = dx * dy * q;
        kt[2 * M1 + s] = dx * dz * q;
        kt[3 * M1 + s] = dy * dy * q;
        kt[4 * M1 + s] = dy * dz * q;
        kt[5 * M1 + s] = dz * dz * q;
      } else {
        const double a1 = kInv8Pi * __ldg(sw + (t ? j0 : p1 - j0)) * area * rinv;
        const double a2 = a1 * rinv2;
        kt[s] = a1 + dx * dx * a2;
        kt[M1 + s] = dx * dy * a2;
        kt[2 * M1 + s] = dx * dz * a2;
        kt[3 * M1 + s] = a1 + dy * dy * a2;
        kt[4 * M1 + s] = dy * dz * a2;
        kt[5 * M1 + s] = a1 + dz * dz * a2;
      }
    }
  }
}

int launch_singular_sl(const double* X, const double* Xt, const double* Xp, const double* R, long nrot,
                       const DevTables& T, double* K, cudaStream_t st) {
  if (nrot <= 0) return VES3D_OK;
  k_singular<false><<<(unsigned)nrot, 256, 0, st>>>(X, Xt, Xp, R, T.p0, T.p1, T.qp, T.sing_w, K);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

int launch_singular_dl(const double* X, const double* Xt, const double* Xp, const double* R, long nrot,
                       const DevTables& T, double* K, cudaStream_t st) {
  if (nrot <= 0) return VES3D_OK;
  k_singular<true><<<(unsigned)nrot, 256, 0, st>>>(X, Xt, Xp, R, T.p0, T.p1, T.qp, T.sing_w, K);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

// One CTA per (vesicle, latitude rotation t), looping over (pole, component) and over
// chunks of jb longitude rotations. For each input vector a (coefficients of one
// (t, j, pole, comp) function): b = Mr_t^T a per degree block, then the inverse phase
// P_j^T, then scatter into SL3[v][c_in][k][c_out][grid] at grid (t, j) for pole 0 and
// (p0 - t, p0 + j) for pole 1, for both (c_in, c_out) orders of the symmetric component.
// The blocks Mr[t][.] are staged in shared memory; each input vector is stored in
// degree-major order (coefficients of one degree contiguous) so the block products read
// contiguous data, and every thread forms one coefficient for 4 rotations at a time.
constexpr int kRtJ = 4;

__global__ void __launch_bounds__(256) k_rotate_transpose_scatter(const double* __restrict__ C, int p0, int jb,
                                                                  int mr_per_t, DevTables T,
                                                                  double* __restrict__ SL3) {
  extern __shared__ double sm[];
  const int nc = p0 * (p0 + 2), ng = 2 * p0 * (p0 + 1);
  const int lda = nc + 2;      // row padding against bank conflicts between rotations
  double* sA = sm;             // jb * lda, degree-major
  double* sB = sm + jb * lda;  // jb * lda, coefficient order
  double* sM = sm + 2 * jb * lda;
  const int t = blockIdx.x;
  const long v = blockIdx.y;
  const int mbase = __ldg(T.mr_off + t * (p0 + 1));
  for (int i = threadIdx.x; i < mr_per_t; i += blockDim.x) sM[i] = __ldg(T.mr + mbase + i);
  for (int pole = 0; pole < 2; pole++) {
    for (int comp = 0; comp < 6; comp++) {
      for (int j0 = 0; j0 < p0; j0 += jb) {
        const int nj = min(jb, p0 - j0);
        __syncthreads();
        for (int i = threadIdx.x; i < nj * nc; i += blockDim.x) {
          const int jj = i / nc, c = i % nc;
          const int n = __ldg(T.n_of_coef + c);
          const int dm = __ldg(T.perm_off + n) + __ldg(T.pos_in_block + c);
          sA[jj * lda + dm] = C[((((v * (p0 + 1) + t) * p0 + j0 + jj) * 2 + pole) * 6 + comp) * (long)nc + c];
        }
        __syncthreads();
        const int njq = (nj + kRtJ - 1) / kRtJ;
        for (int i = threadIdx.x; i < njq * nc; i += blockDim.x) {
          const int c = i % nc, jq = i / nc;
          const int n = __ldg(T.n_of_coef + c), b = __ldg(T.pos_in_block + c);
          const int po = __ldg(T.perm_off + n), bn = __ldg(T.perm_off + n + 1) - po;
          const double* M = sM + (__ldg(T.mr_off + t * (p0 + 1) + n) - mbase) + b * bn;
          const double* a = sA + jq * kRtJ * lda + po;
          double acc[kRtJ];
#pragma unroll
          for (int q = 0; q < kRtJ; q++) acc[q] = 0.0;
          for (int k = 0; k < bn; k++) {
            const double m = M[k];
#pragma unroll
            for (int q = 0; q < kRtJ; q++) acc[q] = fma(a[q * lda + k], m, acc[q]);
          }
#pragma unroll
          for (int q = 0; q < kRtJ; q++)
            if (jq * kRtJ + q < nj) sB[(jq * kRtJ + q) * lda + c] = acc[q];
        }
        __syncthreads();
        // inverse phase and scatter; consecutive threads take consecutive j for coalescing
        for (int i = threadIdx.x; i < nj * nc; i += blockDim.x) {
          const int jj = i % nj, c = i / nj;
          const int j = j0 + jj;
          const int pc = __ldg(T.partner + c);
          double val;
          if (pc < 0) {
            val = sB[jj * lda + c];
          } else {
            const int q = (__ldg(T.m_of_coef + c) * j) % (2 * p0);
            const double cs = __ldg(T.cos_tab + q), sn = __ldg(T.sin_tab + q);
            if (!__ldg(T.is_sin + c)) {
              val = sB[jj * lda + c] * cs - sB[jj * lda + pc] * sn;
            } else {
              val = sB[jj * lda + pc] * sn + sB[jj * lda + c] * cs;
            }
          }
          const int grid = pole == 0 ? t * 2 * p0 + j : (p0 - t) * 2 * p0 + p0 + j;
          const int cin = comp < 3 ? 0 : (comp < 5 ? 1 : 2), cout = comp < 3 ? comp : (comp < 5 ? comp - 2 : 2);  // (0,0) (0,1) (0,2) (1,1) (1,2) (2,2)
          SL3[(((v * 3 + cin) * nc + c) * 3 + cout) * (long)ng + grid] = val;
          if (cin != cout) SL3[(((v * 3 + cout) * nc + c) * 3 + cin) * (long)ng + grid] = val;
        }
      }
    }
  }
}

// The rotate-transpose per (degree, order) item, in the arithmetic type TV: one CTA per
// (latitude rotation t, vesicle v); for each pole and symmetric component the P longitude
// rows of C are staged in degree-major order, then each thread takes one item (degree n,
// order m): the coefficient of cos(m phi) and its sin(m phi) partner (one coefficient for
// m = 0 and m = P), and forms for all P rows the rotation back
//     B[row][po + b] = sum_k A[row][po + k] Mr_{t,n}[b][k]
// at its two positions b, then the inverse longitude phase of the pair in registers and
// the P consecutive grid values of each coefficient as 16-byte vector stores into the
// self-matrix grid SL3, laid out as the other forms'. A thread's rows share the staged
// inputs (broadcast to the lanes of its degree) and its two rotation rows: 18 shared loads
// per 32 FMAs at p = 16. TV = float in the mixed form (C is FP32 after the tensor-core
// build, FP64 after the FP64 ring and rounded when staged; the FP32 grid goes to the FP32
// Grid2SHC); TV = double in the FP64 form at p = 16 (the DMMA kernel below keeps the
// other orders up to 16).
// The 16-byte vector of 16 / sizeof(T) values starting at o[i] (destinations 16-byte aligned).
__device__ __forceinline__ float4 vec16(const float* o, int i) { return make_float4(o[i], o[i + 1], o[i + 2], o[i + 3]); }
__device__ __forceinline__ double2 vec16(const double* o, int i) { return make_double2(o[i], o[i + 1]); }

template <int P, typename TV>
struct RtItemCfg {
  static constexpr int NI = (P + 1) * (P + 2) / 2;  // items (n, m <= n), degree-major: n (n + 1) / 2 + m
  static constexpr int NT = (NI + 31) / 32 * 32;   // one item per thread
  // CTAs per SM the registers are sized for (shared memory allows 4 in FP32, 2 in FP64 at p = 16)
  static constexpr int MINB = P == 16 ? (sizeof(TV) == 4 ? 4 : 2) : 1;
};

template <int P, typename TC, typename TV>
__global__ void __launch_bounds__(RtItemCfg<P, TV>::NT, RtItemCfg<P, TV>::MINB)
    k_rotate_transpose_item(const TC* __restrict__ C, int mr_per_t, DevTables T, TV* __restrict__ SL3) {
  constexpr int nc = P * (P + 2), ng = 2 * P * (P + 1), lda = nc + 1;
  constexpr int NI = RtItemCfg<P, TV>::NI, NT = RtItemCfg<P, TV>::NT;
  extern __shared__ __align__(16) unsigned char smraw[];
  TV* sA = reinterpret_cast<TV*>(smraw);  // [P rows][lda], degree-major
  TV* sM = sA + P * lda;                  // blocks of degree n at sMo[n], rows of bn | 1
  const int msz = mr_per_t + (P + 1) * 2 * P;  // (upper bound of the padded size)
  TV* sCs = sM + msz;                     // cos_tab [2P]
  TV* sSn = sCs + 2 * P;                  // sin_tab [2P]
  int* sMo = reinterpret_cast<int*>(sSn + 2 * P);                        // [P + 2] padded block offsets
  unsigned short* sDm = reinterpret_cast<unsigned short*>(sMo + P + 2);  // degree-major position [nc]
  short* sI0 = reinterpret_cast<short*>(sDm + nc);                       // cos (or single) coefficient [NI]
  short* sI1 = sI0 + NI;                                                 // its sin partner or -1 [NI]
  const int t = blockIdx.x;
  const long v = blockIdx.y;
  const int tid = threadIdx.x;
  if (tid == 0) {
    int o = 0;
    for (int n = 0; n <= P; n++) {
      sMo[n] = o;
      const int bn = __ldg(T.perm_off + n + 1) - __ldg(T.perm_off + n);
      o += bn * (bn | 1);
    }
    sMo[P + 1] = o;
  }
  for (int i = tid; i < NI; i += NT) sI0[i] = sI1[i] = -1;
  for (int i = tid; i < 2 * P; i += NT) {
    sCs[i] = (TV)__ldg(T.cos_tab + i);
    sSn[i] = (TV)__ldg(T.sin_tab + i);
  }
  __syncthreads();
  for (int c = tid; c < nc; c += NT) {
    const int n = __ldg(T.n_of_coef + c), item = n * (n + 1) / 2 + __ldg(T.m_of_coef + c);
    sDm[c] = (unsigned short)(__ldg(T.perm_off + n) + __ldg(T.pos_in_block + c));
    if (__ldg(T.is_sin + c))
      sI1[item] = (short)c;
    else
      sI0[item] = (short)c;
  }
  // the rotation blocks of this t, FP32, rows padded to bn | 1
  for (int n = 0; n <= P; n++) {
    const int bn = __ldg(T.perm_off + n + 1) - __ldg(T.perm_off + n);
    const double* M = T.mr + __ldg(T.mr_off + t * (P + 1) + n);
    for (int i = tid; i < bn * bn; i += NT) {
      const int b = i / bn, k = i - b * bn;
      sM[sMo[n] + b * (bn | 1) + k] = (TV)__ldg(M + i);
    }
  }
  __syncthreads();
  // this thread's item
  int n = 0;
  while ((n + 1) * (n + 2) / 2 <= tid && n < P) n++;
  const bool active = tid < NI && sI0[tid] >= 0;  // (every (n, m <= n) has its cos coefficient)
  const int m = active ? tid - n * (n + 1) / 2 : 0;
  const int c0 = active ? sI0[tid] : 0, c1 = active ? sI1[tid] : -1;
  const int po = __ldg(T.perm_off + n), bn = __ldg(T.perm_off + n + 1) - po;
  const TV* M0 = active ? sM + sMo[n] + (sDm[c0] - po) * (bn | 1) : sM;
  const TV* M1 = c1 >= 0 ? sM + sMo[n] + (sDm[c1] - po) * (bn | 1) : M0;
  for (int pole = 0; pole < 2; pole++) {
    const int grid0 = pole == 0 ? t * 2 * P : (P - t) * 2 * P + P;
    for (int comp = 0; comp < 6; comp++) {
      __syncthreads();
      // stage: A[j][dm(c)] = C[v][t][j][pole][comp][c], eight loads in flight per thread
      for (int i0 = tid; i0 < P * nc; i0 += NT * 8) {
        TV val[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int i = i0 + u * NT;
          if (i < P * nc) {
            const int j = i / nc, c = i - j * nc;
            val[u] = (TV)C[((((v * (P + 1) + t) * P + j) * 2 + pole) * 6 + comp) * (long)nc + c];
          }
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int i = i0 + u * NT;
          if (i < P * nc) {
            const int j = i / nc, c = i - j * nc;
            sA[j * lda + sDm[c]] = val[u];
          }
        }
      }
      __syncthreads();
      if (!active) continue;
      TV acc0[P], acc1[P];
#pragma unroll
      for (int j = 0; j < P; j++) acc0[j] = acc1[j] = TV(0);
      const TV* a = sA + po;
      for (int k = 0; k < bn; k++) {
        const TV m0 = M0[k], m1 = M1[k];
#pragma unroll
        for (int j = 0; j < P; j++) {
          const TV x = a[j * lda + k];
          acc0[j] = fma(x, m0, acc0[j]);
          acc1[j] = fma(x, m1, acc1[j]);
        }
      }
      // inverse longitude phase of the pair: cos row c0, sin row c1
      if (c1 >= 0) {
#pragma unroll
        for (int j = 0; j < P; j++) {
          const int q = (m * j) % (2 * P);
          const TV cs = sCs[q], sn = sSn[q];
          const TV x0 = acc0[j], x1 = acc1[j];
          acc0[j] = fma(-x1, sn, x0 * cs);
          acc1[j] = fma(x0, sn, x1 * cs);
        }
      }
      // symmetric component -> (c_in, c_out): (0,0) (0,1) (0,2) (1,1) (1,2) (2,2)
      const int cin = comp < 3 ? 0 : (comp < 5 ? 1 : 2), cout = comp < 3 ? comp : (comp < 5 ? comp - 2 : 2);
      auto put = [&](int c, const TV* o) {
        TV* d0 = SL3 + (((v * 3 + cin) * nc + c) * 3 + cout) * (long)ng + grid0;
        TV* d1 = SL3 + (((v * 3 + cout) * nc + c) * 3 + cin) * (long)ng + grid0;
        using V = decltype(vec16(o, 0));
        constexpr int W = 16 / sizeof(TV);
#pragma unroll
        for (int q = 0; q < P / W; q++) {
          const V w = vec16(o, W * q);
          reinterpret_cast<V*>(d0)[q] = w;
          if (cin != cout) reinterpret_cast<V*>(d1)[q] = w;
        }
      };
      put(c0, acc0);
      if (c1 >= 0) put(c1, acc1);
    }
  }
}

template <typename TV>
static size_t rt_item_smem(int p0, int mpt) {
  const int nc = p0 * (p0 + 2), lda = nc + 1, ni = (p0 + 1) * (p0 + 2) / 2;
  const size_t fl = (size_t)p0 * lda + mpt + (size_t)(p0 + 1) * 2 * p0 + 4 * p0;
  return fl * sizeof(TV) + (size_t)(p0 + 2) * sizeof(int) + (size_t)nc * 2 + (size_t)ni * 4 + 16;
}

template <int P, typename TC, typename TV = float>
static int launch_rt_item(const TC* C, long nv, const DevTables& T, TV* SL3, cudaStream_t st) {
  const int mpt = mr_per_t(T);
  dim3 grid(P + 1, (unsigned)nv);
  const size_t smem = rt_item_smem<TV>(P, mpt);  // about 48 KB at p = 16 (four CTAs per SM), 149 KB at p = 24
  VES3D_CK(cudaFuncSetAttribute(k_rotate_transpose_item<P, TC, TV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem));
  k_rotate_transpose_item<P, TC, TV><<<grid, RtItemCfg<P, TV>::NT, smem, st>>>(C, mpt, T, SL3);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

int launch_rotate_transpose_f32(const float* C, long nv, const DevTables& T, float* SL3, cudaStream_t st) {
  if (nv <= 0) return VES3D_OK;
  // the FP32 results come from the tensor-core build, which is laid out for p = 16 only
  if (T.p0 != 16) {
    set_error("internal: FP32 rotate-transpose at p = %d (built for p = 16)", T.p0);
    return VES3D_ERR_ARG;
  }
  return launch_rt_item<16>(C, nv, T, SL3, st);
}

bool rotate_transpose_f32_from_f64_supported(int p0) { return p0 == 12 || p0 == 24; }

int launch_rotate_transpose_f32(const double* C, long nv, const DevTables& T, float* SL3, cudaStream_t st) {
  if (nv <= 0) return VES3D_OK;
  switch (T.p0) {
    case 12: return launch_rt_item<12>(C, nv, T, SL3, st);
    case 24: return launch_rt_item<24>(C, nv, T, SL3, st);
    default: break;
  }
  set_error("internal: FP32 rotate-transpose of FP64 results at p = %d (built for p in {12, 24})", T.p0);
  return VES3D_ERR_ARG;
}

// VES3D_TC_ROTATE=0 selects the CUDA-core form of the rotate-transpose (for comparison).
static bool tc_rotate_disabled() {
  static const bool off = [] {
    const char* e = getenv("VES3D_TC_ROTATE");
    return e && e[0] == '0';
  }();
  return off;
}

constexpr int kRtMaxK = 8;  // K steps of 4: rotation blocks up to 32 wide (p0 <= 16)

__device__ __forceinline__ void dmma_rt(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// Row stride >= n with stride = 4 (mod 16) doubles: conflict-free m8n8k4 A fragments.
__host__ __device__ constexpr int pad4_16(int n) { return ((n + 11) / 16) * 16 + 4; }

// RotateTranspose + inverse phase + Rearrange on the FP64 tensor cores. One CTA per
// (latitude rotation t, vesicle v); rows are (pole, component, longitude j), processed in
// blocks of cb components x p0 longitudes. A block's coefficients are staged degree-major
// in shared memory; for every degree n the rotation back is one GEMM
//     Out[row][b] = sum_k In[row][po(n) + k] * M_{t,n}[b][k]       (b, k < bn)
// on mma.sync m8n8k4 (A = In from shared memory, B = M from the L1/L2-resident table,
// masked to the block), written back in place after a barrier; reads of the K padding
// land in the next degree's (finite) columns and meet zeros in B. Then the longitude
// phase is undone and the values are scattered into the self-matrix grid layout, as in
// k_rotate_transpose_scatter.
__global__ void __launch_bounds__(256, 2) k_rotate_transpose_tc(const double* __restrict__ C, int p0, int cb, int ldi,
                                                                DevTables T, double* __restrict__ SL3) {
  extern __shared__ __align__(16) double sm[];
  const int nc = p0 * (p0 + 2), ng = 2 * p0 * (p0 + 1);
  const int rows = cb * p0, rows8 = (rows + 7) & ~7;
  double* sIn = sm;                                                        // rows8 x ldi
  double* sCs = sm + (size_t)rows8 * ldi;                                  // cos_tab [2 p0]
  double* sSn = sCs + 2 * p0;                                              // sin_tab [2 p0]
  unsigned short* sDm = reinterpret_cast<unsigned short*>(sSn + 2 * p0);   // degree-major position [nc]
  short* sPc = reinterpret_cast<short*>(sDm + nc);                        // partner (or -1) [nc]
  unsigned char* sMs = reinterpret_cast<unsigned char*>(sPc + nc);        // m | (is_sin << 7) [nc]
  const int t = blockIdx.x;
  const long v = blockIdx.y;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int grow = lane >> 2, gcol = lane & 3;
  // per-coefficient tables of the phase / scatter step, on chip (the L1 left beside the
  // staging buffer is small, and every element needs them)
  for (int c = tid; c < nc; c += 256) {
    sDm[c] = (unsigned short)(__ldg(T.perm_off + __ldg(T.n_of_coef + c)) + __ldg(T.pos_in_block + c));
    sPc[c] = (short)__ldg(T.partner + c);
    sMs[c] = (unsigned char)(__ldg(T.m_of_coef + c) | (__ldg(T.is_sin + c) ? 0x80 : 0));
  }
  for (int i = tid; i < 2 * p0; i += 256) {
    sCs[i] = __ldg(T.cos_tab + i);
    sSn[i] = __ldg(T.sin_tab + i);
  }
  // zero the K padding of every row and the padding rows once (never overwritten)
  for (int i = tid; i < rows8 * ldi; i += 256) {
    const int r = i / ldi, col = i - r * ldi;
    if (r >= rows || col >= nc) sIn[i] = 0.0;
  }
  const int mtiles = rows8 / 8;
  for (int pole = 0; pole < 2; pole++) {
    for (int comp0 = 0; comp0 < 6; comp0 += cb) {
      __syncthreads();
      // stage: In[(cc, j)][dm(c)] = C[v][t][j][pole][comp0 + cc][c], eight loads in flight
      // per thread before the shared-memory stores
      for (int i0 = tid; i0 < rows * nc; i0 += 256 * 8) {
        double val[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int i = i0 + u * 256;
          if (i < rows * nc) {
            const int r = i / nc, c = i - r * nc;
            const int cc = r / p0, j = r - cc * p0;
            val[u] = C[((((v * (p0 + 1) + t) * p0 + j) * 2 + pole) * 6 + comp0 + cc) * (long)nc + c];
          }
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int i = i0 + u * 256;
          if (i < rows * nc) {
            const int r = i / nc, c = i - r * nc;
            sIn[r * ldi + sDm[c]] = val[u];
          }
        }
      }
      __syncthreads();
      for (int n = 0; n <= p0; n++) {
        const int po = __ldg(T.perm_off + n), bn = __ldg(T.perm_off + n + 1) - po;
        const double* M = T.mr + __ldg(T.mr_off + t * (p0 + 1) + n);
        const int ntiles = (bn + 7) / 8, ksteps = (bn + 3) / 4;
        const int nitems = mtiles * ntiles;
        // at most 3 items per warp held in registers across the barrier (nitems <= 24
        // for rows8 <= 48 and bn <= 32; larger problems loop in rounds)
        for (int base = 0; base < nitems; base += 24) {
          double acc[3][2];
          int item[3];
#pragma unroll
          for (int q = 0; q < 3; q++) {
            item[q] = base + warp + 8 * q;
            acc[q][0] = acc[q][1] = 0.0;
            if (item[q] < nitems) {
              const int mt = item[q] / ntiles, nt = item[q] - mt * ntiles;
              const double* a = sIn + (mt * 8 + grow) * ldi + po + gcol;
              const int nn = nt * 8 + grow;
              // B fragments first (independent loads in flight together), then the MMAs
              double bv[kRtMaxK];
#pragma unroll
              for (int ks = 0; ks < kRtMaxK; ks++) {
                const int kk = ks * 4 + gcol;
                bv[ks] = (ks < ksteps && nn < bn && kk < bn) ? __ldg(M + nn * bn + kk) : 0.0;
              }
#pragma unroll
              for (int ks = 0; ks < kRtMaxK; ks++)
                if (ks < ksteps) dmma_rt(acc[q][0], acc[q][1], a[ks * 4], bv[ks]);
            }
          }
          __syncthreads();
#pragma unroll
          for (int q = 0; q < 3; q++) {
            if (item[q] < nitems) {
              const int mt = item[q] / ntiles, nt = item[q] - mt * ntiles;
              const int row = mt * 8 + grow, col = nt * 8 + 2 * gcol;
              if (row < rows) {
                if (col < bn) sIn[row * ldi + po + col] = acc[q][0];
                if (col + 1 < bn) sIn[row * ldi + po + col + 1] = acc[q][1];
              }
            }
          }
          __syncthreads();
        }
      }
      // inverse phase and scatter; consecutive threads take consecutive j
      for (int i = tid; i < rows * nc; i += 256) {
        const int j = i % p0, rest = i / p0;
        const int c = rest % nc, cc = rest / nc;
        const double* in = sIn + (cc * p0 + j) * ldi;
        const int pc = sPc[c];
        double val;
        if (pc < 0) {
          val = in[sDm[c]];
        } else {
          const int ms = sMs[c];
          const int q = ((ms & 0x7f) * j) % (2 * p0);
          const double cs = sCs[q], sn = sSn[q];
          if (!(ms & 0x80))
            val = in[sDm[c]] * cs - in[sDm[pc]] * sn;
          else
            val = in[sDm[pc]] * sn + in[sDm[c]] * cs;
        }
        const int grid = pole == 0 ? t * 2 * p0 + j : (p0 - t) * 2 * p0 + p0 + j;
        const int comp = comp0 + cc;
        const int cin = comp < 3 ? 0 : (comp < 5 ? 1 : 2), cout = comp < 3 ? comp : (comp < 5 ? comp - 2 : 2);  // (0,0) (0,1) (0,2) (1,1) (1,2) (2,2)
        SL3[(((v * 3 + cin) * nc + c) * 3 + cout) * (long)ng + grid] = val;
        if (cin != cout) SL3[(((v * 3 + cout) * nc + c) * 3 + cin) * (long)ng + grid] = val;
      }
    }
  }
}

int launch_rotate_transpose_scatter(const double* C, long nv, const DevTables& T, double* SL3, cudaStream_t st) {
  if (nv <= 0) return VES3D_OK;
  const int p0 = T.p0, nc = ncoef_(p0);
  // p = 16: the per-item kernel in FP64 (5.8 ms per 512-vesicle build against 9.5 ms for the
  // DMMA form below, which keeps the other orders up to 16)
  if (p0 == 16 && !tc_rotate_disabled()) return launch_rt_item<16, double, double>(C, nv, T, SL3, st);
  {
    // tensor-core form: the largest component block (3, 2 or 1 components x p0 rows)
    // whose staging fits two CTAs per SM; 6 must be a multiple of the block
    const int ldi = pad4_16(nc + 3);
    for (int cb : {3, 2, 1}) {
      const int rows8 = ((cb * p0) + 7) & ~7;
      const size_t smem = ((size_t)rows8 * ldi + 4 * p0) * sizeof(double) + ((size_t)nc * 5 + 15) / 16 * 16;
      if (p0 <= 16 && smem <= 113 * 1024 && !tc_rotate_disabled()) {
        VES3D_CK(cudaFuncSetAttribute(k_rotate_transpose_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        dim3 grid(p0 + 1, (unsigned)nv);
        k_rotate_transpose_tc<<<grid, 256, smem, st>>>(C, p0, cb, ldi, T, SL3);
        VES3D_LAUNCHED();
        return VES3D_OK;
      }
    }
  }
  const int mpt = mr_per_t(T);
  // two CTAs per SM: keep shared memory under ~110 KB; whole groups of kRtJ rotations
  long budget = (110 * 1024) / (long)sizeof(double) - mpt;
  int jb = (int)(budget / (2 * (long)(nc + 2)));
  jb = (jb / kRtJ) * kRtJ;
  if (jb > p0) jb = ((p0 + kRtJ - 1) / kRtJ) * kRtJ;
  if (jb < kRtJ) jb = kRtJ;
  size_t smem = ((size_t)2 * jb * (nc + 2) + mpt) * sizeof(double);
  if (smem > 48 * 1024)
    VES3D_CK(cudaFuncSetAttribute(k_rotate_transpose_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(p0 + 1, (unsigned)nv);
  k_rotate_transpose_scatter<<<grid, 256, smem, st>>>(C, p0, jb, mpt, T, SL3);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

// V[v][col] = sum_row F[v][row] * SL[v][row][col]; one thread per output column.
template <bool ACC>
__global__ void __launch_bounds__(128) k_self_gemv(const double* __restrict__ F, const double* __restrict__ SL,
                                                   int n, double* __restrict__ V) {
  extern __shared__ double sF[];
  const long v = blockIdx.y;
  for (int i = threadIdx.x; i < n; i += blockDim.x) sF[i] = F[v * n + i];
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= n) return;
  const double* M = SL + v * (long)n * n + col;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int r = 0;
  for (; r + 4 <= n; r += 4) {
    s0 = fma(sF[r], __ldg(M + (long)r * n), s0);
    s1 = fma(sF[r + 1], __ldg(M + (long)(r + 1) * n), s1);
    s2 = fma(sF[r + 2], __ldg(M + (long)(r + 2) * n), s2);
    s3 = fma(sF[r + 3], __ldg(M + (long)(r + 3) * n), s3);
  }
  for (; r < n; r++) s0 = fma(sF[r], __ldg(M + (long)r * n), s0);
  const double sum = (s0 + s1) + (s2 + s3);
  V[v * n + col] = ACC ? V[v * n + col] + sum : sum;
}

// Several density vectors per vesicle at once (batched operator applications):
// V[q nv + v][col] = sum_row F[q nv + v][row] SL[v][row][col], q < nvec; every SL column is
// read once for all nvec vectors (the single-vector form reads it per vector).
constexpr int kGemvMaxVec = 8;
template <bool ACC>
__global__ void __launch_bounds__(128) k_self_gemv_multi(const double* __restrict__ F, const double* __restrict__ SL,
                                                         long nv, int nvec, int n, double* __restrict__ V) {
  extern __shared__ double sF[];  // [nvec][n]
  const long v = blockIdx.y;
  for (int i = threadIdx.x; i < nvec * n; i += blockDim.x) {
    const int q = i / n, r = i - q * n;
    sF[i] = F[((long)q * nv + v) * n + r];
  }
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= n) return;
  const double* M = SL + v * (long)n * n + col;
  double acc[kGemvMaxVec];
#pragma unroll
  for (int q = 0; q < kGemvMaxVec; q++) acc[q] = 0.0;
  for (int r = 0; r < n; r++) {
    const double m = __ldg(M + (long)r * n);
#pragma unroll
    for (int q = 0; q < kGemvMaxVec; q++)
      if (q < nvec) acc[q] = fma(sF[q * n + r], m, acc[q]);
  }
#pragma unroll
  for (int q = 0; q < kGemvMaxVec; q++)
    if (q < nvec) {
      double* o = V + ((long)q * nv + v) * n + col;
      *o = ACC ? *o + acc[q] : acc[q];
    }
}

int launch_self_gemv_multi(const double* F, const double* SL, long nv, int nvec, int n, double* V, cudaStream_t st,
                           bool accumulate) {
  if (nv <= 0 || nvec <= 0) return VES3D_OK;
  if (nvec > kGemvMaxVec) {
    set_error("launch_self_gemv_multi: at most %d vectors", kGemvMaxVec);
    return VES3D_ERR_ARG;
  }
  dim3 grid((n + 127) / 128, (unsigned)nv);
  const size_t smem = (size_t)nvec * n * sizeof(double);
  if (accumulate) {
    if (smem > 48 * 1024)
      VES3D_CK(cudaFuncSetAttribute(k_self_gemv_multi<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_self_gemv_multi<true><<<grid, 128, smem, st>>>(F, SL, nv, nvec, n, V);
  } else {
    if (smem > 48 * 1024)
      VES3D_CK(cudaFuncSetAttribute(k_self_gemv_multi<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_self_gemv_multi<false><<<grid, 128, smem, st>>>(F, SL, nv, nvec, n, V);
  }
  VES3D_LAUNCHED();
  return VES3D_OK;
}

int launch_self_gemv(const double* F, const double* SL, long nv, int n, double* V, cudaStream_t st, bool accumulate) {
  if (nv <= 0) return VES3D_OK;
  dim3 grid((n + 127) / 128, (unsigned)nv);
  size_t smem = (size_t)n * sizeof(double);
  if (accumulate) {
    if (smem > 48 * 1024)
      VES3D_CK(cudaFuncSetAttribute(k_self_gemv<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_self_gemv<true><<<grid, 128, smem, st>>>(F, SL, n, V);
  } else {
    if (smem > 48 * 1024)
      VES3D_CK(cudaFuncSetAttribute(k_self_gemv<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_self_gemv<false><<<grid, 128, smem, st>>>(F, SL, n, V);
  }
  VES3D_LAUNCHED();
  return VES3D_OK;
}

}  // namespace ves3d
