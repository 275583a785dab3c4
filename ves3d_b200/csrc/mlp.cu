// Small multilayer perceptron trained and evaluated on the GPU in BF16 (FP32 accumulation,
// FP32 master weights, Adam), used to predict the initial guess of the implicit solve
// from a vesicle's shape coefficients.
//
// Network: x -> [Linear -> ReLU] x (n_layers - 1) -> Linear -> y, all hidden widths equal.
// Loss: mean squared error. Layout: activations row-major [batch][features]; weights
// row-major [in][out].
//
// GEMM: C (FP32) = op(A) op(B) with A, B in BF16, on tensor cores through
// mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32. Fragment layout (PTX ISA, m16n8k16,
// .bf16): with g = lane / 4 and t = lane % 4, A regs {a0, a1, a2, a3} hold
// A[g][2t..2t+1], A[g+8][2t..], A[g][2t+8..], A[g+8][2t+8..]; B regs {b0, b1} hold
// B[2t..2t+1][g], B[2t+8..2t+9][g]; C {c0..c3} = C[g][2t..2t+1], C[g+8][2t..2t+1].
// Tiles are staged in shared memory as sA[m][k], sB[n][k] with rows padded to 40 BF16
// (80 bytes), which makes those 32-bit fragment loads bank-conflict free.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace ves3d {

constexpr int kGT = 64;    // CTA tile M and N
constexpr int kGK = 32;    // CTA tile K
constexpr int kGKP = 40;   // padded K stride in shared memory (BF16 elements)

__device__ __forceinline__ void mma_bf16(float* c, const unsigned* a, const unsigned* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// C[M][N] (ldc) = alpha * sum_k A(m, k) B(k, n) (+ beta * C), with
// A(m, k) = TA ? A[k * lda + m] : A[m * lda + k] and B(k, n) = TB ? B[n * ldb + k] : B[k * ldb + n].
template <bool TA, bool TB>
__global__ void __launch_bounds__(128) k_gemm_bf16(int M, int N, int K, const __nv_bfloat16* __restrict__ A, int lda,
                                                   const __nv_bfloat16* __restrict__ B, int ldb, float* __restrict__ C,
                                                   int ldc, float beta) {
  __shared__ __align__(16) __nv_bfloat16 sA[kGT * kGKP];
  __shared__ __align__(16) __nv_bfloat16 sB[kGT * kGKP];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int m0 = blockIdx.y * kGT, n0 = blockIdx.x * kGT;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;  // warp's 32x32 sub-tile
  const int g = lane >> 2, t = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int r = 0; r < 4; r++) acc[i][j][r] = 0.f;
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  for (int k0 = 0; k0 < K; k0 += kGK) {
    __syncthreads();
    for (int i = tid; i < kGT * kGK; i += 128) {
      const int r = i / kGK, c = i % kGK;  // r: m (or n), c: k
      const int m = m0 + r, kk = k0 + c;
      __nv_bfloat16 va = zero;
      if (m < M && kk < K) va = TA ? A[(long)kk * lda + m] : A[(long)m * lda + kk];
      sA[r * kGKP + c] = va;
      const int n = n0 + r;
      __nv_bfloat16 vb = zero;
      if (n < N && kk < K) vb = TB ? B[(long)n * ldb + kk] : B[(long)kk * ldb + n];
      sB[r * kGKP + c] = vb;
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < kGK; ks += 16) {
      unsigned af[2][4], bf[4][2];
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const __nv_bfloat16* a = sA + (wm + i * 16 + g) * kGKP + ks + 2 * t;
        af[i][0] = *reinterpret_cast<const unsigned*>(a);
        af[i][1] = *reinterpret_cast<const unsigned*>(a + 8 * kGKP);
        af[i][2] = *reinterpret_cast<const unsigned*>(a + 8);
        af[i][3] = *reinterpret_cast<const unsigned*>(a + 8 * kGKP + 8);
      }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const __nv_bfloat16* b = sB + (wn + j * 8 + g) * kGKP + ks + 2 * t;
        bf[j][0] = *reinterpret_cast<const unsigned*>(b);
        bf[j][1] = *reinterpret_cast<const unsigned*>(b + 8);
      }
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) mma_bf16(acc[i][j], af[i], bf[j]);
    }
  }
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const int m = m0 + wm + i * 16 + g + (r >= 2 ? 8 : 0);
        const int n = n0 + wn + j * 8 + 2 * t + (r & 1);
        if (m < M && n < N) {
          float* cp = C + (long)m * ldc + n;
          *cp = acc[i][j][r] + (beta != 0.f ? beta * *cp : 0.f);
        }
      }
}

template <bool TA, bool TB>
static int gemm(int M, int N, int K, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, float* C,
                int ldc, float beta, cudaStream_t st) {
  dim3 grid((N + kGT - 1) / kGT, (M + kGT - 1) / kGT);
  k_gemm_bf16<TA, TB><<<grid, 128, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, beta);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

// ---- elementwise kernels ---------------------------------------------------------------
__global__ void k_to_bf16(const float* __restrict__ x, long n, __nv_bfloat16* __restrict__ y) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16(x[i]);
}

// y = bf16((x - shift[c]) * scale[c]) over rows of cols features
__global__ void k_normalize_bf16(const float* __restrict__ x, const float* __restrict__ shift,
                                 const float* __restrict__ scale, long n, int cols, __nv_bfloat16* __restrict__ y) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % cols);
    y[i] = __float2bfloat16((x[i] - shift[c]) * scale[c]);
  }
}

// out = y * scale[c] + shift[c]
__global__ void k_denormalize(const float* __restrict__ y, const float* __restrict__ shift,
                              const float* __restrict__ scale, long n, int cols, float* __restrict__ out) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % cols);
    out[i] = fmaf(y[i], scale[c], shift[c]);
  }
}

// z = z + b (per column); a = relu ? max(z, 0) : z, stored BF16 (and FP32 if af32)
__global__ void k_bias_act(float* __restrict__ z, const float* __restrict__ b, long rows, int cols, bool relu,
                           __nv_bfloat16* __restrict__ a, float* __restrict__ af32) {
  const long n = rows * cols;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    float v = z[i] + b[i % cols];
    z[i] = v;
    if (relu) v = fmaxf(v, 0.f);
    if (a) a[i] = __float2bfloat16(v);
    if (af32) af32[i] = v;
  }
}

// Mean squared error against the normalised target tn = (t - tshift[c]) * tinv[c]:
// d = 2 (y - tn) / n; loss partial sums per block
__global__ void k_mse_grad(const float* __restrict__ y, const float* __restrict__ t, const float* __restrict__ tshift,
                           const float* __restrict__ tinv, long n, int cols, float scale, float* __restrict__ d,
                           __nv_bfloat16* __restrict__ d16, double* __restrict__ loss_part) {
  __shared__ double red[8];
  double s = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % cols);
    const float e = y[i] - (t[i] - tshift[c]) * tinv[c];
    s += (double)e * e;
    const float g = 2.f * e * scale;
    d[i] = g;
    d16[i] = __float2bfloat16(g);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double u = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) u += red[w];
    loss_part[blockIdx.x] = u;
  }
}

// dz = dh * (z > 0), stored FP32 and BF16
__global__ void k_relu_back(const float* __restrict__ dh, const float* __restrict__ z, long n, float* __restrict__ dz,
                            __nv_bfloat16* __restrict__ dz16) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float v = z[i] > 0.f ? dh[i] : 0.f;
    dz[i] = v;
    dz16[i] = __float2bfloat16(v);
  }
}

// db[c] = sum_r d[r][c]
__global__ void k_colsum(const float* __restrict__ d, long rows, int cols, float* __restrict__ db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (long r = 0; r < rows; r++) s += d[r * cols + c];
  db[c] = s;
}

// Adam (Kingma & Ba, 2015) on FP32 master weights; refresh the BF16 copy
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       long n, float lr, float b1, float b2, float eps, float c1, float c2,
                       __nv_bfloat16* __restrict__ w16) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (w16) w16[i] = __float2bfloat16(wi);
  }
}

static unsigned ew_grid(long n) {
  long b = (n + 255) / 256;
  return (unsigned)(b < 2048 ? (b < 1 ? 1 : b) : 2048);
}

}  // namespace ves3d

using namespace ves3d;

// ---------------------------------------------------------------------------------------
struct ves3d_mlp {
  int n_in = 0, n_hid = 0, n_layers = 0, n_out = 0;
  std::vector<int> din, dout;          // per layer
  std::vector<long> woff, boff;        // offsets into the flat parameter vector
  long nparam = 0;
  float *w = nullptr, *gw = nullptr, *m = nullptr, *v = nullptr;  // FP32 master, gradient, Adam moments
  __nv_bfloat16* w16 = nullptr;
  long step = 0;
  // normalisation: network input (x - in_shift) * in_scale; network output z maps to the
  // prediction z * out_scale + out_shift (out_inv = 1 / out_scale, 0 where out_scale is 0)
  float *in_shift = nullptr, *in_scale = nullptr, *out_shift = nullptr, *out_scale = nullptr, *out_inv = nullptr;
  // activations for a batch
  long cap = 0;
  std::vector<float*> z;               // pre-activations per layer [B][dout]
  std::vector<__nv_bfloat16*> a16;     // inputs per layer (a16[0] = x) [B][din]
  float *y = nullptr, *t = nullptr, *d = nullptr, *dh = nullptr, *xin = nullptr;
  __nv_bfloat16* d16 = nullptr;
  double* loss_part = nullptr;
  cudaStream_t st = nullptr;
  ~ves3d_mlp() {
    free_batch();
    cudaFree(w);
    cudaFree(gw);
    cudaFree(m);
    cudaFree(v);
    cudaFree(w16);
    cudaFree(in_shift);
    cudaFree(in_scale);
    cudaFree(out_shift);
    cudaFree(out_scale);
    cudaFree(out_inv);
    if (st) cudaStreamDestroy(st);
  }
  void free_batch() {
    for (auto p : z) cudaFree(p);
    for (auto p : a16) cudaFree(p);
    z.clear();
    a16.clear();
    cudaFree(y);
    cudaFree(t);
    cudaFree(d);
    cudaFree(dh);
    cudaFree(d16);
    cudaFree(xin);
    cudaFree(loss_part);
    y = t = d = dh = xin = nullptr;
    d16 = nullptr;
    loss_part = nullptr;
    cap = 0;
  }
};

namespace {

int mlp_batch(ves3d_mlp* n, long B) {
  if (B <= n->cap) return VES3D_OK;
  n->free_batch();
  int maxw = std::max(n->n_in, std::max(n->n_hid, n->n_out));
  n->z.assign(n->n_layers, nullptr);
  n->a16.assign(n->n_layers, nullptr);
  for (int l = 0; l < n->n_layers; l++) {
    VES3D_CK(cudaMalloc((void**)&n->z[l], sizeof(float) * B * n->dout[l]));
    VES3D_CK(cudaMalloc((void**)&n->a16[l], sizeof(__nv_bfloat16) * B * n->din[l]));
  }
  VES3D_CK(cudaMalloc((void**)&n->y, sizeof(float) * B * n->n_out));
  VES3D_CK(cudaMalloc((void**)&n->t, sizeof(float) * B * n->n_out));
  VES3D_CK(cudaMalloc((void**)&n->d, sizeof(float) * B * maxw));
  VES3D_CK(cudaMalloc((void**)&n->dh, sizeof(float) * B * maxw));
  VES3D_CK(cudaMalloc((void**)&n->d16, sizeof(__nv_bfloat16) * B * maxw));
  VES3D_CK(cudaMalloc((void**)&n->xin, sizeof(float) * B * n->n_in));
  VES3D_CK(cudaMalloc((void**)&n->loss_part, sizeof(double) * 2048));
  n->cap = B;
  return VES3D_OK;
}

int mlp_forward(ves3d_mlp* n, long B) {
  int s;
  cudaStream_t st = n->st;
  k_normalize_bf16<<<ew_grid(B * n->n_in), 256, 0, st>>>(n->xin, n->in_shift, n->in_scale, B * n->n_in, n->n_in,
                                                         n->a16[0]);
  VES3D_LAUNCHED();
  for (int l = 0; l < n->n_layers; l++) {
    const int di = n->din[l], dd = n->dout[l];
    if ((s = gemm<false, false>((int)B, dd, di, n->a16[l], di, n->w16 + n->woff[l], dd, n->z[l], dd, 0.f, st)))
      return s;
    const bool last = l == n->n_layers - 1;
    k_bias_act<<<ew_grid(B * dd), 256, 0, st>>>(n->z[l], n->w + n->boff[l], B, dd, !last, last ? nullptr : n->a16[l + 1],
                                                last ? n->y : nullptr);
    VES3D_LAUNCHED();
  }
  return VES3D_OK;
}

// gradient of the mean squared error into n->gw; returns the loss
int mlp_backward(ves3d_mlp* n, long B, double* loss) {
  int s;
  cudaStream_t st = n->st;
  const long no = B * n->n_out;
  const unsigned gb = ew_grid(no);
  k_mse_grad<<<gb, 256, 0, st>>>(n->y, n->t, n->out_shift, n->out_inv, no, n->n_out, 1.f / (float)no, n->d, n->d16,
                                 n->loss_part);
  VES3D_LAUNCHED();
  for (int l = n->n_layers - 1; l >= 0; l--) {
    const int di = n->din[l], dd = n->dout[l];
    // dW = a^T d   [di x dd]
    if ((s = gemm<true, false>(di, dd, (int)B, n->a16[l], di, n->d16, dd, n->gw + n->woff[l], dd, 0.f, st))) return s;
    k_colsum<<<(dd + 127) / 128, 128, 0, st>>>(n->d, B, dd, n->gw + n->boff[l]);
    VES3D_LAUNCHED();
    if (l == 0) break;
    // dh = d W^T  [B x di], then through the ReLU of layer l-1 (pre-activation z[l-1])
    if ((s = gemm<false, true>((int)B, di, dd, n->d16, dd, n->w16 + n->woff[l], dd, n->dh, di, 0.f, st))) return s;
    k_relu_back<<<ew_grid(B * di), 256, 0, st>>>(n->dh, n->z[l - 1], B * di, n->d, n->d16);
    VES3D_LAUNCHED();
  }
  std::vector<double> lp(gb);
  VES3D_CK(cudaMemcpyAsync(lp.data(), n->loss_part, gb * sizeof(double), cudaMemcpyDeviceToHost, st));
  VES3D_CK(cudaStreamSynchronize(st));
  double sum = 0;
  for (double x : lp) sum += x;
  *loss = sum / (double)no;
  return VES3D_OK;
}

// NULL arrays mean shift 0 / scale 1
int set_scaling(ves3d_mlp* n, const float* in_shift, const float* in_scale, const float* out_shift,
                const float* out_scale) {
  std::vector<float> a(n->n_in), b(n->n_in), c(n->n_out), d(n->n_out), e(n->n_out);
  for (int i = 0; i < n->n_in; i++) {
    a[i] = in_shift ? in_shift[i] : 0.f;
    b[i] = in_scale ? in_scale[i] : 1.f;
  }
  for (int i = 0; i < n->n_out; i++) {
    c[i] = out_shift ? out_shift[i] : 0.f;
    d[i] = out_scale ? out_scale[i] : 1.f;
    e[i] = d[i] != 0.f ? 1.f / d[i] : 0.f;
  }
  VES3D_CK(cudaMemcpyAsync(n->in_shift, a.data(), sizeof(float) * n->n_in, cudaMemcpyHostToDevice, n->st));
  VES3D_CK(cudaMemcpyAsync(n->in_scale, b.data(), sizeof(float) * n->n_in, cudaMemcpyHostToDevice, n->st));
  VES3D_CK(cudaMemcpyAsync(n->out_shift, c.data(), sizeof(float) * n->n_out, cudaMemcpyHostToDevice, n->st));
  VES3D_CK(cudaMemcpyAsync(n->out_scale, d.data(), sizeof(float) * n->n_out, cudaMemcpyHostToDevice, n->st));
  VES3D_CK(cudaMemcpyAsync(n->out_inv, e.data(), sizeof(float) * n->n_out, cudaMemcpyHostToDevice, n->st));
  VES3D_CK(cudaStreamSynchronize(n->st));
  return VES3D_OK;
}

int in_copy(float* dst, const float* src, long n, int is_device, cudaStream_t st) {
  VES3D_CK(cudaMemcpyAsync(dst, src, n * sizeof(float), is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                           st));
  return VES3D_OK;
}

}  // namespace

extern "C" {

int ves3d_mlp_create(int n_in, int n_hidden, int n_layers, int n_out, unsigned long long seed, ves3d_mlp** out) {
  VES3D_ARG(out != nullptr, "out is null");
  *out = nullptr;
  VES3D_ARG(n_in > 0 && n_hidden > 0 && n_out > 0 && n_layers >= 1 && n_layers <= 16, "bad sizes");
  std::unique_ptr<ves3d_mlp> n(new ves3d_mlp());
  n->n_in = n_in;
  n->n_hid = n_hidden;
  n->n_layers = n_layers;
  n->n_out = n_out;
  long off = 0;
  for (int l = 0; l < n_layers; l++) {
    const int di = l == 0 ? n_in : n_hidden, dd = l == n_layers - 1 ? n_out : n_hidden;
    n->din.push_back(di);
    n->dout.push_back(dd);
    n->woff.push_back(off);
    off += (long)di * dd;
    n->boff.push_back(off);
    off += dd;
  }
  n->nparam = off;
  std::vector<float> w(off, 0.f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < n_layers; l++) {
    std::normal_distribution<float> nd(0.f, std::sqrt(2.f / n->din[l]));  // He initialisation
    for (long i = 0; i < (long)n->din[l] * n->dout[l]; i++) w[n->woff[l] + i] = nd(rng);
  }
  VES3D_CK(cudaStreamCreateWithFlags(&n->st, cudaStreamNonBlocking));
  VES3D_CK(cudaMalloc((void**)&n->w, sizeof(float) * off));
  VES3D_CK(cudaMalloc((void**)&n->gw, sizeof(float) * off));
  VES3D_CK(cudaMalloc((void**)&n->m, sizeof(float) * off));
  VES3D_CK(cudaMalloc((void**)&n->v, sizeof(float) * off));
  VES3D_CK(cudaMalloc((void**)&n->w16, sizeof(__nv_bfloat16) * off));
  VES3D_CK(cudaMemcpyAsync(n->w, w.data(), sizeof(float) * off, cudaMemcpyHostToDevice, n->st));
  VES3D_CK(cudaMemsetAsync(n->m, 0, sizeof(float) * off, n->st));
  VES3D_CK(cudaMemsetAsync(n->v, 0, sizeof(float) * off, n->st));
  k_to_bf16<<<ew_grid(off), 256, 0, n->st>>>(n->w, off, n->w16);
  VES3D_LAUNCHED();
  VES3D_CK(cudaMalloc((void**)&n->in_shift, sizeof(float) * n_in));
  VES3D_CK(cudaMalloc((void**)&n->in_scale, sizeof(float) * n_in));
  VES3D_CK(cudaMalloc((void**)&n->out_shift, sizeof(float) * n_out));
  VES3D_CK(cudaMalloc((void**)&n->out_scale, sizeof(float) * n_out));
  VES3D_CK(cudaMalloc((void**)&n->out_inv, sizeof(float) * n_out));
  {
    int s = set_scaling(n.get(), nullptr, nullptr, nullptr, nullptr);
    if (s) return s;
  }
  VES3D_CK(cudaStreamSynchronize(n->st));
  *out = n.release();
  return VES3D_OK;
}

int ves3d_mlp_destroy(ves3d_mlp* n) {
  delete n;
  return VES3D_OK;
}

long ves3d_mlp_num_params(ves3d_mlp* n) { return n ? n->nparam : -1; }

int ves3d_mlp_get_params(ves3d_mlp* n, float* out) {
  VES3D_ARG(n && out, "null argument");
  VES3D_CK(cudaMemcpyAsync(out, n->w, sizeof(float) * n->nparam, cudaMemcpyDeviceToHost, n->st));
  VES3D_CK(cudaStreamSynchronize(n->st));
  return VES3D_OK;
}

int ves3d_mlp_set_params(ves3d_mlp* n, const float* in) {
  VES3D_ARG(n && in, "null argument");
  VES3D_CK(cudaMemcpyAsync(n->w, in, sizeof(float) * n->nparam, cudaMemcpyHostToDevice, n->st));
  k_to_bf16<<<ew_grid(n->nparam), 256, 0, n->st>>>(n->w, n->nparam, n->w16);
  VES3D_LAUNCHED();
  VES3D_CK(cudaStreamSynchronize(n->st));
  return VES3D_OK;
}

int ves3d_mlp_set_scaling(ves3d_mlp* n, const float* in_shift, const float* in_scale, const float* out_shift,
                          const float* out_scale) {
  VES3D_ARG(n != nullptr, "null network");
  return set_scaling(n, in_shift, in_scale, out_shift, out_scale);
}

int ves3d_mlp_forward(ves3d_mlp* n, const float* X, long batch, float* Y, int is_device) {
  VES3D_ARG(n && X && Y && batch > 0, "bad arguments");
  int s;
  if ((s = mlp_batch(n, batch))) return s;
  if ((s = in_copy(n->xin, X, batch * n->n_in, is_device, n->st))) return s;
  if ((s = mlp_forward(n, batch))) return s;
  const long no = batch * n->n_out;
  k_denormalize<<<ew_grid(no), 256, 0, n->st>>>(n->y, n->out_shift, n->out_scale, no, n->n_out, n->d);
  VES3D_LAUNCHED();
  VES3D_CK(cudaMemcpyAsync(Y, n->d, sizeof(float) * no, is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                           n->st));
  VES3D_CK(cudaStreamSynchronize(n->st));
  return VES3D_OK;
}

int ves3d_mlp_gradients(ves3d_mlp* n, const float* X, const float* T, long batch, float* grads, double* loss,
                        int is_device) {
  VES3D_ARG(n && X && T && batch > 0 && loss, "bad arguments");
  int s;
  if ((s = mlp_batch(n, batch))) return s;
  if ((s = in_copy(n->xin, X, batch * n->n_in, is_device, n->st))) return s;
  if ((s = in_copy(n->t, T, batch * n->n_out, is_device, n->st))) return s;
  if ((s = mlp_forward(n, batch))) return s;
  if ((s = mlp_backward(n, batch, loss))) return s;
  if (grads) {
    VES3D_CK(cudaMemcpyAsync(grads, n->gw, sizeof(float) * n->nparam, cudaMemcpyDeviceToHost, n->st));
    VES3D_CK(cudaStreamSynchronize(n->st));
  }
  return VES3D_OK;
}

int ves3d_mlp_train_step(ves3d_mlp* n, const float* X, const float* T, long batch, float lr, double* loss,
                         int is_device) {
  int s = ves3d_mlp_gradients(n, X, T, batch, nullptr, loss, is_device);
  if (s) return s;
  n->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)n->step), c2 = 1.f - std::pow(b2, (float)n->step);
  k_adam<<<ew_grid(n->nparam), 256, 0, n->st>>>(n->w, n->gw, n->m, n->v, n->nparam, lr, b1, b2, 1e-8f, c1, c2, n->w16);
  VES3D_LAUNCHED();
  VES3D_CK(cudaStreamSynchronize(n->st));
  return VES3D_OK;
}

}  // extern "C"
