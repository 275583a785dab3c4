// C++ caller of the device-pointer parts of include/ves3d_b200.hpp, written the way Ves3D's
// C++ code uses MovePole, Device<GPU>::AggregateRotation, Device<GPU>::DirectStokes<float>
// and Surface (C++03; the CUDA runtime only for device buffers).
//   device_api_test movepole  in out  in: int32 p, nfun, ntrg, targets[2 ntrg], F[nfun np]
//                                     out: [ntrg][nfun np] the rotated functions
//   device_api_test aggregate in out  in: int32 p, nfun, mat[np np], F[nfun np]
//                                     out: [2p][nfun np] (AggregateRotation, one operand)
//   device_api_test stokes32  in out  in: int32 src_m, trg_m, n, head, tail, has_q, then
//                                     float T[3 n trg_m], S[3 n src_m], D[3 n src_m], Q[src_m]
//                                     out: float U[3 n trg_m]
//   device_api_test surface   in out  in: int32 p, nves, X[3 nves ng] (double)
//                                     out: normal, W, H, K, area, volume, centers,
//                                     grad of x, div of X, linearised H of X
#include <cuda_runtime_api.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "ves3d_b200.hpp"

namespace {

template <class T>
bool read_vec(std::FILE* f, std::vector<T>& v, size_t n) {
  v.resize(n);
  return n == 0 || std::fread(&v[0], sizeof(T), n, f) == n;
}

template <class T>
T* to_device(const std::vector<T>& h) {
  void* d = 0;
  if (cudaMalloc(&d, h.size() * sizeof(T) + 16) != cudaSuccess) return 0;
  cudaMemcpy(d, &h[0], h.size() * sizeof(T), cudaMemcpyHostToDevice);
  return (T*)d;
}

template <class T>
void append(std::FILE* f, const T* d, size_t n) {
  std::vector<T> h(n);
  cudaMemcpy(&h[0], d, n * sizeof(T), cudaMemcpyDeviceToHost);
  std::fwrite(&h[0], sizeof(T), n, f);
}

int move_pole(std::FILE* in, std::FILE* out) {
  int hdr[3];
  if (std::fread(hdr, sizeof(int), 3, in) != 3) return 3;
  const int p = hdr[0], nfun = hdr[1], ntrg = hdr[2];
  const size_t np = (size_t)2 * p * (p + 1);
  std::vector<int> trg;
  std::vector<double> F;
  if (!read_vec(in, trg, 2 * (size_t)ntrg) || !read_vec(in, F, nfun * np)) return 3;
  double* dF = to_device(F);
  std::vector<double> zero(nfun * np, 0.0);
  double* dR = to_device(zero);
  const double* arr[1] = {dF};
  double* res[1] = {dR};
  const long nf[1] = {nfun};
  ves3d_b200::MovePole mp(p);
  mp.setOperands(arr, nf, 1, ves3d_b200::MovePole::Direct);
  for (int t = 0; t < ntrg; t++) {
    mp(trg[2 * t], trg[2 * t + 1], res);
    append(out, dR, nfun * np);
  }
  cudaFree(dF);
  cudaFree(dR);
  return 0;
}

int aggregate(std::FILE* in, std::FILE* out) {
  int hdr[2];
  if (std::fread(hdr, sizeof(int), 2, in) != 2) return 3;
  const int p = hdr[0], nfun = hdr[1], nlat = p + 1, nlong = 2 * p;
  const size_t np = (size_t)nlat * nlong;
  std::vector<double> mat, F;
  if (!read_vec(in, mat, np * np) || !read_vec(in, F, nfun * np)) return 3;
  double* dM = to_device(mat);
  double* dF = to_device(F);
  std::vector<double> zero(nfun * np * nlong, 0.0);
  double* dR = to_device(zero);
  std::vector<double*> res(nlong);
  for (int jj = 0; jj < nlong; jj++) res[jj] = dR + jj * nfun * np;
  const double* vec[1] = {dF};
  double* wrk[1] = {0};
  const int n_sub[1] = {nfun};
  ves3d_b200::Device dev;
  dev.AggregateRotation(p, nlat, nlong, 1, n_sub, dM, vec, wrk, &res[0], 1);
  append(out, dR, nfun * np * nlong);
  cudaFree(dM);
  cudaFree(dF);
  cudaFree(dR);
  return 0;
}

int stokes32(std::FILE* in, std::FILE* out) {
  int h[6];
  if (std::fread(h, sizeof(int), 6, in) != 6) return 3;
  const int src_m = h[0], trg_m = h[1], n = h[2], head = h[3], tail = h[4], has_q = h[5];
  std::vector<float> T, S, D, Q, U(3 * (size_t)n * trg_m, 0.f);
  if (!read_vec(in, T, 3 * (size_t)n * trg_m) || !read_vec(in, S, 3 * (size_t)n * src_m) ||
      !read_vec(in, D, 3 * (size_t)n * src_m) || (has_q && !read_vec(in, Q, src_m)))
    return 3;
  float *dT = to_device(T), *dS = to_device(S), *dD = to_device(D), *dU = to_device(U);
  float* dQ = has_q ? to_device(Q) : 0;
  ves3d_b200::DirectStokes(dS, dD, dQ, src_m, trg_m, n, dT, head, tail, dU);
  cudaDeviceSynchronize();
  append(out, dU, U.size());
  cudaFree(dT);
  cudaFree(dS);
  cudaFree(dD);
  cudaFree(dU);
  if (dQ) cudaFree(dQ);
  return 0;
}

int surface(std::FILE* in, std::FILE* out) {
  int hdr[2];
  if (std::fread(hdr, sizeof(int), 2, in) != 2) return 3;
  const int p = hdr[0], nv = hdr[1];
  const size_t ng = (size_t)2 * p * (p + 1);
  std::vector<double> X;
  if (!read_vec(in, X, 3 * nv * ng)) return 3;
  ves3d_b200::Surface<double> S(p, &X[0], X.size());
  std::vector<double> v;
  S.getNormal(v);
  std::fwrite(&v[0], sizeof(double), v.size(), out);
  S.getAreaElement(v);
  std::fwrite(&v[0], sizeof(double), v.size(), out);
  S.getMeanCurv(v);
  std::fwrite(&v[0], sizeof(double), v.size(), out);
  S.getGaussianCurv(v);
  std::fwrite(&v[0], sizeof(double), v.size(), out);
  S.area(v);
  std::fwrite(&v[0], sizeof(double), v.size(), out);
  S.volume(v);
  std::fwrite(&v[0], sizeof(double), v.size(), out);
  S.getCenters(v);
  std::fwrite(&v[0], sizeof(double), v.size(), out);
  // grad of the x coordinate, div of the position field, linearised H of the positions
  std::vector<double> fx(nv * ng), g(3 * nv * ng), d(nv * ng), hl(nv * ng);
  for (int k = 0; k < nv; k++)
    for (size_t i = 0; i < ng; i++) fx[k * ng + i] = X[(3 * k) * ng + i];
  S.grad(&fx[0], &g[0]);
  S.div(&X[0], &d[0]);
  S.linearizedMeanCurv(&X[0], &hl[0]);
  std::fwrite(&g[0], sizeof(double), g.size(), out);
  std::fwrite(&d[0], sizeof(double), d.size(), out);
  std::fwrite(&hl[0], sizeof(double), hl.size(), out);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: device_api_test movepole|aggregate|stokes32|surface in out\n");
    return 2;
  }
  std::FILE* in = std::fopen(argv[2], "rb");
  std::FILE* out = std::fopen(argv[3], "wb");
  if (!in || !out) return 3;
  int rc = 2;
  try {
    if (std::strcmp(argv[1], "movepole") == 0) rc = move_pole(in, out);
    if (std::strcmp(argv[1], "aggregate") == 0) rc = aggregate(in, out);
    if (std::strcmp(argv[1], "stokes32") == 0) rc = stokes32(in, out);
    if (std::strcmp(argv[1], "surface") == 0) rc = surface(in, out);
  } catch (const ves3d_b200::Error& e) {
    std::fprintf(stderr, "error %d: %s\n", e.status(), e.what());
    rc = 5;
  }
  std::fclose(in);
  std::fclose(out);
  return rc;
}
