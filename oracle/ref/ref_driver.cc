// Test infrastructure only. Flat C entry points over the reference's OWN CPU code,
// compiled in place from the reference tree by oracle/ref/Makefile into oracle/_ref/.
// Used by the tests (to pin the Python/C restatement in oracle/) and by bench.py's
// CPU-baseline / reference arm. Never part of the product path.
//
// What each entry point calls (reference file:line):
//   ref_grid2shc        SphericalHarmonics<double>::Grid2SHC      src/SphericalHarmonics.cc:152
//   ref_shc2grid        SphericalHarmonics<double>::SHC2Grid      src/SphericalHarmonics.cc:4
//   ref_shc2pole        SphericalHarmonics<double>::SHC2Pole      src/SphericalHarmonics.cc:325
//   ref_rotate_all      SphericalHarmonics<double>::RotateAll     src/SphericalHarmonics.cc:363
//   ref_*_weights/nodes LegendreNodes/LegendreWeights/SingularWeights :544-604
//   ref_singular_sl     SphericalHarmonics<double>::StokesSingularInteg  :863 (SL and/or DL)
//   ref_alltoall        StokesAlltoAll (double)                    src/CPUKernels.cc:1011
//   ref_direct_stokes   DirectStokesKernel (double)               src/CPUKernels.cc:123
//   ref_direct_stokes_dl DirectStokesDoubleLayerKernel (double)   src/CPUKernels.cc:1060
//   ref_bicgstab_dense  BiCGStab<Container, MatVec, Precond>  src/BiCGStab.cc:45-138
//   ref_stokes_velocity_sl  the non-FMM StokesVelocity composition:
//       u = SHC2Grid(Grid2SHC(f) . SLMatrix)                        (src/StokesVelocity.cc:385-473)
//         + StokesAlltoAll(x, f.area.qw) - DirectStokesKernel(x, f.area, qw)
//                                                                   (src/InterfacialVelocity.cc:1261-1291)
#include <omp.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>
#include <sys/time.h>

#include <SphericalHarmonics.h>
#include <CPUKernels.h>

extern "C" void scipy_openblas_set_num_threads(int);

typedef pvfmm::Vector<double> Vec;
typedef SphericalHarmonics<double> SH;

static double wall() {
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

static void copy_out(const Vec& v, double* out) {
  if (out && v.Dim()) std::memcpy(out, &v[0], sizeof(double) * v.Dim());
}

extern "C" {

// OpenMP threads for the reference loops; BLAS runs single-threaded inside them
// (the reference calls GEMM from inside its own OpenMP regions).
int ref_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
  scipy_openblas_set_num_threads(1);
  return omp_get_max_threads();
}

int ref_grid2shc(const double* X, long nfun, long p0, long p1, double* S) {
  Vec x(nfun * 2 * p0 * (p0 + 1), (double*)X, false), s;
  SH::Grid2SHC(x, p0, p1, s);
  copy_out(s, S);
  return 0;
}

int ref_shc2grid(const double* S, long nfun, long p0, long p1, double* X, double* Xth, double* Xph) {
  Vec s(nfun * p0 * (p0 + 2), (double*)S, false), x, xt, xp;
  SH::SHC2Grid(s, p0, p1, x, Xth ? &xt : NULL, Xph ? &xp : NULL);
  copy_out(x, X);
  if (Xth) copy_out(xt, Xth);
  if (Xph) copy_out(xp, Xph);
  return 0;
}

int ref_shc2pole(const double* S, long nfun, long p0, double* P) {
  Vec s(nfun * p0 * (p0 + 2), (double*)S, false), pole;
  SH::SHC2Pole(s, p0, pole);
  copy_out(pole, P);
  return 0;
}

int ref_rotate_all(const double* S, long nves, long p0, long dof, double* out) {
  Vec s(nves * dof * p0 * (p0 + 2), (double*)S, false), r;
  SH::RotateAll(s, p0, dof, r);
  copy_out(r, out);
  return 0;
}

int ref_legendre_nodes(long p, double* out) { copy_out(SH::LegendreNodes(p), out); return 0; }
int ref_legendre_weights(long p, double* out) { copy_out(SH::LegendreWeights(p), out); return 0; }
int ref_singular_weights(long p, double* out) { copy_out(SH::SingularWeights(p), out); return 0; }

// SL (and optionally DL) self matrices, each nves x (3 Ncoef) x (3 Ncoef).
int ref_singular_matrices(const double* X, long nves, long p0, long p1, double* SL, double* DL) {
  long Ngrid = 2 * p0 * (p0 + 1);
  Vec x(nves * 3 * Ngrid, (double*)X, false), sl, dl;
  SH::StokesSingularInteg(x, p0, p1, SL ? &sl : NULL, DL ? &dl : NULL);
  if (SL) copy_out(sl, SL);
  if (DL) copy_out(dl, DL);
  return 0;
}

int ref_alltoall(const double* src, const double* den, long np, double* pot) {
  StokesAlltoAll(src, den, (size_t)np, pot, NULL);
  return 0;
}

int ref_direct_stokes(int src_stride, int trg_stride, int n_surfs, int trg_idx_head, int trg_idx_tail,
                      const double* qw, const double* trg, const double* src, const double* den,
                      double* pot) {
  DirectStokesKernel(src_stride, trg_stride, n_surfs, trg_idx_head, trg_idx_tail, qw, trg, src, den, pot);
  return 0;
}

extern "C" int ref_direct_stokes_dl(int src_stride, int trg_stride, int n_surfs, int trg_idx_head,
                                    int trg_idx_tail, const double* qw, const double* trg, const double* src,
                                    const double* norm, const double* den, double* pot) {
  DirectStokesDoubleLayerKernel(src_stride, trg_stride, n_surfs, trg_idx_head, trg_idx_tail, qw, trg, src, norm, den,
                                pot);
  return 0;
}

// Area element |X_theta x X_phi| at order p (src/StokesVelocity.cc:252-273) and the
// smooth quadrature weights LegendreWeights(p) replicated over longitudes.
static void area_and_weights(const double* X, long nves, long p, std::vector<double>& area,
                             std::vector<double>& qw) {
  long Ngrid = 2 * p * (p + 1);
  Vec x(nves * 3 * Ngrid, (double*)X, false), shc, xg, xt, xp;
  SH::Grid2SHC(x, p, p, shc);
  SH::SHC2Grid(shc, p, p, xg, &xt, &xp);
  area.assign(nves * Ngrid, 0.0);
  for (long v = 0; v < nves; v++)
    for (long k = 0; k < Ngrid; k++) {
      double ax = xt[(v * 3 + 0) * Ngrid + k], ay = xt[(v * 3 + 1) * Ngrid + k], az = xt[(v * 3 + 2) * Ngrid + k];
      double bx = xp[(v * 3 + 0) * Ngrid + k], by = xp[(v * 3 + 1) * Ngrid + k], bz = xp[(v * 3 + 2) * Ngrid + k];
      double nx = ay * bz - az * by, ny = az * bx - ax * bz, nz = ax * by - ay * bx;
      area[v * Ngrid + k] = std::sqrt(nx * nx + ny * ny + nz * nz);
    }
  Vec& w = SH::LegendreWeights(p);
  qw.assign(Ngrid, 0.0);
  for (long i = 0; i < p + 1; i++)
    for (long j = 0; j < 2 * p; j++) qw[i * 2 * p + j] = w[i];
}

int ref_area_weights(const double* X, long nves, long p, double* area_out, double* qw_out) {
  std::vector<double> area, qw;
  area_and_weights(X, nves, p, area, qw);
  if (area_out) std::memcpy(area_out, &area[0], sizeof(double) * area.size());
  if (qw_out) std::memcpy(qw_out, &qw[0], sizeof(double) * qw.size());
  return 0;
}

// Self part only: vel_self = SHC2Grid(Grid2SHC(f) . SL) given prebuilt SL matrices.
int ref_self_apply(const double* SL, const double* f, long nves, long p, double* vel) {
  long Ngrid = 2 * p * (p + 1), Ncoef = p * (p + 2), n = 3 * Ncoef;
  Vec fv(nves * 3 * Ngrid, (double*)f, false), F, V(nves * n), out;
  SH::Grid2SHC(fv, p, p, F);
#pragma omp parallel for
  for (long v = 0; v < nves; v++) {
    pvfmm::Matrix<double> Mv(1, n, &V[v * n], false), Mf(1, n, &F[v * n], false),
        M(n, n, (double*)&SL[v * n * n], false);
    pvfmm::Matrix<double>::GEMM(Mv, Mf, M);
  }
  SH::SHC2Grid(V, p, p, out);
  copy_out(out, vel);
  return 0;
}

// Far part: all-pairs over the order-p grid with den = f.area.qw, minus the
// same-vesicle sum (DirectStokesKernel with weights area.qw per vesicle).
int ref_far_sl(const double* X, const double* f, long nves, long p, double* vel, double* t_far) {
  long Ngrid = 2 * p * (p + 1), N = nves * Ngrid;
  std::vector<double> area, qw;
  area_and_weights(X, nves, p, area, qw);
  std::vector<double> pos(3 * N), den(3 * N), pot(3 * N), fa(3 * N), self(3 * N);
  for (long v = 0; v < nves; v++)
    for (long c = 0; c < 3; c++)
      for (long k = 0; k < Ngrid; k++) {
        long a = (v * 3 + c) * Ngrid + k, pm = (v * Ngrid + k) * 3 + c;
        pos[pm] = X[a];
        den[pm] = f[a] * area[v * Ngrid + k] * qw[k];
        fa[a] = f[a] * area[v * Ngrid + k];
      }
  double t0 = wall();
  StokesAlltoAll(&pos[0], &den[0], (size_t)N, &pot[0], NULL);
  DirectStokesKernel((int)Ngrid, (int)Ngrid, (int)nves, 0, (int)Ngrid, &qw[0], X, X, &fa[0], &self[0]);
  double t1 = wall();
  if (t_far) *t_far = t1 - t0;
  for (long v = 0; v < nves; v++)
    for (long c = 0; c < 3; c++)
      for (long k = 0; k < Ngrid; k++) {
        long a = (v * 3 + c) * Ngrid + k, pm = (v * Ngrid + k) * 3 + c;
        vel[a] = pot[pm] - self[a];
      }
  return 0;
}

// Full composition; timings in seconds for the self build, self apply and far part.
int ref_stokes_velocity_sl(const double* X, const double* f, long nves, long p, long p_up, double* vel,
                           double* timings) {
  long Ngrid = 2 * p * (p + 1), Ncoef = p * (p + 2), n = 3 * Ncoef;
  std::vector<double> SL(nves * n * n), vs(nves * 3 * Ngrid), vf(nves * 3 * Ngrid);
  double t0 = wall();
  ref_singular_matrices(X, nves, p, p_up, &SL[0], NULL);
  double t1 = wall();
  ref_self_apply(&SL[0], f, nves, p, &vs[0]);
  double t2 = wall();
  double tfar = 0;
  ref_far_sl(X, f, nves, p, &vf[0], &tfar);
  for (long i = 0; i < nves * 3 * Ngrid; i++) vel[i] = vs[i] + vf[i];
  if (timings) {
    timings[0] = t1 - t0;
    timings[1] = t2 - t1;
    timings[2] = tfar;
  }
  return 0;
}

}  // extern "C"

// ---- BiCGStab (include/BiCGStab.h, src/BiCGStab.cc) on a dense matrix -----------------
#include <BiCGStab.h>

namespace refbicg {
struct RVec {
  typedef double value_type;
  std::vector<double> d;
  void replicate(const RVec& o) { d.assign(o.d.size(), 0.0); }
  size_t size() const { return d.size(); }
};
// out = a * x + y
void axpy(double a, const RVec& x, const RVec& y, RVec& out) {
  for (size_t i = 0; i < x.d.size(); i++) out.d[i] = a * x.d[i] + y.d[i];
}
double AlgebraicDot(const RVec& x, const RVec& y) {
  double s = 0;
  for (size_t i = 0; i < x.d.size(); i++) s += x.d[i] * y.d[i];
  return s;
}
struct Dense {
  const double* A;
  long n;
  void operator()(const RVec& x, RVec& y) const {
    for (long i = 0; i < n; i++) {
      double s = 0;
      for (long j = 0; j < n; j++) s += A[i * n + j] * x.d[j];
      y.d[i] = s;
    }
  }
};
struct Ident {
  void operator()(const RVec& in, RVec& out) const { out.d = in.d; }
};
}  // namespace refbicg

extern "C" int ref_bicgstab_dense(const double* A, const double* b, double* x, long n, double* tol, int* max_iter) {
  using namespace refbicg;
  RVec xv, bv;
  xv.d.assign(x, x + n);
  bv.d.assign(b, b + n);
  Dense M = {A, n};
  BiCGStab<RVec, Dense, Ident> solver;
  BiCGSReturn r = solver(M, xv, bv, *max_iter, *tol, Ident());
  std::memcpy(x, &xv.d[0], sizeof(double) * n);
  return (int)r;
}
