/* ves3d_b200.hpp -- header-only C++ mirror of the reference's operator API over the C ABI
 * of ves3d_b200.h, for dropping the B200 path into Ves3D's C++ code. It compiles as C++03
 * (the reference's dialect: -std=gnu++03) and needs no CUDA headers.
 *
 *   reference (lu1and10/ves3d)                              here
 *   StokesVelocity<Real> (include/StokesVelocity.h:9-44)     ves3d_b200::StokesVelocity<double>
 *   SHTrans<Container, Mats> (include/SHTrans.h:21-63)       ves3d_b200::SHTrans<double>
 *   Device<GPU>::DirectStokes (include/Device.h:205-209)     ves3d_b200::DirectStokes (double, float)
 *   Device<GPU>::AggregateRotation (include/Device.h:234-237) ves3d_b200::Device::AggregateRotation
 *   MovePole<Container, Operators> (include/MovePole.h:16-23) ves3d_b200::MovePole
 *   Surface<Sca, Vec> (include/Surface.h:38-77)              ves3d_b200::Surface<double>
 *   InterfacialVelocity implicit solve (src/InterfacialVelocity.cc:203-1172)
 *                                                            StokesVelocity::ImplicitSolve
 *
 * Containers: any type with operator[] and size() holding doubles contiguously (std::vector,
 * the reference's Array-based containers through their begin()/size() via the pointer
 * overloads). Failures throw ves3d_b200::Error carrying the C ABI status and message.
 */
#ifndef VES3D_B200_HPP
#define VES3D_B200_HPP

#include <stdexcept>
#include <string>
#include <vector>

#include "ves3d_b200.h"

namespace ves3d_b200 {

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string& what) : std::runtime_error(what), status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

inline void check(int status, const char* what) {
  if (status != VES3D_OK) {
    const char* msg = ves3d_last_error();
    throw Error(status, std::string(what) + ": " + (msg ? msg : ""));
  }
}

/* StokesVelocity<Real>: single-layer velocity of a suspension at its own surface points
 * (surfaces and densities AxisMajor [n_ves][3][(p+1) 2p], as the reference's containers).
 * The far field is the exact all-pairs sum (the reference's PVFMM is not used); box_size and
 * repul_dist are accepted for signature compatibility, repulsion is not supported. */
template <class Real>
class StokesVelocity {
 public:
  StokesVelocity(int sh_order, int sh_order_up, Real box_size = -1, Real repul_dist = 1e-3,
                 int precision = VES3D_PREC_FP64, int device = -1)
      : sv_(0), p_(sh_order), nv_(0) {
    (void)box_size;
    (void)repul_dist;
    check(ves3d_sv_create(sh_order, sh_order_up, precision, device, &sv_), "StokesVelocity");
  }
  ~StokesVelocity() { ves3d_sv_destroy(sv_); }

  /* SetSrcCoord(S, sh_order_up_self, sh_order_up): the upsample orders are fixed at
   * construction; passing different ones is an error. */
  void SetSrcCoord(const Real* S, size_t n, int sh_order_up_self = -1, int sh_order_up = -1,
                   bool on_device = false) {
    (void)sh_order_up_self;
    (void)sh_order_up;
    const size_t per = 3 * (size_t)2 * p_ * (p_ + 1);
    if (n == 0 || n % per) throw Error(VES3D_ERR_ARG, "SetSrcCoord: size is not a multiple of 3 (p+1) 2p");
    nv_ = (long)(n / per);
    check(ves3d_sv_set_src_coord(sv_, S, nv_, on_device ? 1 : 0), "SetSrcCoord");
  }
  template <class Vec>
  void SetSrcCoord(const Vec& S, int sh_order_up_self = -1, int sh_order_up = -1) {
    SetSrcCoord(&S[0], S.size(), sh_order_up_self, sh_order_up);
  }

  void SetDensitySL(const Real* f, bool add_repul = false, bool on_device = false) {
    if (add_repul) throw Error(VES3D_ERR_ARG, "SetDensitySL: repulsion is not supported");
    check(ves3d_sv_set_density_sl(sv_, f, on_device ? 1 : 0), "SetDensitySL");
  }
  template <class Vec>
  void SetDensitySL(const Vec* force_single, bool add_repul = false) {
    SetDensitySL(&(*force_single)[0], add_repul);
  }
  /* SetTrgCoord(T): off-surface targets [n][3] (NULL: the surface); EvalTrg: their velocities
   * (accurate away from the surfaces) */
  void SetTrgCoord(const Real* T, long n_trg, bool on_device = false) {
    check(ves3d_sv_set_trg_coord(sv_, T, n_trg, on_device ? 1 : 0), "SetTrgCoord");
  }
  void EvalTrg(Real* vel, bool on_device = false) { check(ves3d_sv_eval_trg(sv_, vel, on_device ? 1 : 0), "EvalTrg"); }
  /* MonitorError(tol): the double layer of density 1 against -1/2; adapts the self order */
  Real MonitorError(Real tol) {
    double total = 0;
    check(ves3d_sv_monitor_error(sv_, tol, 0, &total), "MonitorError");
    return (Real)total;
  }
  /* SetDensityDL(f): the double-layer density, NULL to turn the double layer off. */
  void SetDensityDL(const Real* f, bool on_device = false) {
    check(ves3d_sv_set_density_dl(sv_, f, on_device ? 1 : 0), "SetDensityDL");
  }
  template <class Vec>
  void SetDensityDL(const Vec* force_double) {
    SetDensityDL(force_double ? &(*force_double)[0] : (const Real*)0);
  }

  /* operator()(vel): velocity into a caller container of the surfaces' size. */
  void operator()(Real* vel, bool on_device = false) { check(ves3d_sv_eval(sv_, vel, on_device ? 1 : 0), "eval"); }
  template <class Vec>
  void operator()(Vec& vel) {
    operator()(&vel[0]);
  }
  /* operator()(): velocity in an internal host vector. */
  const std::vector<Real>& operator()() {
    vel_.resize((size_t)nv_ * 3 * 2 * p_ * (p_ + 1));
    operator()(&vel_[0]);
    return vel_;
  }

  /* The globally implicit step on the current surfaces (Galerkin form, BiCGStab):
   * x0 (may be NULL: zero guess) and x are grid fields [u; sigma] of 4 N doubles. Returns
   * the BiCGSReturn code (100 success); tol and max_iter are in/out as in BiCGStab. */
  void SetImplicitParams(Real dt, Real bending_modulus, Real shear_rate) {
    check(ves3d_sv_set_implicit_params(sv_, dt, bending_modulus, shear_rate), "SetImplicitParams");
  }
  /* the vesicles' viscosity contrast: one value for all, or one per vesicle (n values) */
  void SetViscosityContrast(const Real* lambda, long n) {
    check(ves3d_sv_set_viscosity_contrast(sv_, lambda, n), "SetViscosityContrast");
  }
  void SetPrecond(int scheme, int refresh_every = 1) {
    check(ves3d_sv_set_precond(sv_, scheme), "SetPrecond");
    check(ves3d_sv_set_precond_refresh(sv_, refresh_every), "SetPrecond");
  }
  int ImplicitSolve(const Real* x0, Real* x, Real& tol, int& max_iter, bool on_device = false) {
    int code = 0;
    double t = tol;
    check(ves3d_sv_implicit_solve(sv_, x0, x, &t, &max_iter, &code, on_device ? 1 : 0), "ImplicitSolve");
    tol = t;
    return code;
  }

  long NumVesicles() const { return nv_; }
  ves3d_sv* handle() { return sv_; }

 private:
  StokesVelocity(const StokesVelocity&);
  StokesVelocity& operator=(const StokesVelocity&);
  ves3d_sv* sv_;
  int p_;
  long nv_;
  std::vector<Real> vel_;
};

/* SHTrans<Real> on device pointers (forward = Grid2SHC, backward = SHC2Grid with the
 * optional longitude / latitude derivatives of backward_dv / backward_du, the low-pass
 * filters and ScaleFreq), in the per-function coefficient order shared by the reference's
 * SHTrans and SphericalHarmonics; coefficient arrays are function-major. */
template <class Real>
class SHTrans {
 public:
  /* filter_freq -1 means 2p/3 and filter_exponent is lowPassFilterPoly's exponent, with the
   * reference constructor's defaults (SHTrans(p, mats, filter_freq, filter_exponent)) */
  explicit SHTrans(int sh_order, void* stream = 0, int filter_freq = -1, Real filter_exponent = 4.0)
      : p_(sh_order), stream_(stream), freq_(filter_freq < 0 ? 2 * sh_order / 3 : filter_freq),
        exponent_(filter_exponent) {}
  int getShOrder() const { return p_; }
  int getShFilterFreq() const { return freq_; }
  Real getShFilterExponent() const { return exponent_; }
  /* the two filters on the host, p(p+2) values each (hard cut / polynomial) */
  void filterCoeffs(std::vector<Real>& hard, std::vector<Real>& poly) const {
    hard.resize((size_t)p_ * (p_ + 2));
    poly.resize(hard.size());
    check(ves3d_sht_filter_coeffs(p_, freq_, 0.0, &hard[0]), "SHTrans::filterCoeffs");
    check(ves3d_sht_filter_coeffs(p_, freq_, exponent_, &poly[0]), "SHTrans::filterCoeffs");
  }
  void lowPassFilter(const Real* in, long n_funs, Real* out) const {
    check(ves3d_sht_lowpass(in, n_funs, p_, freq_, 0.0, out, stream_), "SHTrans::lowPassFilter");
  }
  void lowPassFilterPoly(const Real* in, long n_funs, Real* out) const {
    check(ves3d_sht_lowpass(in, n_funs, p_, freq_, exponent_, out, stream_), "SHTrans::lowPassFilterPoly");
  }
  /* scaling_coeff: device array of p(p+2) values */
  void ScaleFreq(const Real* shc_in, long n_funs, const Real* scaling_coeff, Real* shc_out) const {
    check(ves3d_sht_scale_freq(shc_in, n_funs, p_, scaling_coeff, shc_out, stream_), "SHTrans::ScaleFreq");
  }
  void forward(const Real* in, long n_funs, Real* shc) const {
    check(ves3d_sht_forward(in, n_funs, p_, p_, shc, stream_), "SHTrans::forward");
  }
  void backward(const Real* shc, long n_funs, Real* out, Real* d_longitude = 0, Real* d_latitude = 0) const {
    check(ves3d_sht_backward(shc, n_funs, p_, p_, out, d_longitude, d_latitude, stream_), "SHTrans::backward");
  }
  /* resampling p -> q (SHC2Grid(p, q)) */
  void backward_to(int q, const Real* shc, long n_funs, Real* out) const {
    check(ves3d_sht_backward(shc, n_funs, p_, q, out, 0, 0, stream_), "SHTrans::backward_to");
  }
  /* second derivatives (u latitude, v longitude) */
  void backward_d2u(const Real* shc, long n_funs, Real* out) const {
    check(ves3d_sht_backward_d2(shc, n_funs, p_, out, 0, 0, stream_), "SHTrans::backward_d2u");
  }
  void backward_d2v(const Real* shc, long n_funs, Real* out) const {
    check(ves3d_sht_backward_d2(shc, n_funs, p_, 0, out, 0, stream_), "SHTrans::backward_d2v");
  }
  void backward_duv(const Real* shc, long n_funs, Real* out) const {
    check(ves3d_sht_backward_d2(shc, n_funs, p_, 0, 0, out, stream_), "SHTrans::backward_duv");
  }
  /* SphericalHarmonics::SHC2Pole: pole[2 f + t] = function f at x = -1 (t = 0), x = +1 (t = 1) */
  void SHC2Pole(const Real* shc, long n_funs, Real* pole) const {
    check(ves3d_sht_pole(shc, n_funs, p_, pole, stream_), "SHTrans::SHC2Pole");
  }

 private:
  int p_;
  void* stream_;
  int freq_;
  Real exponent_;
};

/* Device<GPU> (include/Device.h:81-253): the primitives a caller of the operators uses,
 * on device pointers, with the reference's signatures (gemm takes its BLAS arguments by
 * pointer as the reference's does). */
class Device {
 public:
  explicit Device(void* stream = 0) : stream_(stream) {}
  double* axpy(double a, const double* x, const double* y, size_t length, double* out) const {
    check(ves3d_dev_axpy(a, x, y, length, out, stream_), "Device::axpy");
    return out;
  }
  double AlgebraicDot(const double* x, const double* y, size_t length) const {
    double r = 0;
    check(ves3d_dev_algebraic_dot(x, y, length, &r, stream_), "Device::AlgebraicDot");
    return r;
  }
  double* Transpose(const double* in, size_t height, size_t width, double* out) const {
    check(ves3d_dev_transpose(in, height, width, out, stream_), "Device::Transpose");
    return out;
  }
  double* Reduce(const double* x, int x_dim, const double* w, const double* quad_w, size_t stride, size_t ns,
                 double* x_dw) const {
    check(ves3d_dev_reduce(x, x_dim, w, quad_w, stride, ns, x_dw, stream_), "Device::Reduce");
    return x_dw;
  }
  double* gemm(const char* transA, const char* transB, const int* m, const int* n, const int* k, const double* alpha,
               const double* A, const int* lda, const double* B, const int* ldb, const double* beta, double* C,
               const int* ldc) const {
    check(ves3d_dev_gemm(*transA, *transB, *m, *n, *k, *alpha, A, *lda, B, *ldb, *beta, C, *ldc, stream_),
          "Device::gemm");
    return C;
  }
  /* AggregateRotation(sh_order, nlat, nlong, n_vec, n_sub, mat, vec, wrk, res, n_stream):
   * res[n_vec jj + ii] = (mat with columns shifted by jj per latitude) . vec[ii], for every
   * longitude jj; vec, wrk, res are host arrays of device pointers (wrk is not used). */
  void AggregateRotation(int sh_order, int nlat, int nlong, int n_vec, const int* n_sub, const double* mat,
                         const double** vec, double** wrk, double** res, int n_stream = 1) const {
    check(ves3d_dev_aggregate_rotation(sh_order, nlat, nlong, n_vec, n_sub, mat, vec, wrk, res, n_stream, stream_),
          "Device::AggregateRotation");
  }

 private:
  void* stream_;
};

/* SphericalHarmonics::RotateAll / MovePole on device pointers: S [n_vec][3][p(p+2)] ->
 * R [n_vec][p+1][p][3][p(p+2)], grid point (t, j) moved to the pole. */
inline void RotateAll(const double* S, long n_vec, int p, double* R, void* stream = 0) {
  check(ves3d_sht_rotate_all(S, n_vec, p, R, stream), "RotateAll");
}

/* WriteVTK(S, p0, p1, fname, period, v_ptr, comm) (src/StokesVelocity.cc:773-993): the
 * surfaces S (and the field v, or NULL) of order p0, host arrays [n_ves][3][(p0+1) 2p0],
 * taken to order p1 on the GPU and written as <fname>_<rank>.vtp, plus <fname>.pvtp from
 * rank 0. The communicator becomes its rank and size. */
template <class Vec>
void WriteVTK(const Vec& S, long p0, long p1, const char* fname, double period = 0, const Vec* v_ptr = 0,
              int rank = 0, int n_ranks = 1) {
  const size_t per = (size_t)3 * 2 * p0 * (p0 + 1);
  if (S.size() % per) throw Error(VES3D_ERR_ARG, "WriteVTK: size is not a multiple of 3 (p0+1) 2p0");
  if (v_ptr && v_ptr->size() != S.size()) throw Error(VES3D_ERR_ARG, "WriteVTK: field size differs from S");
  const long n_ves = (long)(S.size() / per);
  check(ves3d_vtk_write(n_ves ? &S[0] : 0, v_ptr && n_ves ? &(*v_ptr)[0] : 0, n_ves, (int)p0, (int)p1, fname, period,
                        rank, n_ranks, /*is_device=*/0),
        "WriteVTK");
}

/* Device<GPU>::DirectStokes(src, den, qw, src_stride, trg_stride, n_surfs, trg,
 * trg_idx_head, trg_idx_tail, pot) on device pointers (cuda_stokes). */
inline void DirectStokes(const double* src, const double* den, const double* qw, size_t src_stride,
                         size_t trg_stride, size_t n_surfs, const double* trg, size_t trg_idx_head,
                         size_t trg_idx_tail, double* pot, void* stream = 0) {
  check(ves3d_cuda_stokes_f64((int)src_stride, (int)trg_stride, (int)n_surfs, (int)trg_idx_head, (int)trg_idx_tail,
                              trg, src, den, pot, qw, stream),
        "DirectStokes");
}

/* Device<GPU>::DirectStokesDoubleLayer(src, norm, den, qw, src_stride, trg_stride, n_surfs,
 * trg, trg_idx_head, trg_idx_tail, pot) on device pointers (cuda_stokes_double_layer);
 * qw may be NULL. */
inline void DirectStokesDoubleLayer(const double* src, const double* norm, const double* den, const double* qw,
                                    size_t src_stride, size_t trg_stride, size_t n_surfs, const double* trg,
                                    size_t trg_idx_head, size_t trg_idx_tail, double* pot, void* stream = 0) {
  check(ves3d_cuda_stokes_double_layer_f64((int)src_stride, (int)trg_stride, (int)n_surfs, (int)trg_idx_head,
                                           (int)trg_idx_tail, trg, src, norm, den, pot, qw, stream),
        "DirectStokesDoubleLayer");
}

/* Device<GPU>::DirectStokes for float (cuda_stokes's single-precision overload,
 * src/CudaKernels.cu:751-761): float device arrays; qw may be NULL. */
inline void DirectStokes(const float* src, const float* den, const float* qw, size_t src_stride, size_t trg_stride,
                         size_t n_surfs, const float* trg, size_t trg_idx_head, size_t trg_idx_tail, float* pot,
                         void* stream = 0) {
  check(ves3d_cuda_stokes_f32((int)src_stride, (int)trg_stride, (int)n_surfs, (int)trg_idx_head, (int)trg_idx_tail,
                              trg, src, den, pot, qw, stream),
        "DirectStokes");
}

/* MovePole<Container, Operators> (include/MovePole.h:16-23): setOperands(arr, num) takes
 * num device arrays of grid functions of order p (n_funs[i] functions each, [n][(p+1) 2p]);
 * operator()(trg_i, trg_j, results) writes into results[i] those functions rotated so that
 * grid point (trg_i, trg_j) sits at the x = -1 pole (the reference's Direct scheme; through
 * the coefficients, exact on degrees < p). Only the Direct scheme is offered. */
class MovePole {
 public:
  enum Scheme { Direct = 0 };
  explicit MovePole(int sh_order, void* stream = 0) : p_(sh_order), stream_(stream), arr_(0), n_funs_(0), num_(0) {}
  void setOperands(const double* const* arr, const long* n_funs, int num, Scheme rot_scheme = Direct) {
    (void)rot_scheme;
    arr_ = arr;
    n_funs_ = n_funs;
    num_ = num;
  }
  void operator()(int trg_i, int trg_j, double* const* results) const {
    for (int i = 0; i < num_; i++)
      check(ves3d_move_pole(arr_[i], n_funs_[i], p_, trg_i, trg_j, results[i], stream_), "MovePole");
  }

 private:
  int p_;
  void* stream_;
  const double* const* arr_;
  const long* n_funs_;
  int num_;
};

/* Surface (include/Surface.h:38-77) of n_ves vesicles of order p on host arrays (positions
 * and fields AxisMajor [n_ves][3][(p+1) 2p], scalars [n_ves][(p+1) 2p]): geometry
 * (normal, area element, mean and Gaussian curvature), grad, div, linearizedMeanCurv,
 * area, volume, getCenters. diff_filter_freq: the low-pass filter of the differential
 * operators (0 none, -1 2p/3, > 0 the highest degree kept). */
template <class Real>
class Surface {
 public:
  Surface(int sh_order, const Real* x_in, size_t n, int diff_filter_freq = 0, int device = -1)
      : sv_(0), p_(sh_order), nv_(0) {
    check(ves3d_sv_create(sh_order, 2 * sh_order, VES3D_PREC_FP64, device, &sv_), "Surface");
    if (diff_filter_freq) check(ves3d_sv_set_surface_filter(sv_, diff_filter_freq), "Surface");
    setPosition(x_in, n);
  }
  ~Surface() { ves3d_sv_destroy(sv_); }
  void setPosition(const Real* x, size_t n) {
    const size_t per = 3 * ngrid();
    if (n == 0 || n % per) throw Error(VES3D_ERR_ARG, "Surface: size is not a multiple of 3 (p+1) 2p");
    nv_ = (long)(n / per);
    check(ves3d_sv_set_src_coord(sv_, x, nv_, 0), "Surface::setPosition");
  }
  int getNumberOfSurfaces() const { return (int)nv_; }
  int getShOrder() const { return p_; }
  /* unit outward normal [n_ves][3][Ngrid], area element W, mean curvature H (sphere of
   * radius R: -1/R), Gaussian curvature K, each [n_ves][Ngrid] */
  void getNormal(std::vector<Real>& n) const { geometry_part(4, 3, n); }
  void getAreaElement(std::vector<Real>& w) const { geometry_part(3, 1, w); }
  void getMeanCurv(std::vector<Real>& h) const { geometry_part(13, 1, h); }
  void getGaussianCurv(std::vector<Real>& k) const { geometry_part(14, 1, k); }
  void grad(const Real* f_in, Real* grad_f_out) const {
    check(ves3d_sv_surface_op(sv_, VES3D_OP_GRAD, f_in, grad_f_out, 0), "Surface::grad");
  }
  void div(const Real* f_in, Real* div_f_out) const {
    check(ves3d_sv_surface_op(sv_, VES3D_OP_DIV, f_in, div_f_out, 0), "Surface::div");
  }
  void linearizedMeanCurv(const Real* x_new, Real* h_lin) const {
    check(ves3d_sv_surface_op(sv_, VES3D_OP_LIN_MEANCURV, x_new, h_lin, 0), "Surface::linearizedMeanCurv");
  }
  void area(std::vector<Real>& a) const {
    a.resize(nv_);
    check(ves3d_sv_integrals(sv_, &a[0], 0, 0, 0), "Surface::area");
  }
  void volume(std::vector<Real>& v) const {
    v.resize(nv_);
    check(ves3d_sv_integrals(sv_, 0, &v[0], 0, 0), "Surface::volume");
  }
  void getCenters(std::vector<Real>& c) const {
    c.resize(3 * nv_);
    check(ves3d_sv_integrals(sv_, 0, 0, &c[0], 0), "Surface::getCenters");
  }

 private:
  size_t ngrid() const { return (size_t)2 * p_ * (p_ + 1); }
  // components [c0, c0 + nc) of the geometry record [n_ves][15][Ngrid]
  void geometry_part(int c0, int nc, std::vector<Real>& out) const {
    const size_t ng = ngrid();
    std::vector<Real> geo((size_t)nv_ * 15 * ng);
    check(ves3d_sv_surface_op(sv_, VES3D_OP_GEOMETRY, 0, &geo[0], 0), "Surface geometry");
    out.resize((size_t)nv_ * nc * ng);
    for (long v = 0; v < nv_; v++)
      for (int c = 0; c < nc; c++)
        for (size_t i = 0; i < ng; i++) out[((size_t)v * nc + c) * ng + i] = geo[((size_t)v * 15 + c0 + c) * ng + i];
  }
  Surface(const Surface&);
  Surface& operator=(const Surface&);
  ves3d_sv* sv_;
  int p_;
  long nv_;
};

}  // namespace ves3d_b200

#endif /* VES3D_B200_HPP */
