// Kernel launchers of the ves3d_b200 CUDA library (device pointers, one stream).
#pragma once

#include <string>
#include <cuda_runtime.h>

namespace ves3d {

inline int ncoef_(int p) { return p * (p + 2); }
inline int ngrid_(int p) { return 2 * p * (p + 1); }

// Device copies of the tables of one (p0, p1) pair (layouts as in sh_tables.h).
struct DevTables {
  int p0 = 0, p1 = 0;
  double *ana_four = nullptr, *ana_leg = nullptr;                   // Grid2SHC(p0, p0)
  double *syn0_leg = nullptr, *syn0_dleg = nullptr, *syn0_four = nullptr, *syn0_dfour = nullptr;
  double *syn1_leg = nullptr, *syn1_dleg = nullptr, *syn1_four = nullptr, *syn1_dfour = nullptr;
  double *synT_four = nullptr;                                      // [2p1][2p0]
  int *jf_of_coef = nullptr, *blk_off = nullptr, *m_of_coef = nullptr, *n_of_coef = nullptr;
  int *partner = nullptr, *is_sin = nullptr;
  double* mr = nullptr;
  int mr_total = 0;  // doubles in mr; (p0+1) equal parts, one per latitude rotation t
  int *mr_off = nullptr, *perm = nullptr, *perm_off = nullptr, *pos_in_block = nullptr;
  double *sing_w = nullptr, *smooth_w0 = nullptr, *qp = nullptr, *cos_tab = nullptr, *sin_tab = nullptr;
  double *syn0_d2leg = nullptr, *syn0_d2four = nullptr;
  // syn1_leg / syn1_dleg transposed to [latitude][coefficient] (contiguous per latitude)
  double *syn1_leg_t = nullptr, *syn1_dleg_t = nullptr;
};

// Geometry record per point: E, F, G (divided by W^2), W, n[3], cu[3], cv[3], H, K.
constexpr int kGeoComps = 15;

typedef int (*MatVecFn)(void* ctx, const double* x, double* y);

int launch_analysis(const double* in, long nfun, int pin, int pout, const double* four, const double* leg,
                    const int* jf, double* out, cudaStream_t st);
// Grid2SHC(p, p): tensor-core kernel where instantiated (2p % 8 == 0), generic otherwise;
// VES3D_TC_ANALYSIS=0 forces the generic kernel.
int launch_grid2shc(const double* in, long nfun, int p, const double* four, const double* leg, const int* jf,
                    double* out, cudaStream_t st);
// The same for FP32 grid values (FP64 arithmetic and output), p in {4, 8, 12, 16}.
int launch_grid2shc_f32(const float* in, long nfun, int p, const double* four, const double* leg, const int* jf,
                        double* out, cudaStream_t st);
// shc_out[f][c] = shc_in[f][c] * scale[c] for nfun functions of nc coefficients
int launch_scale_freq(const double* in, long nfun, int nc, const double* scale, double* out, cudaStream_t st);
// SHC2Pole: P[2 f + t] = values of function f at x = -1 (t = 0) and x = +1 (t = 1) from its
// order-p0 coefficients; qp = [2][p0+1] pole weights.
int launch_shc2pole(const double* S, long nfun, int p0, const double* qp, double* P, cudaStream_t st);
int launch_synthesis(const double* S, long nfun, int p0, int q, const double* leg, const double* dleg,
                     const double* four, const double* dfour, const int* blk_off, double* X, double* Xt,
                     double* Xp, cudaStream_t st);

// RotateAll with dof = 3 (src/SphericalHarmonics.cc:363-449):
// S [nv][3][Ncoef] -> R [nv][p0+1][p0][3][Ncoef].
int launch_rotate_all(const double* S, long nv, const DevTables& T, double* R, cudaStream_t st);
// One rotation (MovePole): S [n_fun][Ncoef] -> R [n_fun][Ncoef] with grid point (t, j),
// j in [0, 2 p0), moved to the x = -1 pole.
int launch_rotate_one(const double* S, long n_fun, int t, int j, const DevTables& T, double* R, cudaStream_t st);
// Device::AggregateRotation: res = mat . (vec with longitudes shifted by jj), see device_prims.cu
int launch_aggregate_rotation(const double* mat, int nlat, int nlong, int jj, const double* vec, int nsub,
                              double* res, cudaStream_t st);
// Near-singular correction at off-surface targets (near_kernels.cu)
constexpr int kNearMax = 4;  // near vesicles per target
int launch_centroid_radius(const double* X, long nv, int p, double* cen_r, unsigned long long* rmax_bits,
                           cudaStream_t st);
int launch_near_find(const double* trg, long M, const double* cen_r, long nv, const double* pos_up, int p_up,
                     double r_near, int* count, int* near_v, int* near_k, cudaStream_t st);
int launch_near_correct(const double* trg, long M, const int* count, const int* near_v, const int* near_k,
                        const double* Sx, const double* Vc, const double* Gc, const double* pos_up,
                        const double* den_up, const double* nrm_up, const double* dden_up, const double* theta_up,
                        const int* blk_off, int p, int p_up, double r_near, double* corr, double* vel,
                        cudaStream_t st);
// the single-precision cuda_stokes
int launch_direct_stokes_f32(int src_m, int trg_m, int n, int t_head, int t_tail, const float* T, const float* S,
                             const float* D, float* U, const float* Q, cudaStream_t st);
// Singular kernel (src/SphericalHarmonics.cc:971-1068) for nrot rotated surfaces:
// X, Xt, Xp [nrot][3][M1], R [nrot][3][Ncoef] -> K [nrot][2][6][M1].
int launch_singular_sl(const double* X, const double* Xt, const double* Xp, const double* R, long nrot,
                       const DevTables& T, double* K, cudaStream_t st);
// the same pole-target kernel for the double layer (DLMatrix of StokesSingularInteg)
int launch_singular_dl(const double* X, const double* Xt, const double* Xp, const double* R, long nrot,
                       const DevTables& T, double* K, cudaStream_t st);
// RotateTranspose with dof = 12 (:452-541) fused with the Rearrange (:1090-1172):
// C [nv][p0+1][p0][2][6][Ncoef] -> SL3 [nv][3][Ncoef][3][Ngrid].
int launch_rotate_transpose_scatter(const double* C, long nv, const DevTables& T, double* SL3, cudaStream_t st);
// The same from FP32 transposed-DFT results (the tensor-core build's), rotated back in FP32,
// into an FP32 grid.
int launch_rotate_transpose_f32(const float* C, long nv, const DevTables& T, float* SL3, cudaStream_t st);
// The same from the FP64 ring's results (rounded to FP32 when staged), at the orders it is
// instantiated for (the mixed form's self matrices at p = 12 and 24).
bool rotate_transpose_f32_from_f64_supported(int p0);
int launch_rotate_transpose_f32(const double* C, long nv, const DevTables& T, float* SL3, cudaStream_t st);
// Fused per-rotation build (FP64 tensor cores): R [nrot][3][Nc] -> C [nrot][2][6][Nc],
// i.e. upsampled synthesis + singular kernel + transposed synthesis in one kernel.
bool fused_build_supported(int p0, int p1);
int launch_build_ring(const double* R, long nrot, const DevTables& T, double* C, cudaStream_t st);
// Mixed form of the fused build: the DFT GEMMs on tcgen05 tensor cores as split-BF16
// products with FP32 accumulation (Legendre sums, kernel and targets FP64); same layouts.
bool tc_build_supported(int p0, int p1);
int launch_build_ring_tc(const double* R, long nrot, const DevTables& T, float* C, cudaStream_t st);
// Error flag of the tensor-core build (a bounded wait ran out), optionally reset.
int tc_build_error(bool reset);
// V[v] = F[v] . SL[v] (src/StokesVelocity.cc:397-416), n = 3 Ncoef.
int launch_self_gemv(const double* F, const double* SL, long nv, int n, double* V, cudaStream_t st,
                     bool accumulate = false);
// nvec density vectors per vesicle, layout [q][nv][n]; nvec <= 8
int launch_self_gemv_multi(const double* F, const double* SL, long nv, int nvec, int n, double* V, cudaStream_t st,
                           bool accumulate = false);
// out[i] = c[(i / per) % nc] x[i] + beta z[i] (z null: the first term alone): a per-vesicle
// coefficient (nc vesicles, per values each, repeated over batched copies)
int launch_scale_vesicles(const double* x, long n, long per, const double* c, long nc, const double* z, double beta,
                          double* out, cudaStream_t st);
// area element |X_theta x X_phi| and far-field sources: pos/den point-major [N][3],
// den = f * area * smooth_w[lat]; X, f, Xt, Xp AxisMajor [nv][3][ng].
int launch_far_sources(const double* X, const double* f, const double* Xt, const double* Xp, long nv, int p0,
                       const double* smooth_w, double* area, double* pos, double* den, cudaStream_t st);
// den only, from a stored area element.
int launch_far_density(const double* f, const double* area, long nv, int p0, const double* smooth_w, double* den,
                       cudaStream_t st);
// Far field: out (AxisMajor per vesicle) = add (may be null) + sum over other vesicles'
// sources; far_out (may be null) receives the far part alone. off [nves+1] point offsets,
// max_nt the largest vesicle; part is a [part_cap_segments][N][3] FP64 work buffer.
// mixed selects the packed-FP32 pair arithmetic with FP64 accumulation.
// With nseg_out given, only the segment kernels run (no reduce) and their count comes back
// for launch_far_reduce, which may then run on another stream after the self part.
int launch_far(bool mixed, const double* pos, const double* den, const long* off, long nves, long N, int max_nt,
               const double* add, double* out, double* far_out, double* part, long part_cap_segments,
               cudaStream_t st, int* nseg_out = nullptr);
int launch_far_reduce(const double* part, int nseg, const long* off, long nves, long N, const double* add, double* out,
                      double* far_out, cudaStream_t st, const double* part2 = nullptr, int nseg2 = 0,
                      double scale2 = 0.0);
// Far double layer over the points of the other vesicles (FP64, or packed FP32 pairs with
// FP64 sub-tile sums when mixed): pos, unit normals nrm and densities dden (times area and
// weights) point-major; the segments' unscaled partials go to part (at most
// part_cap_segments), their count to *nseg_out, for launch_far_reduce's second set with
// scale kDl.
int launch_far_dl(bool mixed, const double* pos, const double* nrm, const double* dden, const long* off, long nves,
                  long N, int max_nt, double* part, long part_cap_segments, cudaStream_t st, int* nseg_out);
// Velocity at M off-surface targets (point-major [M][3]) from N surface points: single
// layer of den, plus with nrm non-null the double layer of nrm and dden (all point-major,
// densities times area and weights).
int launch_targets_f64(const double* pos, const double* den, const double* nrm, const double* dden, long N,
                       const double* trg, long M, double* out, cudaStream_t st);
// Unit outward normals (X_theta x X_phi) / |X_theta x X_phi| of nv surfaces at order p0,
// AxisMajor derivatives in, point-major [N][3] out.
int launch_unit_normals(const double* Xt, const double* Xp, long nv, int p0, double* nrm, cudaStream_t st);
// Device<GPU>::DirectStokesDoubleLayer (cuda_stokes_double_layer): per surface, AxisMajor,
// sources with unit normals N and densities D, weights Q (null: none).
int launch_direct_stokes_dl_f64(int src_m, int trg_m, int n, int t_head, int t_tail, const double* T,
                                const double* S, const double* N, const double* D, double* U, const double* Q,
                                cudaStream_t st);
constexpr long kFarMaxSegments = 32;
// Vesicles [v0, v0 + nv) all with nt points: one far-field launch each, sized for nt.
struct FarGroup {
  long v0, nv;
  int nt;
};
// far-field launch-shape autotuner (far_kernels.cu)
int set_autotune(int on);
int set_far_shape(int waves, int nthr, int tpt);
std::string autotune_report();
int launch_far_groups(bool mixed, const double* pos, const double* den, const long* off, long nves, long N,
                      const FarGroup* groups, int ngroups, const double* add, double* out, double* far_out,
                      double* part, long part_cap_segments, cudaStream_t st, int* nseg_out = nullptr);
// launch_far_dl over order groups (a polydisperse suspension): per-group block shapes, one
// segment layout.
int launch_far_dl_groups(bool mixed, const double* pos, const double* nrm, const double* dden, const long* off,
                         long nves, long N, const FarGroup* groups, int ngroups, double* part, long part_cap_segments,
                         cudaStream_t st, int* nseg_out);
// out = a + b elementwise.
int launch_add(const double* a, const double* b, long n, double* out, cudaStream_t st);
// All pairs, point-major in/out (StokesAlltoAll semantics).
int launch_alltoall_f64(const double* pos, const double* den, long np, double* pot, cudaStream_t st);
// Per-surface DirectStokes with weights (cuda_stokes semantics).
int launch_direct_stokes_f64(int src_m, int trg_m, int n, int t_head, int t_tail, const double* T,
                             const double* S, const double* D, double* U, const double* Q, cudaStream_t st);

// surface geometry and tractions (geometry_kernels.cu); fields AxisMajor [nv][comp][ng]
int launch_geometry(const double* xu, const double* xv, const double* xuu, const double* xuv, const double* xvv,
                    long nv, int ng, double* geo, cudaStream_t st);
int launch_grad_combine(const double* fu, const double* fv, const double* geo, long nv, int ng, double* out,
                        cudaStream_t st,
    long geo_nv = 0);
int launch_div_combine(const double* Fu, const double* Fv, const double* geo, long nv, int ng, double scale,
                       double* out, cudaStream_t st,
    long geo_nv = 0);
int launch_linH_combine(const double* duu, const double* duv, const double* dvv, const double* geo, long nv, int ng,
                        double* out, cudaStream_t st,
    long geo_nv = 0);
int launch_bend_combine(const double* h, const double* lap, const double* geo, long nv, int ng, double kappa,
                        const double* add, double* out, cudaStream_t st,
    long geo_nv = 0);
int launch_tension_combine(const double* sigma, const double* gsig, const double* geo, long nv, int ng,
                           const double* add, double* out, cudaStream_t st,
    long geo_nv = 0);
int launch_shear(const double* X, long nv, int ng, double rate, double* out, cudaStream_t st);
// out = add + drho (g . x) n  (g: host array of 3)
int launch_gravity_combine(const double* x, const double* geo, long nv, int ng, double drho, const double* g,
                           const double* add, double* out, cudaStream_t st, long geo_nv = 0);
// per vesicle {area, volume, centre x, y, z} (Xu latitude, Xv longitude derivatives)
int launch_integrals(const double* X, const double* Xu, const double* Xv, const double* w, long nv, int p,
                     double* out, cudaStream_t st);

// BiCGStab (bicgstab.cu)
int dot_f64(const double* x, const double* y, long n, double* scratch, double* result, cudaStream_t st);
int lincomb_f64(long n, double a, const double* x, double b, const double* y, double c, const double* z, double* out,
                cudaStream_t st);
size_t bicgstab_workspace_doubles(long n);
double* bicgstab_dot_scratch(double* ws, long n);  // scratch of dot_f64 inside a workspace
// P (optional, NULL = identity): right preconditioner y = P x
int bicgstab_run(MatVecFn A, void* ctx, double* x, const double* b, long n, double* tol, int* max_iter, int* code,
                 double* ws, cudaStream_t st, MatVecFn P = nullptr, void* pctx = nullptr);

}  // namespace ves3d
