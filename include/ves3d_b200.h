/* ves3d_b200 -- B200-native StokesVelocity path for Ves3D, C ABI.
 *
 * Every entry point returns an int status (0 = VES3D_OK) and never aborts; the
 * message of the last failure on the calling thread is ves3d_last_error().
 * Plain pointers and sizes only. Pointers documented as "device" are CUDA device
 * pointers on the context's device; "host" pointers are ordinary host memory
 * (pageable or pinned; the library stages through its own pinned buffers).
 *
 * Layouts follow the reference's containers (AxisMajor, src/Scalars.cc:36-44):
 *   surface field   [n_ves][3][(p+1)*2p]   latitude-major Gauss-Legendre x uniform grid
 *   SH coefficients [n_fun][p*(p+2)]        blocks by Fourier index, degrees m..p
 *                                            (src/SphericalHarmonics.cc:32-38)
 *   self matrix     [n_ves][3*Ncoef][3*Ncoef] row = input density coefficient,
 *                                            column = output velocity coefficient
 */
#ifndef VES3D_B200_H
#define VES3D_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum ves3d_status {
  VES3D_OK = 0,
  VES3D_ERR_ARG = 1,      /* invalid argument (sizes, orders, null pointers) */
  VES3D_ERR_CUDA = 2,     /* a CUDA runtime call failed */
  VES3D_ERR_NOMEM = 3,    /* device or pinned host allocation failed */
  VES3D_ERR_STATE = 4,    /* call out of order (e.g. eval before set_src_coord) */
  VES3D_ERR_NODEV = 5,    /* no CUDA device / not an sm_100 device */
  VES3D_ERR_NUMERIC = 6,  /* non-finite input or result detected */
  VES3D_ERR_IO = 7        /* a file could not be written */
};

enum ves3d_precision {
  VES3D_PREC_FP64 = 0,    /* plain form: FP64 throughout */
  VES3D_PREC_MIXED = 1    /* FP32 far field with compensated sums; FP64 pole quadrature */
};

int ves3d_version(void);
const char* ves3d_last_error(void);
/* Number of kernels this library launched since load (all entry points). */
long long ves3d_kernel_launches(void);

/* ---------------------------------------------------------------------------
 * StokesVelocity operator context.
 * Replaces StokesVelocity<Real> (include/StokesVelocity.h:16-44,
 * src/StokesVelocity.cc:11-539) for surface targets, single and double layer:
 *   StokesVelocity(sh_order, sh_order_up)      -> ves3d_sv_create
 *   SetSrcCoord(S, up_self, up)                -> ves3d_sv_set_src_coord
 *   SetDensitySL(f)                            -> ves3d_sv_set_density_sl
 *   SetDensityDL(f)                            -> ves3d_sv_set_density_dl
 *   operator()(vel)                            -> ves3d_sv_eval
 * The far field is the exact all-pairs sum over other vesicles' grid points
 * (StokesAlltoAll - DirectStokesKernel, src/InterfacialVelocity.cc:1261-1291) in
 * place of the reference's PVFMM call (src/StokesVelocity.cc:477-490).
 * ------------------------------------------------------------------------- */
typedef struct ves3d_sv ves3d_sv;

/* sh_order_up <= 0 selects 2*sh_order (src/Parameters.cc:140). device < 0 uses the
 * current device. */
int ves3d_sv_create(int sh_order, int sh_order_up, int precision, int device, ves3d_sv** out);
int ves3d_sv_destroy(ves3d_sv* sv);
/* Bind a CUDA stream (cudaStream_t cast to void*) for all later work; NULL = the
 * context's own stream. */
int ves3d_sv_set_stream(ves3d_sv* sv, void* stream);

/* Source surfaces, AxisMajor [n_ves][3][Ngrid]. Invalidates the cached self matrices
 * (src/StokesVelocity.cc:26-57). is_device: 0 host pointer, 1 device pointer. */
int ves3d_sv_set_src_coord(ves3d_sv* sv, const double* S, long n_ves, int is_device);
/* Single-layer density, same layout as the surfaces (src/StokesVelocity.cc:66-97). */
int ves3d_sv_set_density_sl(ves3d_sv* sv, const double* f, int is_device);
/* Double-layer density, same layout (src/StokesVelocity.cc:107-142); NULL turns the double
 * layer off. While set, ves3d_sv_eval adds its velocity: the self part through the DL
 * matrices of StokesSingularInteg (src/StokesVelocity.cc:418-436) and the far part as the
 * exact FP64 sum over the other vesicles' points of the reference's double-layer kernel
 * (stokes_dl_uKernel, src/PVFMMInterface.cc:285-360) with unit outward normals and
 * densities times area and smooth weights (in both precision forms). Cleared by
 * ves3d_sv_set_src_coord; the implicit step applies the single layer alone. */
int ves3d_sv_set_density_dl(ves3d_sv* sv, const double* f, int is_device);
/* Copy the double-layer self matrices out, [n_ves][3Ncoef][3Ncoef] (needs a double-layer
 * density; builds them if the surfaces changed). */
int ves3d_sv_get_dl_matrix(ves3d_sv* sv, double* DL, int is_device);
/* Velocity at the surface points, same layout (src/StokesVelocity.cc:164-539).
 * Builds the self matrices first if the surfaces changed. */
int ves3d_sv_eval(ves3d_sv* sv, double* vel, int is_device);
/* StokesVelocity::SetTrgCoord(T) (src/StokesVelocity.cc:146-161): off-surface targets,
 * point-major [n_trg][3]; NULL (or n_trg = 0) returns to the surface points. Kept across
 * ves3d_sv_set_src_coord. */
int ves3d_sv_set_trg_coord(ves3d_sv* sv, const double* T, long n_trg, int is_device);
/* Velocity at the targets, point-major [n_trg][3]: the smooth quadrature over every surface
 * point (FP64) of the single layer and, when set, the double layer. The reference corrects
 * targets near a surface with its NearSingular module, which this build does not have:
 * the result is accurate only away from the surfaces (a few grid spacings). */
int ves3d_sv_eval_trg(ves3d_sv* sv, double* vel, int is_device);
/* Near-singular correction of the off-surface targets (NearSingular, src/NearSingular.cc,
 * as StokesVelocity composes it for SetTrgCoord targets, src/StokesVelocity.cc:475-500),
 * off by default. With it on, ves3d_sv_eval_trg sums every vesicle's smooth quadrature at
 * the far upsampling order p_up, and for a target closer than r_near = r_ves 2 / sqrt(p_up)
 * to a vesicle (r_ves: the largest distance of a surface point from its vesicle's
 * centroid) replaces that vesicle's contribution by the reference's interpolation: 8
 * Lagrange nodes along the line from the target's projection P on the surface (the
 * on-surface singular-quadrature velocity at P, plus +-g(P)/2 for the double layer
 * outside / inside, and the smooth quadrature at P + r_near (1 + (l - 1)/6) d, l = 1..7).
 * The projection is Gauss-Newton on the spherical-harmonic surface (the reference uses
 * quadratic patches); at most 4 near vesicles per target (more is an error). FP64; orders
 * up to 31. */
int ves3d_sv_set_near_singular(ves3d_sv* sv, int on);
/* r_near of the last corrected target evaluation and the number of (target, vesicle) pairs
 * it corrected. */
int ves3d_sv_near_info(ves3d_sv* sv, double* r_near, long* n_near);
/* The self part's upsampling order (sh_order_up_self, src/StokesVelocity.cc:26-57): new
 * operator tables, the self matrices rebuilt on next use. */
int ves3d_sv_set_order_up(ves3d_sv* sv, int sh_order_up);
int ves3d_sv_get_order_up(ves3d_sv* sv, int* sh_order_up);
/* StokesVelocity::MonitorError(tol) (src/StokesVelocity.cc:553-685): evaluates the double
 * layer of density 1 (single layer off), whose exact value is -1/2 on each surface and 0
 * on the others; err3 (may be NULL) = {max|self + 1/2|, 0 (no near-singular correction in
 * this build), max|far|}, *total (may be NULL) their sum. Moves the self upsampling order
 * by 2 up when the self error is above tol, down below tol/2, as the reference; the far
 * field is exact on the order-p grid and has no order to adapt. The densities set before
 * are restored. */
int ves3d_sv_monitor_error(ves3d_sv* sv, double tol, double* err3, double* total);
/* Build the self matrices now (the reference builds them lazily inside operator()). */
int ves3d_sv_setup(ves3d_sv* sv);
/* Copy the self matrices out, [n_ves][3Ncoef][3Ncoef]. */
int ves3d_sv_get_self_matrix(ves3d_sv* sv, double* SL, int is_device);
/* Split of the last eval into its parts: self (singular) and far (other vesicles),
 * each AxisMajor like vel. Either pointer may be NULL. */
int ves3d_sv_get_parts(ves3d_sv* sv, double* vel_self, double* vel_far, int is_device);
/* Device time in ms of the last setup / eval stages:
 * ms[0] self-matrix build, ms[1] self apply, ms[2] far-field kernel, ms[3] whole eval
 * (everything after the build). */
int ves3d_sv_stage_times(ves3d_sv* sv, float* ms);
/* Device time in ms of the far double layer's kernels in the last evaluation with a
 * double-layer density set (0 without one); a diagnostic of this library. */
int ves3d_sv_far_dl_time(ves3d_sv* sv, float* ms);
/* Device pointers of the context's resident buffers (for zero-copy callers):
 * which = 0 surfaces, 1 density, 2 velocity. Valid until the next set_src_coord. */
int ves3d_sv_device_buffer(ves3d_sv* sv, int which, double** ptr, size_t* n_elems);
/* Evaluate using the resident density buffer (which=1) and write the resident
 * velocity buffer (which=2); no host transfer. */
int ves3d_sv_eval_resident(ves3d_sv* sv);
/* Record the resident evaluation (density buffer -> velocity buffer: self part + far
 * field) as a CUDA graph on the context's stream (must not be the legacy default stream);
 * builds the self matrices first if needed and runs one eager evaluation. The graph reads
 * the buffers in place: write new densities into the density buffer and relaunch.
 * Invalidated by ves3d_sv_set_src_coord and ves3d_sv_set_stream. */
int ves3d_sv_capture_eval(ves3d_sv* sv);
/* Launch the captured evaluation on the context's stream, asynchronously (synchronise the
 * stream before reading the velocity buffer). */
int ves3d_sv_launch_eval_graph(ves3d_sv* sv);

/* Far-field launch-shape autotuner (no reference counterpart), process-wide, off by
 * default (or VES3D_AUTOTUNE=1): on the first far-field launch of a configuration
 * (precision, points, vesicles and their sizes) every candidate shape -- waves of CTAs
 * per SM in {4, 8, 16} x threads per CTA in {256, 384} (two targets each; the mixed form
 * 256 only, for its accuracy) -- is timed once with CUDA events and the fastest is kept.
 * Never tunes during stream capture. */
int ves3d_set_autotune(int on);
/* Fix the far-field launch shape instead (waves in {4, 8, 16}, threads per CTA in
 * {256, 384}, targets per thread 2); waves = 0 returns to the default / autotuned shape. */
int ves3d_set_far_shape(int waves, int threads, int targets_per_thread);
/* Text report of the tuned configurations, one line each ("key waves=W threads=T ms=M");
 * *len receives its length (buf may be NULL). */
int ves3d_autotune_report(char* buf, size_t cap, size_t* len);

/* ---------------------------------------------------------------------------
 * Polydisperse suspensions: vesicles of different SH orders p in one evaluation (the
 * reference needs one StokesVelocity per order; here the self part runs per order group
 * and the far field is one all-pairs launch over every point). Surfaces, densities and
 * velocities are the per-vesicle AxisMajor blocks [3][(p_v+1) 2 p_v] concatenated in
 * vesicle order; vesicles of equal order must be contiguous (runs of any order sequence).
 * Upsample order 2 p_v per vesicle.
 * ------------------------------------------------------------------------- */
typedef struct ves3d_svp ves3d_svp;
int ves3d_svp_create(int precision, int device, ves3d_svp** out);
int ves3d_svp_destroy(ves3d_svp* g);
int ves3d_svp_set_src_coord(ves3d_svp* g, const double* S, const int* orders, long n_ves, int is_device);
int ves3d_svp_set_density_sl(ves3d_svp* g, const double* f, int is_device);
/* SetDensityDL over the suspension (src/StokesVelocity.cc:107-142): the double layer of g
 * (same layout as f; NULL: off) is added to ves3d_svp_eval's velocity, each vesicle's self
 * part at its own order and the far double layer (FP64) over every point of the other
 * vesicles. Invalidated by ves3d_svp_set_src_coord and by an implicit solve under a
 * viscosity contrast (which takes the double-layer buffers for its operator). */
int ves3d_svp_set_density_dl(ves3d_svp* g, const double* gdl, int is_device);
/* Viscosity contrast of the suspension's implicit step (VesicleProps::viscosity_contrast,
 * as ves3d_sv_set_viscosity_contrast): lambda[n], n = 1 (every vesicle) or n_ves in vesicle
 * order; NULL or n = 0 removes it. The operator becomes (1 + lambda)/2 u - S[f] -
 * D[(1 - lambda) u] with the double layer over the whole suspension. */
int ves3d_svp_set_viscosity_contrast(ves3d_svp* g, const double* lambda, long n);
int ves3d_svp_setup(ves3d_svp* g);
int ves3d_svp_eval(ves3d_svp* g, double* vel, int is_device);
/* ms[0] self-matrix builds, ms[1] self parts, ms[2] far field, ms[3] whole last eval. */
int ves3d_svp_stage_times(ves3d_svp* g, float* ms);
/* The evaluation (self parts of every order group + the one far-field pass) recorded as a
 * CUDA graph on the context's stream (builds the self matrices and runs one eager pass
 * first); relaunch after ves3d_svp_set_density_sl with new densities. vel (may be NULL)
 * receives the velocity; invalidated by ves3d_svp_set_src_coord. */
int ves3d_svp_capture_eval(ves3d_svp* g);
int ves3d_svp_launch_eval_graph(ves3d_svp* g, double* vel, int is_device);
/* The globally implicit step of a polydisperse suspension (the reference's
 * InterfacialVelocity::updateImplicit over vesicles of one order,
 * src/InterfacialVelocity.cc:203-330, here across orders): the forces of each vesicle at
 * its own order, one single layer over every point between them, BiCGStab (FP64) or mixed
 * iterative refinement (mixed context) over the order groups' SH coefficients. Grid vectors
 * x0 (may be NULL: zero guess) and x are [u (the per-vesicle [3][ng_v] blocks); sigma (the
 * per-vesicle [ng_v] blocks)], 4 N doubles. Parameters, gravity and the preconditioner
 * (VES3D_PRECOND_*, rebuilt every refresh_every surface updates) apply to every order
 * group; tol and max_iter are in/out as in ves3d_sv_implicit_solve. */
int ves3d_svp_set_implicit_params(ves3d_svp* g, double dt, double bending_modulus, double shear_rate);
int ves3d_svp_set_gravity(ves3d_svp* g, double excess_density, double gx, double gy, double gz);
/* ves3d_sv_set_surface_filter for every order group (-1: 2p/3 of each group's order). */
int ves3d_svp_set_surface_filter(ves3d_svp* g, int filter_freq);
int ves3d_svp_set_precond(ves3d_svp* g, int scheme, int refresh_every);
int ves3d_svp_implicit_solve(ves3d_svp* g, const double* x0, double* x, double* tol, int* max_iter, int* code,
                             int is_device);
/* Last solve: outer refinements (FP64 matvecs) and inner iterations. */
int ves3d_svp_solver_stats(ves3d_svp* g, int* outer, int* inner);
/* Residual-minimising combination of n_cand (1..8) candidate grid vectors as the start of
 * the next ves3d_svp_implicit_solve (as ves3d_sv_implicit_combine; e.g. the last two
 * solutions, whose span holds the linear extrapolation in time). Candidate images come from
 * the operator the inner solves use (FP32 far field in a mixed context); the FP64
 * right-hand side is kept for the solve on the same surfaces. weights[n_cand]; relres
 * [n_cand + 1]: each candidate's relative residual, then the combination's. */
int ves3d_svp_implicit_combine(ves3d_svp* g, int n_cand, const double* const* cand, double* x0, double* weights,
                               double* relres, int is_device);

/* ---------------------------------------------------------------------------
 * Surface geometry, tractions and the globally implicit step on the context's surfaces
 * (Surface, src/Surface.cc:212-569; InterfacialForce, src/InterfacialForce.cc:21-125;
 * InterfacialVelocity::ImplicitMatvecPhysical / AssembleRhsVel, src/InterfacialVelocity.cc:
 * 716-979). Fields are AxisMajor per vesicle; scalars [n_ves][Ngrid], vectors
 * [n_ves][3][Ngrid]; the implicit unknown is [u (vector) ; sigma (scalar)].
 * ------------------------------------------------------------------------- */
enum ves3d_surface_op {
  VES3D_OP_GEOMETRY = 0,     /* out [n_ves][15][Ngrid]: E,F,G (/W^2), W, n (outward), cu, cv, H, K (sphere of radius R: H = -1/R) */
  VES3D_OP_GRAD = 1,         /* scalar -> vector: surface gradient                         */
  VES3D_OP_DIV = 2,          /* vector -> scalar: surface divergence                       */
  VES3D_OP_LIN_MEANCURV = 3, /* vector -> scalar: linearised mean curvature                */
  VES3D_OP_LIN_BENDING = 4,  /* vector -> vector: linear bending traction -kappa (Lap h + 2h(H^2-K)) n, h = H_lin(x) */
  VES3D_OP_BENDING = 5,      /* (in unused) -> vector: bending traction -kappa (Lap H + 2H(H^2-K)) n
                              * (bending_coeff = -bending_modulus, src/VesicleProps.cc:39-41) */
  VES3D_OP_TENSION = 6,      /* scalar -> vector: tension traction 2 sigma H n + grad sigma */
  VES3D_OP_IMPLICIT_MATVEC = 7, /* [u;sigma] -> [u - S f ; -div S f], f = linbend(dt u) + tension(sigma) */
  VES3D_OP_IMPLICIT_RHS = 8,    /* (in unused) -> [u_inf + S f_b ; div(u_inf + S f_b)]       */
  VES3D_OP_GRAVITY = 9          /* vector -> vector: excess_density (g . x) n                 */
};
/* Surface integrals per vesicle (Surface::area / volume / getCenters, src/Surface.cc:378-440,
 * with GaussLegendreIntegrator weights, src/GLIntegrator.cc:33-80): area[n_ves],
 * volume[n_ves], centers[n_ves][3]; any may be NULL. The normal is that of
 * Surface::updateFirstForms (x_theta x x_phi / W, outward), so volumes are positive. */
int ves3d_sv_integrals(ves3d_sv* sv, double* area, double* volume, double* centers, int is_device);
/* Parameters of the implicit step: time step, bending modulus, shear rate of the
 * background flow u = (rate * y, 0, 0). */
int ves3d_sv_set_implicit_params(ves3d_sv* sv, double dt, double kappa, double shear_rate);
/* Gravity (InterfacialForce::gravityForce, src/InterfacialForce.cc:127-184): the traction
 * excess_density (g . x) n enters the explicit jump with x = the positions and the
 * linearised jump with x = dt u. Default excess_density 0 (off), g = (0, 0, -1). */
/* The reference Surface's low-pass filter (SHTrans::lowPassFilter at diff_filter_freq,
 * src/Surface.cc:310-311, :336, :371, :564) on H, K, surface gradients, divergences and the
 * linearised curvature of the geometry ops and the implicit step: 0 turns it off (the
 * default), -1 keeps degrees <= 2p/3 (the reference's default), a positive value is the
 * highest degree kept. For the Surface-level operations (SurfaceTest's quantities). The
 * implicit step is best left unfiltered: the reference computes its forces at the
 * upsampled order 2p and filters at 2/3 of that (4p/3), which removes nothing resolved at
 * order p, while a filter at 2p/3 of p leaves the tension modes above the filter degree
 * without force and the implicit system singular (BiCGStab then stops at max_iter). */
int ves3d_sv_set_surface_filter(ves3d_sv* sv, int filter_freq);
int ves3d_sv_set_gravity(ves3d_sv* sv, double excess_density, double gx, double gy, double gz);
/* Viscosity contrast of the vesicles (interior / exterior viscosity; VesicleProps,
 * src/VesicleProps.cc:17-49): n = 1 value for all vesicles or one per vesicle, NULL (or
 * n = 0) for none. With a contrast other than 1 the implicit operator becomes
 * [(1 + l)/2 u - S[f] - D[(1 - l) u]; -div(S[f] + D[(1 - l) u])] (ImplicitApply,
 * src/InterfacialVelocity.cc:934-966) with the double layer of ves3d_sv_set_density_dl; the
 * right-hand side is unchanged (AssembleRhsVel, :717-745). The solve then uses the
 * context's double-layer density buffer (a density set before is cleared). */
int ves3d_sv_set_viscosity_contrast(ves3d_sv* sv, const double* lambda, long n);
int ves3d_sv_surface_op(ves3d_sv* sv, int op, const double* in, double* out, int is_device);
/* Solve the implicit system with BiCGStab in its Galerkin form (unknowns: SH coefficients
 * of u and sigma, ImplicitApply src/InterfacialVelocity.cc:982-1052; the reference's
 * default, params.pseudospectral = false). x0 (NULL = zero) and x are grid fields
 * [u; sigma]; on return *tol is the relative residual of the coefficient system,
 * *max_iter the iterations, *code the BiCGSReturn code (100 success, 101 max iterations,
 * 102/103 breakdown, 104 NaN). */
int ves3d_sv_implicit_solve(ves3d_sv* sv, const double* x0, double* x, double* tol, int* max_iter, int* code,
                            int is_device);

/* Iterations of the last implicit solve in the mixed form: FP64 residual evaluations of
 * the outer refinement loop, and inner (mixed-operator) BiCGStab iterations. In the mixed
 * form the solve is an iterative refinement: outer residuals with the FP64 operator,
 * corrections by BiCGStab on the mixed operator. */
int ves3d_sv_solver_stats(ves3d_sv* sv, int* outer, int* inner);

/* Preconditioner of the implicit solve (right preconditioning, BiCGStab::operator()
 * src/BiCGStab.cc:45-138 with its Precond argument):
 *   NONE           identity (default)
 *   DIAG_SPECTRAL  the reference's diagonal spectral scaling (ConfigurePrecond /
 *                  ImplicitPrecond, src/InterfacialVelocity.cc:665-713, 1055-1109)
 *   SELF_BLOCK     per-vesicle inverse of the isolated-vesicle operator (the implicit
 *                  operator with the self part of the single layer only); no counterpart in
 *                  the reference. Rebuilt on the first solve after the surfaces or dt /
 *                  kappa change: 4 nc operator applications plus one dense LU per vesicle
 *                  (cuSOLVER), stored in FP32, (4 nc)^2 * 4 bytes per vesicle.
 * The solution's accuracy is set by the tolerance on the true residual in every case. */
enum ves3d_precond { VES3D_PRECOND_NONE = 0, VES3D_PRECOND_DIAG_SPECTRAL = 1, VES3D_PRECOND_SELF_BLOCK = 2 };
int ves3d_sv_set_precond(ves3d_sv* sv, int scheme);
/* Rebuild the preconditioner only every `every` surface updates (default 1: after every
 * ves3d_sv_set_src_coord). A lagged preconditioner is one built for surfaces a few time
 * steps old; with right preconditioning it changes the iteration count, never the
 * tolerance the solution meets. A change of vesicle count, dt or kappa always rebuilds. */
int ves3d_sv_set_precond_refresh(ves3d_sv* sv, int every);
/* Device time of the last preconditioner build, ms[3] = {total, operator assembly, LU
 * factorisation and inversion} in ms, the bytes the preconditioner holds, and (age, may
 * be NULL) the surface updates since it was built (0: built for the current surfaces,
 * -1: not built yet or invalidated). */
int ves3d_sv_precond_info(ves3d_sv* sv, double* ms, size_t* bytes, int* age);

/* ---------------------------------------------------------------------------
 * Initial guess of the implicit solve. The reference starts each solve from the previous
 * step's solution (InterfacialVelocity::AssembleInitial, src/InterfacialVelocity.cc:874-919);
 * these entry points add a learned per-vesicle guess and a residual-based choice among
 * candidates. They have no counterpart in the reference. nc = p (p + 2) SH coefficients
 * per scalar function, in this library's coefficient order (index 0 = degree 0).
 * ------------------------------------------------------------------------- */
/* feat [n_ves][3 nc] (FP32): SH coefficients of each vesicle's x, y, z with the degree-0
 * coefficients set to 0 (translation removed). */
int ves3d_sv_guess_features(ves3d_sv* sv, float* feat, int is_device);
/* tgt [n_ves][4 nc] (FP32): SH coefficients of [u - u_inf; sigma] of the grid field x
 * (u_inf = (shear_rate * y, 0, 0), the background flow of the implicit step). */
int ves3d_sv_guess_targets(ves3d_sv* sv, const double* x, float* tgt, int is_device);
/* Inverse of ves3d_sv_guess_targets: grid [u; sigma] from coefficients tgt. */
int ves3d_sv_guess_from_targets(ves3d_sv* sv, const float* tgt, double* x0, int is_device);
/* Residual-minimising combination of n_cand (1..8) candidate guesses cand[i] (grid
 * [u; sigma], 4 N doubles each): x0 = sum_i weights[i] cand[i] minimises the true
 * residual |b - A x0| of the Galerkin system over the candidates' span (FP64 operator).
 * relres[0..n_cand-1] are the candidates' own relative residuals, relres[n_cand] that of
 * x0 (never above the smallest of them, up to rounding). Candidates with non-finite
 * images get weight 0. Costs n_cand + 1 FP64 operator applications. */
int ves3d_sv_implicit_combine(ves3d_sv* sv, int n_cand, const double* const* cand, double* x0, double* weights,
                              double* relres, int is_device);

/* Multilayer perceptron with hand-written BF16 tensor-core kernels (FP32 accumulation,
 * FP32 master weights, Adam): x -> [Linear -> ReLU] x (n_layers - 1) -> Linear. Inputs
 * are normalised by (x - in_shift) * in_scale; the network's output z maps to the
 * prediction z * out_scale + out_shift, and the loss is the mean squared error in the
 * normalised output space. Parameters are one flat FP32 vector: per layer W [in][out]
 * (row-major) then b [out]. Host pointers unless is_device. */
typedef struct ves3d_mlp ves3d_mlp;
int ves3d_mlp_create(int n_in, int n_hidden, int n_layers, int n_out, unsigned long long seed, ves3d_mlp** out);
int ves3d_mlp_destroy(ves3d_mlp* net);
long ves3d_mlp_num_params(ves3d_mlp* net);
int ves3d_mlp_get_params(ves3d_mlp* net, float* out);
int ves3d_mlp_set_params(ves3d_mlp* net, const float* in);
/* NULL arrays mean shift 0 / scale 1. */
int ves3d_mlp_set_scaling(ves3d_mlp* net, const float* in_shift, const float* in_scale, const float* out_shift,
                          const float* out_scale);
/* Y [batch][n_out] = prediction for X [batch][n_in]. */
int ves3d_mlp_forward(ves3d_mlp* net, const float* X, long batch, float* Y, int is_device);
/* Loss and its gradient with respect to the parameters (grads: host, may be NULL). */
int ves3d_mlp_gradients(ves3d_mlp* net, const float* X, const float* T, long batch, float* grads, double* loss,
                        int is_device);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) at learning rate lr; *loss is the loss
 * before the step. */
int ves3d_mlp_train_step(ves3d_mlp* net, const float* X, const float* T, long batch, float lr, double* loss,
                         int is_device);

/* BiCGStab on device vectors of length n (BiCGStab::operator(), src/BiCGStab.cc:45-138,
 * identity preconditioner); A computes y = A x on device pointers and returns 0 on success. */
typedef int (*ves3d_matvec_fn)(void* ctx, const double* x, double* y);
int ves3d_bicgstab_f64(ves3d_matvec_fn A, void* ctx, double* x, const double* b, size_t n, double* tol,
                       int* max_iter, int* code, void* stream);

/* ---------------------------------------------------------------------------
 * Spherical-harmonic transforms on device pointers (SHTrans, include/SHTrans.h:21-63;
 * math of SphericalHarmonics::Grid2SHC / SHC2Grid, src/SphericalHarmonics.cc:4-235).
 * ------------------------------------------------------------------------- */
/* grid at order p0 -> coefficients at order p1 (Grid2SHC). */
int ves3d_sht_forward(const double* X, long n_fun, int p0, int p1, double* S, void* stream);
/* coefficients at order p0 -> grid at order p1 (SHC2Grid), with optional longitude
 * (X_theta) and latitude (X_phi) derivatives as named by the reference; NULL skips. */
int ves3d_sht_backward(const double* S, long n_fun, int p0, int p1, double* X, double* X_theta,
                       double* X_phi, void* stream);
/* SHTrans::backward_d2u / backward_d2v / backward_duv (include/SHTrans.h:21-63): second
 * derivatives on the order-p grid of order-p coefficients S ([n_fun][p(p+2)], device),
 * u the latitude and v the longitude of the grid as in SHTrans; any output may be NULL.
 * Device pointers; builds the order-p tables for the call. */
int ves3d_sht_backward_d2(const double* S, long n_fun, int p, double* X_uu, double* X_vv, double* X_uv,
                          void* stream);
/* SphericalHarmonics::RotateAll (src/SphericalHarmonics.cc:363-449), the coefficient
 * rotation behind MovePole (include/MovePole.h:16-23): every vector field of S (device,
 * [n_vec][3][p(p+2)] coefficients) rotated so that each grid point (latitude t = 0..p,
 * longitude j = 0..p-1) moves to the north pole (its antipode to the south pole), into R
 * (device, [n_vec][p+1][p][3][p(p+2)]). MovePole::operator()(t, j, ...) for j < p is the
 * (t, j) slice. Builds the order-p rotation tables for the call. */
int ves3d_sht_rotate_all(const double* S, long n_vec, int p, double* R, void* stream);
/* MovePole<Container, Operators>::operator()(trg_i, trg_j, results) (include/MovePole.h:16-23,
 * src/MovePole.cc:159-195): n_fun grid functions X [n_fun][(p+1) 2p] (device) rotated so
 * that grid point (latitude trg_i, longitude trg_j), trg_j in [0, 2p), sits at the x = -1
 * pole, as the reference's precomputed rotations place it; Y [n_fun][(p+1) 2p] on the same
 * grid. Computed through the coefficients (Grid2SHC, the rotation of RotateAll for that
 * point, SHC2Grid): it equals the reference's Direct scheme on functions of degree < p and
 * differs from it on the degree-p (Nyquist) band, which a grid of 2p longitudes cannot
 * rotate exactly. Returns when the work is done. */
int ves3d_move_pole(const double* X, long n_fun, int p, int trg_i, int trg_j, double* Y, void* stream);
/* SHTrans's frequency filters (constructor, src/SHTrans.cc:8-45) written to a host array of
 * p(p+2) values in the per-function coefficient order (Fourier blocks, degrees ascending):
 * exponent <= 0 gives lowPassFilter's hard cut (1 for degree n <= filter_freq, else 0),
 * exponent > 0 lowPassFilterPoly's 1 - (n/filter_freq)^exponent for n < filter_freq, else 0
 * (the reference's default exponent is 4); filter_freq -1 means 2p/3. Host only. */
int ves3d_sht_filter_coeffs(int p, int filter_freq, double exponent, double* coeff);
/* SHTrans::ScaleFreq (src/SHTrans.cc:190-223): shc_out[f][c] = shc_in[f][c] * scale[c] for
 * n_fun functions of p(p+2) coefficients; device pointers, in place allowed. The arrays are
 * function-major (the layout of ves3d_sht_forward); the reference's SHTrans keeps each
 * frequency block of all functions together, with the same per-function scale order. */
int ves3d_sht_scale_freq(const double* shc_in, long n_fun, int p, const double* scale, double* shc_out,
                         void* stream);
/* SHTrans::lowPassFilter / lowPassFilterPoly (src/SHTrans.cc:172-188) of grid functions at
 * order p: analysis, the filter of ves3d_sht_filter_coeffs, synthesis; in place allowed. */
int ves3d_sht_lowpass(const double* in, long n_fun, int p, int filter_freq, double exponent, double* out,
                      void* stream);
/* SphericalHarmonics::SHC2Pole (src/SphericalHarmonics.cc:325-360): P[2 f + t] = the value
 * of function f at x = -1 (t = 0) and x = +1 (t = 1), from the m = 0 block of its order-p
 * coefficients S ([n_fun][p(p+2)], the layout of ves3d_sht_forward). Device pointers. */
int ves3d_sht_pole(const double* S, long n_fun, int p, double* P, void* stream);

/* ---------------------------------------------------------------------------
 * Device<GPU> primitives (include/Device.h:81-253) on device pointers; each returns when
 * its work on the stream is done.
 * ------------------------------------------------------------------------- */
/* Device::axpy (:158-160): out[i] = a x[i] + y[i], out may be y. */
int ves3d_dev_axpy(double a, const double* x, const double* y, size_t length, double* out, void* stream);
/* Device::AlgebraicDot (:228-229): *result (host) = sum_i x[i] y[i], fixed-order reduction. */
int ves3d_dev_algebraic_dot(const double* x, const double* y, size_t length, double* result, void* stream);
/* Device::Transpose (:225-226): out[j height + i] = in[i width + j], out of place. */
int ves3d_dev_transpose(const double* in, size_t height, size_t width, double* out, void* stream);
/* Device::Reduce (:181-183; src/DeviceCPU.cc:444-497): the smooth surface integral
 * x_dw[s x_dim + d] = sum_i x[(s x_dim + d) stride + i] w[s stride + i] quad_w[i] for ns
 * surfaces, or with x NULL x_dw[s] = sum_i w[s stride + i] quad_w[i] (the areas). */
int ves3d_dev_reduce(const double* x, int x_dim, const double* w, const double* quad_w, size_t stride, size_t ns,
                     double* x_dw, void* stream);
/* Device::gemm (:199-203): C = alpha op(A) op(B) + beta C in column-major BLAS semantics
 * (trans 'N', 'T' or 'C'), through cuBLAS. */
int ves3d_dev_gemm(char trans_a, char trans_b, int m, int n, int k, double alpha, const double* A, int lda,
                   const double* B, int ldb, double beta, double* C, int ldc, void* stream);
/* Device::AggregateRotation(sh_order, nlat, nlong, n_vec, n_sub, mat, vec, wrk, res, n_stream)
 * (include/Device.h:234-237; the argument order of the declaration and of Device<CPU>,
 * src/DeviceCPU.cc:646-680, which MovePole::updateEagerResults calls): for every longitude
 * jj < nlong and operand ii < n_vec, res[n_vec jj + ii] = Permute(mat, jj) . vec[ii], where
 * mat is an np x np rotation (np = nlat nlong, column-major) whose columns are shifted by
 * jj within every latitude block (CircShift / PermuteGpu), vec[ii] holds n_sub[ii] grid
 * functions of np values. vec and res are HOST arrays of DEVICE pointers, as in the
 * reference; wrk and n_stream are accepted and unused (the permuted matrix is never
 * formed). Returns when the work is done. (src/DeviceGPU.cc:314 defines the GPU version
 * with n_vec second, a different order from its declaration; this follows the
 * declaration.) */
int ves3d_dev_aggregate_rotation(int sh_order, int nlat, int nlong, int n_vec, const int* n_sub, const double* mat,
                                 const double* const* vec, double* const* wrk, double* const* res, int n_stream,
                                 void* stream);

/* ---------------------------------------------------------------------------
 * Direct Stokes sums on device pointers.
 * ves3d_cuda_stokes: same arguments and meaning as the reference's
 *   cuda_stokes(int src_m, int trg_m, int n, int t_head, int t_tail, const T* T,
 *               const T* S, const T* D, T* U, const T* Q)   (include/CudaKernels.h,
 *   src/CudaKernels.cu:1996-2006) i.e. Device<GPU>::DirectStokes
 *   (include/Device.h:205-209): per-surface single layer with weights Q, targets
 *   [t_head, t_tail) of each surface, AxisMajor strides src_m / trg_m, n surfaces.
 * ------------------------------------------------------------------------- */
/* ves3d_cuda_stokes_double_layer: the reference's cuda_stokes_double_layer(int src_m, int
 *   trg_m, int n, int t_head, int t_tail, T, S, N, D, U, Q) (src/CudaKernels.cu:895-918, i.e.
 *   Device<GPU>::DirectStokesDoubleLayer, src/DeviceGPU.cc:263-271; the declaration in
 *   include/CudaKernels.h:42 omits trg_m): per surface, targets [t_head, t_tail), sources
 *   with unit normals N and densities D, weights Q (NULL: none),
 *   U = 3/(4 pi) sum (r.n)(r.d) r / |r|^5 with r = target - source. */
int ves3d_cuda_stokes_double_layer_f64(int src_m, int trg_m, int n, int t_head, int t_tail, const double* T,
                                       const double* S, const double* N, const double* D, double* U, const double* Q,
                                       void* stream);
int ves3d_cuda_stokes_f64(int src_m, int trg_m, int n, int t_head, int t_tail, const double* T,
                          const double* S, const double* D, double* U, const double* Q, void* stream);
/* The single-precision overload cuda_stokes(..., const float* T, ...) (src/CudaKernels.cu:
 * 751-761, used by SINGLE_PREC builds of the reference): float arrays, FP32 pair
 * arithmetic, FP64 sums across 128-source tiles. Q may be NULL (unit weights) here and in
 * the double version. Both are asynchronous on the given stream. */
int ves3d_cuda_stokes_f32(int src_m, int trg_m, int n, int t_head, int t_tail, const float* T,
                          const float* S, const float* D, float* U, const float* Q, void* stream);

/* All-pairs interaction with the reference's VesInteraction handle signature
 * (include/VesInteraction.h:21, matched by StokesAlltoAll, include/CPUKernels.h:46-49):
 * HOST pointers, point-major xyz, np points; pot[t] = sum over all s of the Stokeslet
 * of den[s] (coincident points contribute nothing). *ctx may hold a library-owned
 * workspace between calls; free it with ves3d_interaction_free(ctx). Errors are
 * reported through ves3d_last_error() and leave pot filled with NaN. */
void ves3d_stokes_alltoall_f64(const double* src, const double* den, size_t np, double* pot, void** ctx);
void ves3d_interaction_free(void** ctx);
/* Same on device pointers, with an int status. */
int ves3d_stokes_alltoall_device_f64(const double* src, const double* den, size_t np, double* pot,
                                     void* stream);

/* All-to-all interaction that allocates nothing (no counterpart in the reference: it is
 * an addition of this library). For programs whose device memory is owned by another
 * allocator (a pool that has reserved the GPU already, or a framework that forbids
 * cudaMalloc/cudaFree between time steps), which cannot let the library allocate. Same
 * HOST-pointer arguments and result as ves3d_stokes_alltoall_f64, plus an optional
 * stream (NULL = legacy default stream); returns an int status. The call is synchronous:
 * it waits for its result on that stream before returning. Inputs are staged through one
 * fixed device array of
 * VES3D_NOALLOC_MAX_POINTS points (36 MiB, held by every GPU that loads the library
 * until exit); np above that is rejected with VES3D_ERR_ARG. On any error pot (3 np
 * doubles) is filled with NaN, as by the allocating call; np = 0 leaves it untouched.
 * The first call on each device does the set-up (looks up the array's device address and
 * keeps it): make it before any stream capture. The kept address does not survive
 * cudaDeviceReset. Calls share the array: calls whose GPU work overlaps race. */
#define VES3D_NOALLOC_MAX_POINTS 524288
int ves3d_stokes_alltoall_noalloc_f64(const double* src, const double* den, size_t np, double* pot,
                                      void* stream);

/* ---------------------------------------------------------------------------
 * VTK output of surfaces (WriteVTK, src/StokesVelocity.cc:773-993): one XML PolyData file
 * <fname>_<rank as 6 digits>.vtp per rank with raw appended data, and from rank 0 the index
 * <fname>.pvtp naming the n_ranks pieces. Per vesicle the points are the (p1+1) x 2p1 grid
 * of order p1 (latitude-major) followed by the poles at x = -1 and x = +1; the polygons are
 * 2p1 pairs of pole triangles, then p1 x 2p1 quads. The optional field becomes the point
 * data "value" (3 components). With period > 0 each vesicle is shifted by the multiple of
 * period nearest its mean point (the field is not shifted).
 * ------------------------------------------------------------------------- */
/* The writer alone, host only (no GPU needed): host arrays X1 (and V1)
 * [n_ves][3][(p1+1) 2p1] of grid values at order p1 and Xp (and Vp) [n_ves][3][2] of pole
 * values (x = -1, then x = +1); V1 and Vp NULL write no point data. */
int ves3d_vtk_write_grid(const double* X1, const double* Xp, const double* V1, const double* Vp, long n_ves,
                         int p1, const char* fname, double period, int rank, int n_ranks);
/* WriteVTK(S, p0, p1, fname, period, v_ptr, comm): positions X (and the optional field V,
 * NULL for none) [n_ves][3][(p0+1) 2p0] at order p0, host or device pointers, taken to order
 * p1 on the GPU (Grid2SHC at p0, SHC2Grid at p1, SHC2Pole) and written as above. */
int ves3d_vtk_write(const double* X, const double* V, long n_ves, int p0, int p1, const char* fname, double period,
                    int rank, int n_ranks, int is_device);

/* ---------------------------------------------------------------------------
 * Diagnostics (host only, no GPU needed): copy one of the FP64 operator tables the
 * library builds for (p0, p1) into out (capacity cap doubles); *n receives its length.
 * Names: "nodes0", "weights0", "nodes1", "smooth_w0", "sing_w", "mr", "ana_leg",
 * "ana_four", "syn1_leg", "syn1_dleg", "syn1_four", "syn1_dfour", "qp".
 * ------------------------------------------------------------------------- */
int ves3d_tables_export(int p0, int p1, const char* name, double* out, size_t cap, size_t* n);

#ifdef __cplusplus
}
#endif

#endif /* VES3D_B200_H */
