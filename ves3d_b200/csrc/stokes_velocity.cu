// StokesVelocity operator context and the C ABI (include/ves3d_b200.h).
//
// Pipeline (plain FP64 form), all on one stream:
//   set_src_coord: X -> Sx = Grid2SHC(X); (X_theta, X_phi) = SHC2Grid(Sx) at p;
//                  area = |X_theta x X_phi|; far-field source positions.
//   setup        : per chunk of vesicles: RotateAll(Sx) -> SHC2Grid(p -> p_up, +grads)
//                  -> singular kernel -> SHC2GridTranspose(p_up -> p) -> RotateTranspose
//                  + Rearrange -> Grid2SHC -> SL [v][3Nc][3Nc]
//                  (SphericalHarmonics::StokesSingularInteg_, src/SphericalHarmonics.cc:954-1180)
//   eval         : Fc = Grid2SHC(f); Vc = Fc . SL; Vself = SHC2Grid(Vc)
//                  (src/StokesVelocity.cc:385-473); den = f * area * qw;
//                  vel = Vself + sum over other vesicles (exact all-pairs far field).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include <cusolverDn.h>

#include "common.cuh"
#include "kernels.h"
#include "sh_tables.h"

namespace ves3d {

static thread_local char g_err[1024] = {0};

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

std::atomic<long long>& launch_counter() {
  static std::atomic<long long> c{0};
  return c;
}

template <class T>
static int dalloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) return VES3D_OK;
  VES3D_CK(cudaMalloc((void**)p, n * sizeof(T)));
  return VES3D_OK;
}

template <class T>
static int dupload(T** p, const std::vector<T>& v, cudaStream_t st) {
  int s = dalloc(p, v.size());
  if (s) return s;
  if (!v.empty()) VES3D_CK(cudaMemcpyAsync(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return VES3D_OK;
}

static void dfree(void* p) {
  if (p) cudaFree(p);
}

struct TablesOwner {
  ShTables h;
  DevTables d;
  ~TablesOwner() {
    void* ptrs[] = {d.ana_four, d.ana_leg, d.syn0_leg, d.syn0_dleg, d.syn0_four, d.syn0_dfour, d.syn1_leg,
                    d.syn1_dleg, d.syn1_four, d.syn1_dfour, d.synT_four, d.jf_of_coef, d.blk_off, d.m_of_coef,
                    d.n_of_coef, d.partner, d.is_sin, d.mr, d.mr_off, d.perm, d.perm_off, d.pos_in_block,
                    d.sing_w, d.smooth_w0, d.qp, d.cos_tab, d.sin_tab, d.syn0_d2leg, d.syn0_d2four,
                    d.syn1_leg_t, d.syn1_dleg_t};
    for (void* p : ptrs) dfree(p);
  }
  int upload(cudaStream_t st) {
    d.p0 = h.p0;
    d.p1 = h.p1;
    d.mr_total = (int)h.mr.size();
    int s = 0;
    s |= dupload(&d.ana_four, h.ana.four, st);
    s |= dupload(&d.ana_leg, h.ana.leg, st);
    s |= dupload(&d.syn0_leg, h.syn0.leg, st);
    s |= dupload(&d.syn0_dleg, h.syn0.dleg, st);
    s |= dupload(&d.syn0_four, h.syn0.four, st);
    s |= dupload(&d.syn0_dfour, h.syn0.dfour, st);
    s |= dupload(&d.syn1_leg, h.syn1.leg, st);
    s |= dupload(&d.syn1_dleg, h.syn1.dleg, st);
    {
      // [coefficient][latitude] -> [latitude][coefficient]
      const size_t nc = (size_t)ncoef_(h.p0), nl = (size_t)h.p1 + 1;
      std::vector<double> a(nc * nl), b(nc * nl);
      if (h.syn1.leg.size() == nc * nl && h.syn1.dleg.size() == nc * nl) {
        for (size_t c = 0; c < nc; c++)
          for (size_t l = 0; l < nl; l++) {
            a[l * nc + c] = h.syn1.leg[c * nl + l];
            b[l * nc + c] = h.syn1.dleg[c * nl + l];
          }
        s |= dupload(&d.syn1_leg_t, a, st);
        s |= dupload(&d.syn1_dleg_t, b, st);
      }
    }
    s |= dupload(&d.syn1_four, h.syn1.four, st);
    s |= dupload(&d.syn1_dfour, h.syn1.dfour, st);
    s |= dupload(&d.synT_four, h.synT.four, st);
    s |= dupload(&d.jf_of_coef, h.jf_of_coef, st);
    s |= dupload(&d.blk_off, h.blk_off, st);
    s |= dupload(&d.m_of_coef, h.m_of_coef, st);
    s |= dupload(&d.n_of_coef, h.n_of_coef, st);
    s |= dupload(&d.partner, h.partner, st);
    s |= dupload(&d.is_sin, h.is_sin, st);
    s |= dupload(&d.mr, h.mr, st);
    s |= dupload(&d.mr_off, h.mr_off, st);
    s |= dupload(&d.perm, h.perm, st);
    s |= dupload(&d.perm_off, h.perm_off, st);
    s |= dupload(&d.pos_in_block, h.pos_in_block, st);
    s |= dupload(&d.sing_w, h.sing_w, st);
    s |= dupload(&d.smooth_w0, h.smooth_w0, st);
    s |= dupload(&d.qp, h.qp, st);
    s |= dupload(&d.cos_tab, h.cos_tab, st);
    s |= dupload(&d.sin_tab, h.sin_tab, st);
    s |= dupload(&d.syn0_d2leg, h.syn0_d2leg, st);
    s |= dupload(&d.syn0_d2four, h.syn0_d2four, st);
    if (s) return VES3D_ERR_NOMEM;
    VES3D_CK(cudaStreamSynchronize(st));
    return VES3D_OK;
  }
};

}  // namespace ves3d

using namespace ves3d;

constexpr int kPcStreams = 32;  // streams of the preconditioner factorisation
constexpr int kPcBatch = 8;     // operator columns per application in its assembly

struct ves3d_sv {
  int p = 0, pup = 0, prec = 0, device = 0;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  // the far field runs on this stream beside the self-matrix build and the self part
  // (they share no inputs and use different pipes); fork and join events
  cudaStream_t side = nullptr, hi = nullptr;  // side: lowest priority; hi: the build, highest
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_built = nullptr;
  // VES3D_FAR_OVERLAP=1: far field on the side stream beside the build. Off by default:
  // measured at 512 vesicles, p = 16 it saves 2-3% of a step (97.6-98.9 ms against 100.9)
  // because both kernels already fill the SMs, and each kernel's own duration (the
  // roofline denominator) then includes the sharing
  bool overlap = false;
  bool far_dl_f32 = false;  // the mixed form's far double layer in FP32 pairs (opt-in, VES3D_FAR_DL_F32=1)
  std::unique_ptr<TablesOwner> tab;
  long nves = 0, cap_ves = 0;
  // resident buffers
  double *X = nullptr, *F = nullptr, *V = nullptr, *Vself = nullptr, *Vfar = nullptr;
  double *Sx = nullptr, *Xt = nullptr, *Xp = nullptr, *area = nullptr, *pos = nullptr, *den = nullptr;
  double *SL = nullptr, *Fc = nullptr, *Vc = nullptr, *part = nullptr;
  // double layer (allocated when a double-layer density is first set): density G and its
  // coefficients Gc, the self matrices DL, unit normals and weighted densities of the far
  // sum (point-major) and its segment partials
  double *G = nullptr, *Gc = nullptr, *DL = nullptr, *nrm = nullptr, *dden = nullptr, *part_dl = nullptr;
  long dl_cap = 0;
  bool have_dl = false, dl_valid = false;
  int nseg_dl = 0;
  float dl_ms = 0;  // last double-layer self-matrix build (device ms)
  // viscosity contrast of the implicit step (VesicleProps, src/VesicleProps.cc:17-49): lambda
  // per vesicle (one value: all), and on device vel_coeff = (1 + l)/2, dl_coeff = 1 - l
  std::vector<double> lam;
  bool contrast = false;
  // off-surface targets (SetTrgCoord): point-major [trg_n][3] and their velocities
  double *trg = nullptr, *vtrg = nullptr;
  long trg_n = 0, trg_cap = 0;
  // near-singular correction of the targets (NearSingular): the upsampled sources of every
  // vesicle (surface, tangents, density, double-layer density at p_up, AxisMajor; area;
  // point-major positions, weighted densities, normals), vesicle centroids and radii,
  // near lists and per-slot corrections of the targets, the upsampled grid's latitudes
  // and smooth weights
  bool near_on = false;
  double *nu_X = nullptr, *nu_Xt = nullptr, *nu_Xp = nullptr, *nu_F = nullptr, *nu_G = nullptr, *nu_area = nullptr;
  double *nu_pos = nullptr, *nu_den = nullptr, *nu_nrm = nullptr, *nu_dden = nullptr, *nu_cen = nullptr;
  double *nu_theta = nullptr, *nu_w = nullptr, *nu_corr = nullptr;
  unsigned long long* nu_rmax = nullptr;
  int *nu_count = nullptr, *nu_v = nullptr, *nu_k = nullptr;
  long nu_ves_cap = 0, nu_trg_cap = 0;
  double near_r = 0.0;  // r_near of the last corrected evaluation
  void free_near() {
    double* ps[] = {nu_X, nu_Xt, nu_Xp, nu_F, nu_G, nu_area, nu_pos, nu_den, nu_nrm, nu_dden, nu_cen, nu_theta, nu_w,
                    nu_corr};
    for (double* q : ps) dfree(q);
    nu_X = nu_Xt = nu_Xp = nu_F = nu_G = nu_area = nu_pos = nu_den = nu_nrm = nu_dden = nu_cen = nullptr;
    nu_theta = nu_w = nu_corr = nullptr;
    dfree(nu_rmax);
    dfree(nu_count);
    dfree(nu_v);
    dfree(nu_k);
    nu_rmax = nullptr;
    nu_count = nu_v = nu_k = nullptr;
    nu_ves_cap = nu_trg_cap = 0;
  }
  double *velc = nullptr, *dlc = nullptr;
  long contrast_nves = -1;  // vesicle count the device coefficients were made for
  long* off = nullptr;  // [nves+1] point offsets of the vesicles
  long off_nves = -1;   // vesicle count the offsets were uploaded for
  // setup scratch (one chunk of vesicles)
  long chunk = 0;
  double *R = nullptr, *Xu = nullptr, *Xut = nullptr, *Xup = nullptr, *K = nullptr, *C = nullptr, *SL3 = nullptr;
  bool have_src = false, have_den = false, sl_valid = false, parts_valid = false;
  // sl_tc: the current self matrices come from the mixed form's FP32 build stages (the
  // tensor-core build at p = 16, the FP32 rotate-transpose and Grid2SHC at p = 12, 24);
  // implicit_on: implicit parameters were set, whose FP64 residuals need FP64 self matrices
  bool sl_tc = false, implicit_on = false;
  // implicit step: geometry record and work fields (allocated on first use)
  double *geo = nullptr, *wc = nullptr, *w[8] = {nullptr}, *bws = nullptr;
  long geo_cap = 0, bws_cap = 0;
  bool geo_valid = false;
  double dt = 0.01, kappa = 0.05, shear = 1.0;
  double drho = 0.0, grav[3] = {0.0, 0.0, -1.0};  // excess density and gravity field
  // the reference Surface's low-pass filter of H, K, grad, div and the linearised
  // curvature (0: off; else the highest degree kept) and its coefficients [nc] on device
  int filter_freq = 0;
  double* filt = nullptr;
  int far_force_fp64 = 0;      // 1: evaluate the far field in FP64 even in the mixed form
  int ir_outer = 0, ir_inner = 0;  // last mixed solve: outer refinements, inner iterations
  // preconditioner of the implicit solve (VES3D_PRECOND_*); the self-block form stores one
  // inverse per vesicle, [nv][n][n] column-major in FP32 (n = 4 nc)
  int precond = 0;
  float* pc_inv = nullptr;
  double* pc_diag = nullptr;   // diagonal-spectral scales [4 nc]
  long pc_cap = 0;
  bool pc_valid = false;
  int pc_refresh = 1;          // rebuild after this many surface updates (1 = every update)
  int pc_age = 0;              // surface updates since the last build
  long pc_nves = 0;            // vesicle count the preconditioner was built for
  double pc_ms[3] = {0, 0, 0};  // last build: total, assembly, factorisation (device ms)
  // CUDA graph of the resident evaluation (density buffer -> velocity buffer)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  void drop_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    graph_exec = nullptr;
    graph = nullptr;
  }
  cudaEvent_t pc_ev[3 + kPcStreams] = {};
  cudaEvent_t ev[10] = {};
  float ms[4] = {0, 0, 0, 0};
  float far_dl_ms = 0;  // the far double layer's segment kernels in the last evaluation

  ~ves3d_sv() {
    free_near();
    dfree(filt);
    dfree(velc);
    dfree(dlc);
    dfree(trg);
    dfree(vtrg);
    drop_graph();
    free_precond();
    for (auto& e : pc_ev)
      if (e) cudaEventDestroy(e);
    free_implicit();
    free_buffers();
    free_scratch();
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    tab.reset();
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (ev_built) cudaEventDestroy(ev_built);
    if (side) cudaStreamDestroy(side);
    if (hi) cudaStreamDestroy(hi);
    if (own_stream) cudaStreamDestroy(own_stream);
  }
  void free_dl() {
    double* ps[] = {G, Gc, DL, nrm, dden, part_dl};
    for (double* q : ps) dfree(q);
    G = Gc = DL = nrm = dden = part_dl = nullptr;
    dl_cap = 0;
    have_dl = dl_valid = false;
  }
  void free_buffers() {
    free_dl();
    double* ps[] = {X, F, V, Vself, Vfar, Sx, Xt, Xp, area, pos, den, SL, Fc, Vc, part};
    for (double* q : ps) dfree(q);
    dfree(off);
    off = nullptr;
    X = F = V = Vself = Vfar = Sx = Xt = Xp = area = pos = den = SL = Fc = Vc = part = nullptr;
    cap_ves = 0;
    off_nves = -1;
  }
  void free_implicit() {
    dfree(geo);
    dfree(wc);
    for (auto& q : w) {
      dfree(q);
      q = nullptr;
    }
    dfree(bws);
    geo = wc = bws = nullptr;
    geo_cap = bws_cap = 0;
    geo_valid = false;
  }
  void free_precond() {
    if (pc_inv) cudaFree(pc_inv);
    dfree(pc_diag);
    pc_inv = nullptr;
    pc_diag = nullptr;
    pc_cap = 0;
    pc_valid = false;
  }
  void free_scratch() {
    double* ps[] = {R, Xu, Xut, Xup, K, C, SL3};
    for (double* q : ps) dfree(q);
    R = Xu = Xut = Xup = K = C = SL3 = nullptr;
    chunk = 0;
  }
  long npts() const { return nves * ngrid_(p); }
};

namespace {

int check_sv(ves3d_sv* sv) {
  if (!sv) {
    set_error("invalid argument: null context");
    return VES3D_ERR_ARG;
  }
  VES3D_CK(cudaSetDevice(sv->device));
  return VES3D_OK;
}

int alloc_resident(ves3d_sv* sv, long nves) {
  if (nves <= sv->cap_ves) return VES3D_OK;
  sv->free_buffers();
  const size_t ng = ngrid_(sv->p), nc = ncoef_(sv->p), n = 3 * nc, fld = (size_t)nves * 3 * ng;
  int s = 0;
  s |= dalloc(&sv->X, fld);
  s |= dalloc(&sv->F, fld);
  s |= dalloc(&sv->V, fld);
  s |= dalloc(&sv->Vself, fld);
  s |= dalloc(&sv->Vfar, fld);
  s |= dalloc(&sv->Sx, (size_t)nves * 3 * nc);
  s |= dalloc(&sv->Xt, fld);
  s |= dalloc(&sv->Xp, fld);
  s |= dalloc(&sv->area, (size_t)nves * ng);
  s |= dalloc(&sv->pos, fld);
  s |= dalloc(&sv->den, fld);
  s |= dalloc(&sv->SL, (size_t)nves * n * n);
  s |= dalloc(&sv->Fc, (size_t)nves * n);
  s |= dalloc(&sv->Vc, (size_t)nves * n);
  s |= dalloc(&sv->part, (size_t)kFarMaxSegments * fld);
  s |= dalloc(&sv->off, (size_t)nves + 1);
  if (s) {
    sv->free_buffers();
    return s;
  }
  sv->cap_ves = nves;
  return VES3D_OK;
}

// Double-layer buffers for the resident capacity (first double-layer density).
int alloc_dl(ves3d_sv* sv) {
  if (sv->dl_cap >= sv->cap_ves && sv->DL) return VES3D_OK;
  sv->free_dl();
  const long nves = sv->cap_ves;
  const size_t ng = ngrid_(sv->p), n = 3 * (size_t)ncoef_(sv->p), fld = (size_t)nves * 3 * ng;
  int s = 0;
  s |= dalloc(&sv->G, fld);
  s |= dalloc(&sv->Gc, (size_t)nves * n);
  s |= dalloc(&sv->DL, (size_t)nves * n * n);
  s |= dalloc(&sv->nrm, fld);
  s |= dalloc(&sv->dden, fld);
  s |= dalloc(&sv->part_dl, (size_t)kFarMaxSegments * fld);
  if (s) {
    sv->free_dl();
    return s;
  }
  sv->dl_cap = nves;
  return VES3D_OK;
}

// The fused per-rotation build is used when it is instantiated for (p, p_up);
// VES3D_FUSED_BUILD=0 forces the unfused stage-by-stage pipeline (A/B checks).
bool use_fused(const ves3d_sv* sv) {
  const char* env = getenv("VES3D_FUSED_BUILD");
  if (env && env[0] == '0') return false;
  return fused_build_supported(sv->p, sv->pup);
}

// The mixed form builds with the DFT GEMMs on tcgen05 tensor cores where that kernel is
// laid out for (p, p_up); VES3D_TC_BUILD=0 keeps the FP64 ring (A/B checks).
bool use_tc_build(const ves3d_sv* sv) {
  if (sv->prec != VES3D_PREC_MIXED || sv->implicit_on || !tc_build_supported(sv->p, sv->pup)) return false;
  const char* env = getenv("VES3D_TC_BUILD");
  return !(env && env[0] == '0');
}

// The mixed form's other fused orders (p = 12, 24): the FP64 ring's results rotated back and
// taken to coefficients in FP32 (as after the tensor-core build); the same conditions and
// switch as the tensor-core build.
bool use_f32_post(const ves3d_sv* sv) {
  if (sv->prec != VES3D_PREC_MIXED || sv->implicit_on || !rotate_transpose_f32_from_f64_supported(sv->p)) return false;
  const char* env = getenv("VES3D_TC_BUILD");
  return !(env && env[0] == '0');
}

// A context that takes implicit steps keeps FP64 self matrices: the mixed refinement's
// outer residuals are those of the FP64 system. Self matrices from the tensor-core build
// are rebuilt on next use.
void mark_implicit(ves3d_sv* sv) {
  if (sv->implicit_on) return;
  sv->implicit_on = true;
  if (sv->sl_tc) sv->sl_valid = false;
}

// Doubles of setup scratch per vesicle.
size_t scratch_per_vesicle(int p0, int p1, bool fused) {
  const size_t npr = (size_t)p0 * (p0 + 1), nc = ncoef_(p0), M1 = ngrid_(p1), ng = ngrid_(p0);
  return npr * 3 * nc                            // R
         + (fused ? 0 : 3 * npr * 3 * M1)        // Xu, Xut, Xup
         + (fused ? 0 : npr * 12 * M1)           // K
         + npr * 12 * nc                         // C
         + 3 * nc * 3 * ng;                      // SL3
}

int alloc_scratch(ves3d_sv* sv) {
  const long want = sv->nves;
  // the double layer is built stage by stage: those stage buffers are kept while a
  // double-layer density is set (the fused single-layer build needs a subset of them)
  const bool stages = !use_fused(sv) || sv->have_dl || sv->contrast;
  const bool layout_ok = !stages || sv->K != nullptr;
  if (sv->chunk >= want && layout_ok) return VES3D_OK;  // the whole suspension in one chunk already
  const bool fused = !stages;
  size_t per = scratch_per_vesicle(sv->p, sv->pup, fused) * sizeof(double);
  size_t free_b = 0, total_b = 0;
  VES3D_CK(cudaMemGetInfo(&free_b, &total_b));
  // Scratch budget for one chunk of the self-matrix build: 16 GiB by default (the 512
  // vesicles of p = 16 take 10.6 GB, one chunk), capped at a third of free memory;
  // VES3D_SCRATCH_MB overrides (e.g. to keep profiler captures small).
  size_t budget = (size_t)16 << 30;
  if (const char* env = getenv("VES3D_SCRATCH_MB")) {
    long mb = atol(env);
    if (mb > 0) budget = (size_t)mb << 20;
  }
  if (budget > free_b / 3) budget = free_b / 3;
  long chunk = (long)(budget / per);
  if (chunk < 1) chunk = 1;
  if (chunk > want) chunk = want;
  if (chunk <= sv->chunk && layout_ok) return VES3D_OK;
  sv->free_scratch();
  const size_t npr = (size_t)sv->p * (sv->p + 1), nc = ncoef_(sv->p), M1 = ngrid_(sv->pup), ng = ngrid_(sv->p);
  int s = 0;
  s |= dalloc(&sv->R, chunk * npr * 3 * nc);
  if (!fused) {
    s |= dalloc(&sv->Xu, chunk * npr * 3 * M1);
    s |= dalloc(&sv->Xut, chunk * npr * 3 * M1);
    s |= dalloc(&sv->Xup, chunk * npr * 3 * M1);
    s |= dalloc(&sv->K, chunk * npr * 12 * M1);
  }
  s |= dalloc(&sv->C, chunk * npr * 12 * nc);
  s |= dalloc(&sv->SL3, chunk * 3 * nc * 3 * ng);
  if (s) {
    sv->free_scratch();
    return s;
  }
  sv->chunk = chunk;
  return VES3D_OK;
}

int copy_in(double* dst, const double* src, size_t n, int is_device, cudaStream_t st) {
  VES3D_CK(cudaMemcpyAsync(dst, src, n * sizeof(double), is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                           st));
  return VES3D_OK;
}

int copy_out(double* dst, const double* src, size_t n, int is_device, cudaStream_t st) {
  VES3D_CK(cudaMemcpyAsync(dst, src, n * sizeof(double), is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                           st));
  if (!is_device) VES3D_CK(cudaStreamSynchronize(st));
  return VES3D_OK;
}

int alloc_scratch(ves3d_sv* sv);
int run_setup(ves3d_sv* sv, bool dl = false);

// The self matrices of every vesicle: the single layer (SL), or with dl the double layer
// (DL, always by the stage-by-stage pipeline).
int run_setup(ves3d_sv* sv, bool dl) {
  NvtxRange nvtx(dl ? "ves3d build dl" : "ves3d build");
  const DevTables& T = sv->tab->d;
  const int p0 = sv->p, p1 = sv->pup, nc = ncoef_(p0), ng = ngrid_(p0), M1 = ngrid_(p1);
  const long npr = (long)p0 * (p0 + 1);
  cudaStream_t st = sv->stream;
  int s = alloc_scratch(sv);
  if (s) return s;
  const bool fused = !dl && use_fused(sv);
  const bool tc = fused && use_tc_build(sv);
  const bool f32post = fused && !tc && use_f32_post(sv);
  double* M = dl ? sv->DL : sv->SL;
  if ((!fused && !sv->K) || !M) {
    set_error("internal: self-matrix build without its buffers");
    return VES3D_ERR_STATE;
  }
  VES3D_CK(cudaEventRecord(sv->ev[0], st));
  for (long v0 = 0; v0 < sv->nves; v0 += sv->chunk) {
    const long nb = std::min(sv->chunk, sv->nves - v0);
    const long nrot = nb * npr;
    if ((s = launch_rotate_all(sv->Sx + v0 * 3 * nc, nb, T, sv->R, st))) return s;
    // the tensor-core build leaves FP32 transposed-DFT results (in the first half of C),
    // rotated back in FP32; the FP64 builds leave FP64 ones
    float* Cf = reinterpret_cast<float*>(sv->C);
    if (fused && tc) {
      if ((s = launch_build_ring_tc(sv->R, nrot, T, Cf, st))) return s;
    } else if (fused) {
      if ((s = launch_build_ring(sv->R, nrot, T, sv->C, st))) return s;
    } else {
      if ((s = launch_synthesis(sv->R, nrot * 3, p0, p1, T.syn1_leg, T.syn1_dleg, T.syn1_four, T.syn1_dfour,
                                T.blk_off, sv->Xu, sv->Xut, sv->Xup, st)))
        return s;
      if ((s = (dl ? launch_singular_dl : launch_singular_sl)(sv->Xu, sv->Xut, sv->Xup, sv->R, nrot, T, sv->K, st)))
        return s;
      if ((s = launch_analysis(sv->K, nrot * 12, p1, p0, T.synT_four, T.syn1_leg, T.jf_of_coef, sv->C, st)))
        return s;
    }
    double* Mv = M + v0 * (long)(3 * nc) * (3 * nc);
    if (tc || f32post) {  // FP32 grid between the rotation back and Grid2SHC
      float* SLf = reinterpret_cast<float*>(sv->SL3);
      if ((s = tc ? launch_rotate_transpose_f32(Cf, nb, T, SLf, st)
                  : launch_rotate_transpose_f32(sv->C, nb, T, SLf, st)))
        return s;
      if ((s = launch_grid2shc_f32(SLf, nb * 3 * nc * 3, p0, T.ana_four, T.ana_leg, T.jf_of_coef, Mv, st))) return s;
    } else {
      if ((s = launch_rotate_transpose_scatter(sv->C, nb, T, sv->SL3, st))) return s;
      if ((s = launch_grid2shc(sv->SL3, nb * 3 * nc * 3, p0, T.ana_four, T.ana_leg, T.jf_of_coef, Mv, st))) return s;
    }
    (void)ng;
    (void)M1;
  }
  VES3D_CK(cudaEventRecord(sv->ev[1], st));
  VES3D_CK(cudaEventSynchronize(sv->ev[1]));
  VES3D_CK(cudaEventElapsedTime(dl ? &sv->dl_ms : &sv->ms[0], sv->ev[0], sv->ev[1]));
  if (tc && tc_build_error(true)) {
    set_error("self-matrix build on the tensor cores: a bounded wait of the kernel ran out");
    return VES3D_ERR_CUDA;
  }
  if (dl) {
    sv->dl_valid = true;
  } else {
    sv->sl_valid = true;
    sv->sl_tc = tc || f32post;
  }
  return VES3D_OK;
}

// Self part of an evaluation: Vself = SHC2Grid(Grid2SHC(F) . SL) and the weighted far-field
// density den = F * area * qw, written to the given buffers (the context's own, or slices
// of a polydisperse suspension's global arrays). With nrm given, the double layer of the
// density in G as well: Grid2SHC(G) . DL added in coefficients, and the far double layer's
// unit normals (nrm) and weighted density dden = G * area * qw.
int run_self(ves3d_sv* sv, double* vself, double* den, double* nrm = nullptr, double* dden = nullptr) {
  const DevTables& T = sv->tab->d;
  const int p0 = sv->p, n = 3 * ncoef_(p0);
  cudaStream_t st = sv->stream;
  int s;
  if ((s = launch_grid2shc(sv->F, sv->nves * 3, p0, T.ana_four, T.ana_leg, T.jf_of_coef, sv->Fc, st))) return s;
  if ((s = launch_self_gemv(sv->Fc, sv->SL, sv->nves, n, sv->Vc, st))) return s;
  if (nrm) {
    if ((s = launch_grid2shc(sv->G, sv->nves * 3, p0, T.ana_four, T.ana_leg, T.jf_of_coef, sv->Gc, st))) return s;
    if ((s = launch_self_gemv(sv->Gc, sv->DL, sv->nves, n, sv->Vc, st, /*accumulate=*/true))) return s;
  }
  if ((s = launch_synthesis(sv->Vc, sv->nves * 3, p0, p0, T.syn0_leg, T.syn0_dleg, T.syn0_four, T.syn0_dfour,
                            T.blk_off, vself, nullptr, nullptr, st)))
    return s;
  if ((s = launch_far_density(sv->F, sv->area, sv->nves, p0, T.smooth_w0, den, st))) return s;
  if (!nrm) return VES3D_OK;
  if ((s = launch_unit_normals(sv->Xt, sv->Xp, sv->nves, p0, nrm, st))) return s;
  return launch_far_density(sv->G, sv->area, sv->nves, p0, T.smooth_w0, dden, st);
}

// Self part alone: Vself = SHC2Grid(Grid2SHC(F) . SL [+ Grid2SHC(G) . DL]) on the
// context's stream (src/StokesVelocity.cc:385-452: SL_vel + DL_vel in coefficients).
int run_self_apply(ves3d_sv* sv, bool dl) {
  NvtxRange nvtx("ves3d self");
  const DevTables& T = sv->tab->d;
  const int p0 = sv->p, n = 3 * ncoef_(p0);
  cudaStream_t st = sv->stream;
  int s;
  if ((s = launch_grid2shc(sv->F, sv->nves * 3, p0, T.ana_four, T.ana_leg, T.jf_of_coef, sv->Fc, st))) return s;
  if ((s = launch_self_gemv(sv->Fc, sv->SL, sv->nves, n, sv->Vc, st))) return s;
  if (dl) {
    if ((s = launch_grid2shc(sv->G, sv->nves * 3, p0, T.ana_four, T.ana_leg, T.jf_of_coef, sv->Gc, st))) return s;
    if ((s = launch_self_gemv(sv->Gc, sv->DL, sv->nves, n, sv->Vc, st, /*accumulate=*/true))) return s;
  }
  return launch_synthesis(sv->Vc, sv->nves * 3, p0, p0, T.syn0_leg, T.syn0_dleg, T.syn0_four, T.syn0_dfour,
                          T.blk_off, sv->Vself, nullptr, nullptr, st);
}

// Fork: the weighted density and the far-field segments on the side stream, which waits
// for everything the context's stream has queued (surfaces, densities, the previous
// evaluation's reduce). ev_far[0..1] (may be null) bracket the segment kernels.
int fork_far(ves3d_sv* sv, int* nseg, cudaEvent_t ev_far0, cudaEvent_t ev_far1, bool dl) {
  NvtxRange nvtx("ves3d far");
  const DevTables& T = sv->tab->d;
  int s;
  cudaStream_t fs = sv->overlap ? sv->side : sv->stream;
  VES3D_CK(cudaEventRecord(sv->ev_fork, sv->stream));
  VES3D_CK(cudaStreamWaitEvent(fs, sv->ev_fork, 0));
  if ((s = launch_far_density(sv->F, sv->area, sv->nves, sv->p, T.smooth_w0, sv->den, fs))) return s;
  if (ev_far0) VES3D_CK(cudaEventRecord(ev_far0, fs));
  if ((s = launch_far(sv->prec == VES3D_PREC_MIXED && !sv->far_force_fp64, sv->pos, sv->den, sv->off, sv->nves,
                      sv->npts(), ngrid_(sv->p), nullptr, nullptr, nullptr, sv->part, kFarMaxSegments, fs, nseg)))
    return s;
  if (ev_far1) VES3D_CK(cudaEventRecord(ev_far1, fs));
  sv->nseg_dl = 0;
  if (dl) {  // the far double layer after the single layer's segments: FP64 (FP32 pairs on request)
    if ((s = launch_unit_normals(sv->Xt, sv->Xp, sv->nves, sv->p, sv->nrm, fs))) return s;
    if ((s = launch_far_density(sv->G, sv->area, sv->nves, sv->p, T.smooth_w0, sv->dden, fs))) return s;
    if (ev_far0) VES3D_CK(cudaEventRecord(sv->ev[8], fs));
    const bool dl32 = sv->prec == VES3D_PREC_MIXED && !sv->far_force_fp64 && sv->far_dl_f32;
    if ((s = launch_far_dl(dl32, sv->pos, sv->nrm, sv->dden, sv->off, sv->nves, sv->npts(), ngrid_(sv->p),
                           sv->part_dl, kFarMaxSegments, fs, &sv->nseg_dl)))
      return s;
    if (ev_far0) VES3D_CK(cudaEventRecord(sv->ev[9], fs));
  }
  VES3D_CK(cudaEventRecord(sv->ev_join, fs));
  return VES3D_OK;
}

// The self-matrix build on the high-priority stream (after everything queued on the
// context's stream), the context's stream waiting for it.
int run_setup_hi(ves3d_sv* sv) {
  if (!sv->overlap) return run_setup(sv);
  VES3D_CK(cudaStreamWaitEvent(sv->hi, sv->ev_fork, 0));
  cudaStream_t saved = sv->stream;
  sv->stream = sv->hi;
  const int s = run_setup(sv);
  sv->stream = saved;
  if (s) return s;
  VES3D_CK(cudaEventRecord(sv->ev_built, sv->hi));
  VES3D_CK(cudaStreamWaitEvent(sv->stream, sv->ev_built, 0));
  return VES3D_OK;
}

// Join: the reduce of the far partials, added to the self part, on the context's stream.
int join_far(ves3d_sv* sv, int nseg, bool dl) {
  VES3D_CK(cudaStreamWaitEvent(sv->stream, sv->ev_join, 0));
  return launch_far_reduce(sv->part, nseg, sv->off, sv->nves, sv->npts(), sv->Vself, sv->V, sv->Vfar, sv->stream,
                           dl ? sv->part_dl : nullptr, dl ? sv->nseg_dl : 0, kDl);
}

// The evaluation proper, stream-ordered and free of host synchronisation (it is what the
// CUDA graph of ves3d_sv_capture_eval records): the far field forked to the side stream,
// the self part on the context's stream, joined by the reduce.
int run_eval_body(ves3d_sv* sv, bool dl) {
  int s, nseg = 0;
  if ((s = fork_far(sv, &nseg, nullptr, nullptr, dl))) return s;
  if ((s = run_self_apply(sv, dl))) return s;
  return join_far(sv, nseg, dl);
}

// One evaluation; dl adds the double layer of the density G (the operator's own
// evaluation when a double-layer density is set; the implicit step applies the single
// layer alone).
int run_eval(ves3d_sv* sv, bool dl) {
  cudaStream_t st = sv->stream;
  int s, nseg = 0;
  if (!sv->have_src || !sv->have_den) {
    set_error("eval before set_src_coord / set_density_sl");
    return VES3D_ERR_STATE;
  }
  // the far field first (on the side stream when overlapping the self-matrix build, else
  // on the context's stream); events ev[4], ev[5] bracket its segment kernels (the
  // roofline denominator)
  if (dl && !sv->G) {
    set_error("double layer requested without a double-layer density");
    return VES3D_ERR_STATE;
  }
  if ((s = fork_far(sv, &nseg, sv->ev[4], sv->ev[5], dl))) return s;
  if (!sv->sl_valid && (s = run_setup_hi(sv))) return s;
  if (dl && !sv->dl_valid && (s = run_setup(sv, true))) return s;
  VES3D_CK(cudaEventRecord(sv->ev[2], st));
  if ((s = run_self_apply(sv, dl))) return s;
  VES3D_CK(cudaEventRecord(sv->ev[3], st));
  if ((s = join_far(sv, nseg, dl))) return s;
  VES3D_CK(cudaEventRecord(sv->ev[6], st));
  VES3D_CK(cudaEventSynchronize(sv->ev[6]));
  VES3D_CK(cudaEventElapsedTime(&sv->ms[1], sv->ev[2], sv->ev[3]));
  VES3D_CK(cudaEventElapsedTime(&sv->ms[2], sv->ev[4], sv->ev[5]));
  VES3D_CK(cudaEventElapsedTime(&sv->ms[3], sv->ev[2], sv->ev[6]));
  sv->far_dl_ms = 0;
  if (dl) VES3D_CK(cudaEventElapsedTime(&sv->far_dl_ms, sv->ev[8], sv->ev[9]));
  sv->parts_valid = true;
  return VES3D_OK;
}

}  // namespace

namespace {

// Targets with the near-singular correction (near_kernels.cu): the self part of the
// current densities (its coefficients are the on-surface values), the upsampled sources of
// every vesicle, the smooth quadrature of all of them at the targets, then the correction
// of the targets near a vesicle.
int eval_trg_near(ves3d_sv* sv) {
  const DevTables& T = sv->tab->d;
  cudaStream_t st = sv->stream;
  const int p = sv->p, q = sv->pup, nc = ncoef_(p);
  const long nv = sv->nves, M = sv->trg_n, ng1 = ngrid_(q);
  const bool dl = sv->have_dl;
  int s;
  if (!sv->sl_valid && (s = run_setup(sv))) return s;
  if (dl && !sv->dl_valid && (s = run_setup(sv, true))) return s;
  if ((s = run_self_apply(sv, dl))) return s;  // Fc (Gc) and the self coefficients Vc
  if (sv->nu_ves_cap < nv || (dl && !sv->nu_G)) {
    double* ps[] = {sv->nu_X, sv->nu_Xt, sv->nu_Xp, sv->nu_F, sv->nu_G, sv->nu_area, sv->nu_pos, sv->nu_den,
                    sv->nu_nrm, sv->nu_dden, sv->nu_cen, sv->nu_theta, sv->nu_w};
    for (double* x : ps) dfree(x);
    const size_t f = (size_t)nv * 3 * ng1;
    s = 0;
    s |= dalloc(&sv->nu_X, f);
    s |= dalloc(&sv->nu_Xt, f);
    s |= dalloc(&sv->nu_Xp, f);
    s |= dalloc(&sv->nu_F, f);
    s |= dalloc(&sv->nu_G, f);
    s |= dalloc(&sv->nu_area, (size_t)nv * ng1);
    s |= dalloc(&sv->nu_pos, f);
    s |= dalloc(&sv->nu_den, f);
    s |= dalloc(&sv->nu_nrm, f);
    s |= dalloc(&sv->nu_dden, f);
    s |= dalloc(&sv->nu_cen, 4 * (size_t)nv);
    if (!sv->nu_rmax) s |= dalloc(&sv->nu_rmax, 1);
    // the upsampled grid's latitudes and smooth weights (LegendreWeights(p_up))
    std::vector<double> x, w, th(q + 1), sw(q + 1);
    gauss_legendre(q + 1, x, w);
    for (int i = 0; i <= q; i++) {
      th[i] = std::acos(x[i]);
      sw[i] = w[i] * M_PI / q / std::sqrt(1.0 - x[i] * x[i]);
    }
    if (!s) s = dupload(&sv->nu_theta, th, st);
    if (!s) s = dupload(&sv->nu_w, sw, st);
    if (s) {
      sv->free_near();
      return s;
    }
    sv->nu_ves_cap = nv;
  }
  if (sv->nu_trg_cap < M) {
    dfree(sv->nu_count);
    dfree(sv->nu_v);
    dfree(sv->nu_k);
    dfree(sv->nu_corr);
    sv->nu_count = sv->nu_v = sv->nu_k = nullptr;
    sv->nu_corr = nullptr;
    s = 0;
    s |= dalloc(&sv->nu_count, (size_t)M);
    s |= dalloc(&sv->nu_v, (size_t)M * kNearMax);
    s |= dalloc(&sv->nu_k, (size_t)M * kNearMax);
    s |= dalloc(&sv->nu_corr, (size_t)M * kNearMax * 3);
    if (s) {
      sv->free_near();
      return s;
    }
    sv->nu_trg_cap = M;
  }
  // upsampled sources
  if ((s = launch_synthesis(sv->Sx, nv * 3, p, q, T.syn1_leg, T.syn1_dleg, T.syn1_four, T.syn1_dfour, T.blk_off,
                            sv->nu_X, sv->nu_Xt, sv->nu_Xp, st)))
    return s;
  if ((s = launch_synthesis(sv->Fc, nv * 3, p, q, T.syn1_leg, T.syn1_dleg, T.syn1_four, T.syn1_dfour, T.blk_off,
                            sv->nu_F, nullptr, nullptr, st)))
    return s;
  if ((s = launch_far_sources(sv->nu_X, sv->nu_F, sv->nu_Xt, sv->nu_Xp, nv, q, sv->nu_w, sv->nu_area, sv->nu_pos,
                              sv->nu_den, st)))
    return s;
  if (dl) {
    if ((s = launch_synthesis(sv->Gc, nv * 3, p, q, T.syn1_leg, T.syn1_dleg, T.syn1_four, T.syn1_dfour, T.blk_off,
                              sv->nu_G, nullptr, nullptr, st)))
      return s;
    if ((s = launch_unit_normals(sv->nu_Xt, sv->nu_Xp, nv, q, sv->nu_nrm, st))) return s;
    if ((s = launch_far_density(sv->nu_G, sv->nu_area, nv, q, sv->nu_w, sv->nu_dden, st))) return s;
  }
  // the smooth quadrature of every vesicle at every target
  if ((s = launch_targets_f64(sv->nu_pos, sv->nu_den, dl ? sv->nu_nrm : nullptr, dl ? sv->nu_dden : nullptr,
                              nv * ng1, sv->trg, M, sv->vtrg, st)))
    return s;
  // r_near = r_ves 2 / sqrt(p_up) (src/NearSingular.cc:160, :119-158)
  if ((s = launch_centroid_radius(sv->X, nv, p, sv->nu_cen, sv->nu_rmax, st))) return s;
  unsigned long long bits = 0;
  VES3D_CK(cudaMemcpyAsync(&bits, sv->nu_rmax, sizeof(bits), cudaMemcpyDeviceToHost, st));
  VES3D_CK(cudaStreamSynchronize(st));
  double r_ves;
  std::memcpy(&r_ves, &bits, sizeof(double));
  sv->near_r = r_ves * 2.0 / std::sqrt((double)q);
  if ((s = launch_near_find(sv->trg, M, sv->nu_cen, nv, sv->nu_pos, q, sv->near_r, sv->nu_count, sv->nu_v, sv->nu_k,
                            st)))
    return s;
  {  // more near vesicles than slots for some target: an error, not a silent truncation
    std::vector<int> c(M);
    VES3D_CK(cudaMemcpyAsync(c.data(), sv->nu_count, M * sizeof(int), cudaMemcpyDeviceToHost, st));
    VES3D_CK(cudaStreamSynchronize(st));
    for (long t = 0; t < M; t++)
      if (c[t] > kNearMax) {
        set_error("target %ld is near more than %d vesicles (the near-singular correction's limit)", t, kNearMax);
        return VES3D_ERR_ARG;
      }
  }
  return launch_near_correct(sv->trg, M, sv->nu_count, sv->nu_v, sv->nu_k, sv->Sx, sv->Vc, dl ? sv->Gc : nullptr,
                             sv->nu_pos, sv->nu_den, dl ? sv->nu_nrm : nullptr, dl ? sv->nu_dden : nullptr,
                             sv->nu_theta, T.blk_off, p, q, sv->near_r, sv->nu_corr, sv->vtrg, st);
}

}  // namespace

extern "C" {

int ves3d_version(void) { return 100; }

const char* ves3d_last_error(void) { return g_err; }

long long ves3d_kernel_launches(void) { return launch_counter().load(); }

int ves3d_sv_create(int sh_order, int sh_order_up, int precision, int device, ves3d_sv** out) {
  VES3D_ARG(out != nullptr, "out is null");
  *out = nullptr;
  VES3D_ARG(sh_order >= 2 && sh_order <= 64, "sh_order must be in [2, 64]");
  if (sh_order_up <= 0) sh_order_up = 2 * sh_order;
  VES3D_ARG(sh_order_up >= sh_order && sh_order_up <= 128, "sh_order_up must be in [sh_order, 128]");
  VES3D_ARG(precision == VES3D_PREC_FP64 || precision == VES3D_PREC_MIXED, "unknown precision");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    set_error("no CUDA device: %s", cudaGetErrorString(e));
    return VES3D_ERR_NODEV;
  }
  if (device < 0) VES3D_CK(cudaGetDevice(&device));
  VES3D_ARG(device < ndev, "device index out of range");
  VES3D_CK(cudaSetDevice(device));
  cudaDeviceProp prop;
  VES3D_CK(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) {
    set_error("device %d is sm_%d%d; this library is built for sm_100a", device, prop.major, prop.minor);
    return VES3D_ERR_NODEV;
  }
  std::unique_ptr<ves3d_sv> sv(new ves3d_sv());
  sv->p = sh_order;
  sv->pup = sh_order_up;
  sv->prec = precision;
  sv->device = device;
  VES3D_CK(cudaStreamCreateWithFlags(&sv->own_stream, cudaStreamNonBlocking));
  sv->stream = sv->own_stream;
  {
    // the far field yields to the build: as SMs free up, the build's CTAs are dispatched
    // first and the far field's fill the room left beside them
    int least = 0, greatest = 0;
    VES3D_CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    VES3D_CK(cudaStreamCreateWithPriority(&sv->side, cudaStreamNonBlocking, least));
    VES3D_CK(cudaStreamCreateWithPriority(&sv->hi, cudaStreamNonBlocking, greatest));
    const char* e = getenv("VES3D_FAR_OVERLAP");
    sv->overlap = e && e[0] == '1';
    const char* d = getenv("VES3D_FAR_DL_F32");
    sv->far_dl_f32 = d && d[0] == '1';
  }
  VES3D_CK(cudaEventCreateWithFlags(&sv->ev_fork, cudaEventDisableTiming));
  VES3D_CK(cudaEventCreateWithFlags(&sv->ev_join, cudaEventDisableTiming));
  VES3D_CK(cudaEventCreateWithFlags(&sv->ev_built, cudaEventDisableTiming));
  for (auto& ev : sv->ev) VES3D_CK(cudaEventCreate(&ev));
  sv->tab.reset(new TablesOwner());
  build_tables(sh_order, sh_order_up, sv->tab->h);
  int s = sv->tab->upload(sv->stream);
  if (s) return s;
  *out = sv.release();
  return VES3D_OK;
}

int ves3d_sv_destroy(ves3d_sv* sv) {
  if (!sv) return VES3D_OK;
  cudaSetDevice(sv->device);
  if (sv->stream) cudaStreamSynchronize(sv->stream);
  delete sv;
  return VES3D_OK;
}

int ves3d_sv_set_stream(ves3d_sv* sv, void* stream) {
  int s = check_sv(sv);
  if (s) return s;
  sv->stream = stream ? (cudaStream_t)stream : sv->own_stream;
  sv->drop_graph();
  return VES3D_OK;
}

int ves3d_sv_set_src_coord(ves3d_sv* sv, const double* S, long n_ves, int is_device) {
  NvtxRange nvtx("ves3d set_src_coord");
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(S != nullptr, "S is null");
  VES3D_ARG(n_ves >= 1, "n_ves must be >= 1");
  if ((s = alloc_resident(sv, n_ves))) return s;
  sv->nves = n_ves;
  const int p0 = sv->p, ng = ngrid_(p0);
  const DevTables& T = sv->tab->d;
  if ((s = copy_in(sv->X, S, (size_t)n_ves * 3 * ng, is_device, sv->stream))) return s;
  if (sv->off_nves != n_ves) {  // point offsets of the vesicles, uploaded when the count changes
    std::vector<long> off(n_ves + 1);
    for (long v = 0; v <= n_ves; v++) off[v] = v * ng;
    VES3D_CK(cudaMemcpyAsync(sv->off, off.data(), off.size() * sizeof(long), cudaMemcpyHostToDevice, sv->stream));
    VES3D_CK(cudaStreamSynchronize(sv->stream));
    sv->off_nves = n_ves;
  }
  if ((s = launch_grid2shc(sv->X, n_ves * 3, p0, T.ana_four, T.ana_leg, T.jf_of_coef, sv->Sx, sv->stream)))
    return s;
  if ((s = launch_synthesis(sv->Sx, n_ves * 3, p0, p0, T.syn0_leg, T.syn0_dleg, T.syn0_four, T.syn0_dfour, T.blk_off,
                            sv->Vself /* scratch: filtered grid, unused */, sv->Xt, sv->Xp, sv->stream)))
    return s;
  if ((s = launch_far_sources(sv->X, nullptr, sv->Xt, sv->Xp, n_ves, p0, T.smooth_w0, sv->area, sv->pos, nullptr,
                              sv->stream)))
    return s;
  VES3D_CK(cudaStreamSynchronize(sv->stream));
  sv->have_src = true;
  sv->have_den = false;
  sv->have_dl = false;  // densities belong to the surfaces they were set for
  sv->dl_valid = false;
  sv->sl_valid = false;
  sv->parts_valid = false;
  sv->geo_valid = false;
  sv->drop_graph();
  // a lagged preconditioner survives pc_refresh - 1 surface updates (right
  // preconditioning: it steers the iteration only, the tolerance is on the true residual)
  if (sv->pc_valid && sv->pc_nves == n_ves && sv->pc_age + 1 < sv->pc_refresh)
    sv->pc_age++;
  else
    sv->pc_valid = false;
  return VES3D_OK;
}

int ves3d_sv_set_density_sl(ves3d_sv* sv, const double* f, int is_device) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(f != nullptr, "f is null");
  if (!sv->have_src) {
    set_error("set_density_sl before set_src_coord");
    return VES3D_ERR_STATE;
  }
  if ((s = copy_in(sv->F, f, (size_t)sv->npts() * 3, is_device, sv->stream))) return s;
  sv->have_den = true;
  sv->parts_valid = false;
  return VES3D_OK;
}

int ves3d_sv_set_density_dl(ves3d_sv* sv, const double* g, int is_device) {
  int s = check_sv(sv);
  if (s) return s;
  if (!sv->have_src) {
    set_error("set_density_dl before set_src_coord");
    return VES3D_ERR_STATE;
  }
  if (!g) {  // SetDensityDL(NULL): the double layer off
    if (sv->have_dl) sv->drop_graph();
    sv->have_dl = false;
    sv->parts_valid = false;
    return VES3D_OK;
  }
  if ((s = alloc_dl(sv))) return s;
  if ((s = copy_in(sv->G, g, (size_t)sv->npts() * 3, is_device, sv->stream))) return s;
  if (!sv->have_dl) sv->drop_graph();  // a captured evaluation without the double layer
  sv->have_dl = true;
  sv->parts_valid = false;
  return VES3D_OK;
}

int ves3d_sv_get_dl_matrix(ves3d_sv* sv, double* DL, int is_device) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(DL != nullptr, "DL is null");
  if (!sv->have_src || !sv->have_dl) {
    set_error("no surfaces or no double-layer density set");
    return VES3D_ERR_STATE;
  }
  if (!sv->dl_valid && (s = run_setup(sv, true))) return s;
  const size_t n = 3 * (size_t)ncoef_(sv->p);
  return copy_out(DL, sv->DL, (size_t)sv->nves * n * n, is_device, sv->stream);
}

int ves3d_sv_set_trg_coord(ves3d_sv* sv, const double* T, long n_trg, int is_device) {
  int s = check_sv(sv);
  if (s) return s;
  if (!T || n_trg == 0) {  // SetTrgCoord(NULL): the surface points again
    sv->trg_n = 0;
    return VES3D_OK;
  }
  VES3D_ARG(n_trg > 0, "n_trg < 0");
  if (n_trg > sv->trg_cap) {
    dfree(sv->trg);
    dfree(sv->vtrg);
    sv->trg = sv->vtrg = nullptr;
    sv->trg_cap = 0;
    if ((s = dalloc(&sv->trg, 3 * (size_t)n_trg)) || (s = dalloc(&sv->vtrg, 3 * (size_t)n_trg))) return s;
    sv->trg_cap = n_trg;
  }
  if ((s = copy_in(sv->trg, T, 3 * (size_t)n_trg, is_device, sv->stream))) return s;
  sv->trg_n = n_trg;
  return VES3D_OK;
}

int ves3d_sv_eval_trg(ves3d_sv* sv, double* vel, int is_device) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(vel != nullptr, "vel is null");
  if (!sv->have_src || !sv->have_den || sv->trg_n <= 0) {
    set_error("eval_trg needs surfaces, a single-layer density and targets");
    return VES3D_ERR_STATE;
  }
  NvtxRange nvtx("ves3d targets");
  const DevTables& T = sv->tab->d;
  cudaStream_t st = sv->stream;
  if ((s = launch_far_density(sv->F, sv->area, sv->nves, sv->p, T.smooth_w0, sv->den, st))) return s;
  const double *nrm = nullptr, *dden = nullptr;
  if (sv->have_dl) {
    if ((s = launch_unit_normals(sv->Xt, sv->Xp, sv->nves, sv->p, sv->nrm, st))) return s;
    if ((s = launch_far_density(sv->G, sv->area, sv->nves, sv->p, T.smooth_w0, sv->dden, st))) return s;
    nrm = sv->nrm;
    dden = sv->dden;
  }
  if (sv->near_on) {
    if ((s = eval_trg_near(sv))) return s;
  } else if ((s = launch_targets_f64(sv->pos, sv->den, nrm, dden, sv->npts(), sv->trg, sv->trg_n, sv->vtrg, st))) {
    return s;
  }
  return copy_out(vel, sv->vtrg, 3 * (size_t)sv->trg_n, is_device, st);
}

int ves3d_sv_set_near_singular(ves3d_sv* sv, int on) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(sv->p + 1 <= 32, "the near-singular correction supports orders up to 31");
  sv->near_on = on != 0;
  return VES3D_OK;
}

int ves3d_sv_near_info(ves3d_sv* sv, double* r_near, long* n_near) {
  int s = check_sv(sv);
  if (s) return s;
  if (r_near) *r_near = sv->near_r;
  if (n_near) {
    long n = 0;
    if (sv->near_on && sv->nu_count && sv->trg_n > 0) {
      std::vector<int> c(sv->trg_n);
      VES3D_CK(cudaMemcpyAsync(c.data(), sv->nu_count, c.size() * sizeof(int), cudaMemcpyDeviceToHost, sv->stream));
      VES3D_CK(cudaStreamSynchronize(sv->stream));
      for (int x : c) n += x;
    }
    *n_near = n;
  }
  return VES3D_OK;
}

int ves3d_sv_set_order_up(ves3d_sv* sv, int sh_order_up) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(sh_order_up >= sv->p && sh_order_up <= 128, "sh_order_up must be in [sh_order, 128]");
  if (sh_order_up == sv->pup) return VES3D_OK;
  std::unique_ptr<TablesOwner> t(new TablesOwner());
  build_tables(sv->p, sh_order_up, t->h);
  if ((s = t->upload(sv->stream))) return s;
  VES3D_CK(cudaDeviceSynchronize());  // nothing queued still reads the old tables
  sv->tab = std::move(t);
  sv->pup = sh_order_up;
  sv->sl_valid = sv->dl_valid = false;  // self matrices of the new order on next use
  sv->parts_valid = false;
  sv->pc_valid = false;
  sv->free_scratch();  // its size depends on the order
  sv->drop_graph();
  return VES3D_OK;
}

int ves3d_sv_monitor_error(ves3d_sv* sv, double tol, double* err3, double* total) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(std::isfinite(tol) && tol > 0.0, "tol must be positive");
  if (!sv->have_src) {
    set_error("monitor_error before set_src_coord");
    return VES3D_ERR_STATE;
  }
  NvtxRange nvtx("ves3d monitor");
  const size_t n = (size_t)sv->npts() * 3;
  if ((s = alloc_dl(sv))) return s;
  // save the densities (src/StokesVelocity.cc:556-562)
  const bool had_den = sv->have_den, had_dl = sv->have_dl;
  std::vector<double> keepF, keepG;
  if (had_den) {
    keepF.resize(n);
    if ((s = copy_out(keepF.data(), sv->F, n, 0, sv->stream))) return s;
  }
  if (had_dl) {
    keepG.resize(n);
    if ((s = copy_out(keepG.data(), sv->G, n, 0, sv->stream))) return s;
  }
  // no single layer, double-layer density 1 (:564-578)
  const std::vector<double> ones(n, 1.0);
  VES3D_CK(cudaMemsetAsync(sv->F, 0, n * sizeof(double), sv->stream));
  if ((s = copy_in(sv->G, ones.data(), n, 0, sv->stream))) return s;
  sv->have_den = sv->have_dl = true;
  s = run_eval(sv, true);
  std::vector<double> vs(n), vf(n);
  if (!s) s = copy_out(vs.data(), sv->Vself, n, 0, sv->stream);
  if (!s) s = copy_out(vf.data(), sv->Vfar, n, 0, sv->stream);
  // restore (:627-633)
  int r = VES3D_OK;
  if (had_den) r = copy_in(sv->F, keepF.data(), n, 0, sv->stream);
  if (!r && had_dl) r = copy_in(sv->G, keepG.data(), n, 0, sv->stream);
  if (!r) r = cuda_status(cudaStreamSynchronize(sv->stream), "restore densities", __FILE__, __LINE__);
  sv->have_den = had_den;
  sv->have_dl = had_dl;
  sv->parts_valid = false;
  if (s) return s;
  if (r) return r;
  // error norms (:615-622): the self part against -1/2, the far part against 0; this build
  // has no near-singular correction (its norm is 0)
  double e0 = 0.0, e2 = 0.0;
  for (size_t i = 0; i < n; i++) {
    e0 = std::max(e0, std::fabs(vs[i] + 0.5));
    e2 = std::max(e2, std::fabs(vf[i]));
  }
  // the self order follows the error (:636-645); the far field here is exact on the order-p
  // grid and has no order of its own
  int pup = sv->pup;
  if (e0 > tol)
    pup += 2;
  else if (e0 < 0.5 * tol)
    pup -= 2;
  pup = std::max(sv->p, std::min(pup, 128));
  if (pup != sv->pup && (s = ves3d_sv_set_order_up(sv, pup))) return s;
  if (err3) {
    err3[0] = e0;
    err3[1] = 0.0;
    err3[2] = e2;
  }
  if (total) *total = e0 + e2;
  return VES3D_OK;
}

int ves3d_sv_get_order_up(ves3d_sv* sv, int* sh_order_up) {
  VES3D_ARG(sv != nullptr && sh_order_up != nullptr, "null argument");
  *sh_order_up = sv->pup;
  return VES3D_OK;
}

int ves3d_sv_setup(ves3d_sv* sv) {
  int s = check_sv(sv);
  if (s) return s;
  if (!sv->have_src) {
    set_error("setup before set_src_coord");
    return VES3D_ERR_STATE;
  }
  return run_setup(sv);
}

int ves3d_sv_eval(ves3d_sv* sv, double* vel, int is_device) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(vel != nullptr, "vel is null");
  if ((s = run_eval(sv, sv->have_dl))) return s;
  return copy_out(vel, sv->V, (size_t)sv->npts() * 3, is_device, sv->stream);
}

int ves3d_sv_eval_resident(ves3d_sv* sv) {
  int s = check_sv(sv);
  if (s) return s;
  return run_eval(sv, sv->have_dl);
}

int ves3d_set_autotune(int on) { return set_autotune(on); }

int ves3d_set_far_shape(int waves, int threads, int targets_per_thread) {
  return set_far_shape(waves, threads, targets_per_thread);
}

int ves3d_autotune_report(char* buf, size_t cap, size_t* len) {
  VES3D_ARG(len != nullptr, "len is null");
  const std::string r = autotune_report();
  *len = r.size();
  if (buf && cap) {
    const size_t n = std::min(cap - 1, r.size());
    memcpy(buf, r.data(), n);
    buf[n] = 0;
  }
  return VES3D_OK;
}

int ves3d_sv_capture_eval(ves3d_sv* sv) {
  int s = check_sv(sv);
  if (s) return s;
  if (!sv->have_src) {
    set_error("no surfaces set");
    return VES3D_ERR_STATE;
  }
  if (sv->stream == nullptr) {
    set_error("graph capture needs a non-default stream");
    return VES3D_ERR_STATE;
  }
  sv->drop_graph();
  if (!sv->sl_valid && (s = run_setup(sv))) return s;
  // one eager pass first: every launcher sets its kernel attributes outside the capture
  sv->have_den = true;
  if ((s = run_eval(sv, sv->have_dl))) return s;
  VES3D_CK(cudaStreamBeginCapture(sv->stream, cudaStreamCaptureModeThreadLocal));
  s = run_eval_body(sv, sv->have_dl);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(sv->stream, &g);
  if (!s && e != cudaSuccess) s = cuda_status(e, "cudaStreamEndCapture", __FILE__, __LINE__);
  if (s) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  sv->graph = g;
  const cudaError_t ei = cudaGraphInstantiate(&sv->graph_exec, g, 0);
  if (ei != cudaSuccess) {
    sv->drop_graph();
    return cuda_status(ei, "cudaGraphInstantiate", __FILE__, __LINE__);
  }
  return VES3D_OK;
}

int ves3d_sv_launch_eval_graph(ves3d_sv* sv) {
  int s = check_sv(sv);
  if (s) return s;
  if (!sv->graph_exec) {
    set_error("no captured evaluation (call ves3d_sv_capture_eval after setting the surfaces)");
    return VES3D_ERR_STATE;
  }
  VES3D_CK(cudaGraphLaunch(sv->graph_exec, sv->stream));
  VES3D_LAUNCHED();
  sv->parts_valid = true;
  return VES3D_OK;
}

int ves3d_sv_get_self_matrix(ves3d_sv* sv, double* SL, int is_device) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(SL != nullptr, "SL is null");
  if (!sv->have_src) {
    set_error("no surfaces set");
    return VES3D_ERR_STATE;
  }
  if (!sv->sl_valid && (s = run_setup(sv))) return s;
  const size_t n = 3 * (size_t)ncoef_(sv->p);
  return copy_out(SL, sv->SL, (size_t)sv->nves * n * n, is_device, sv->stream);
}

int ves3d_sv_get_parts(ves3d_sv* sv, double* vel_self, double* vel_far, int is_device) {
  int s = check_sv(sv);
  if (s) return s;
  if (!sv->parts_valid) {
    set_error("no evaluation since the last input change");
    return VES3D_ERR_STATE;
  }
  const size_t n = (size_t)sv->npts() * 3;
  if (vel_self && (s = copy_out(vel_self, sv->Vself, n, is_device, sv->stream))) return s;
  if (vel_far && (s = copy_out(vel_far, sv->Vfar, n, is_device, sv->stream))) return s;
  return VES3D_OK;
}

int ves3d_sv_stage_times(ves3d_sv* sv, float* ms) {
  VES3D_ARG(sv != nullptr && ms != nullptr, "null argument");
  for (int i = 0; i < 4; i++) ms[i] = sv->ms[i];
  return VES3D_OK;
}

int ves3d_sv_far_dl_time(ves3d_sv* sv, float* ms) {
  VES3D_ARG(sv != nullptr && ms != nullptr, "null argument");
  *ms = sv->far_dl_ms;
  return VES3D_OK;
}

int ves3d_sv_device_buffer(ves3d_sv* sv, int which, double** ptr, size_t* n_elems) {
  VES3D_ARG(sv != nullptr && ptr != nullptr, "null argument");
  if (!sv->have_src) {
    set_error("no surfaces set");
    return VES3D_ERR_STATE;
  }
  double* p = which == 0 ? sv->X : which == 1 ? sv->F : which == 2 ? sv->V : nullptr;
  VES3D_ARG(p != nullptr, "which must be 0, 1 or 2");
  *ptr = p;
  if (n_elems) *n_elems = (size_t)sv->npts() * 3;
  if (which == 1) {
    sv->have_den = true;  // caller writes the density in place
    sv->parts_valid = false;
  }
  return VES3D_OK;
}

int ves3d_sht_forward(const double* X, long n_fun, int p0, int p1, double* S, void* stream) {
  VES3D_ARG(X && S, "null pointer");
  VES3D_ARG(p0 >= 1 && p1 >= 1 && p0 <= 128 && p1 <= 128, "orders must be in [1, 128]");
  VES3D_ARG(n_fun >= 0, "n_fun < 0");
  cudaStream_t st = (cudaStream_t)stream;
  AnalysisTables A;
  build_analysis_tables(p0, p1, A);
  std::vector<int> blk, jf;
  coef_blocks(p1, blk, jf);
  double *dfour = nullptr, *dleg = nullptr;
  int* djf = nullptr;
  int s = 0;
  s |= dupload(&dfour, A.four, st);
  s |= dupload(&dleg, A.leg, st);
  s |= dupload(&djf, jf, st);
  if (!s) s = launch_analysis(X, n_fun, p0, p1, dfour, dleg, djf, S, st);
  cudaError_t e = cudaStreamSynchronize(st);
  dfree(dfour);
  dfree(dleg);
  dfree(djf);
  if (s) return s;
  VES3D_CK(e);
  return VES3D_OK;
}

int ves3d_sht_backward(const double* S, long n_fun, int p0, int p1, double* X, double* X_theta, double* X_phi,
                       void* stream) {
  VES3D_ARG(S && X, "null pointer");
  VES3D_ARG(p0 >= 1 && p1 >= 1 && p0 <= 128 && p1 <= 128, "orders must be in [1, 128]");
  VES3D_ARG(n_fun >= 0, "n_fun < 0");
  cudaStream_t st = (cudaStream_t)stream;
  SynthTables syn;
  build_synth_tables(p0, p1, syn);
  std::vector<int> blk, jf;
  coef_blocks(p0, blk, jf);
  double *dl = nullptr, *ddl = nullptr, *df = nullptr, *ddf = nullptr;
  int* db = nullptr;
  int s = 0;
  s |= dupload(&dl, syn.leg, st);
  s |= dupload(&ddl, syn.dleg, st);
  s |= dupload(&df, syn.four, st);
  s |= dupload(&ddf, syn.dfour, st);
  s |= dupload(&db, blk, st);
  if (!s) s = launch_synthesis(S, n_fun, p0, p1, dl, ddl, df, ddf, db, X, X_theta, X_phi, st);
  cudaError_t e = cudaStreamSynchronize(st);
  dfree(dl);
  dfree(ddl);
  dfree(df);
  dfree(ddf);
  dfree(db);
  if (s) return s;
  VES3D_CK(e);
  return VES3D_OK;
}

int ves3d_sht_rotate_all(const double* S, long n_vec, int p, double* R, void* stream) {
  VES3D_ARG(S && R, "null pointer");
  VES3D_ARG(p >= 1 && p <= 127, "order must be in [1, 127]");
  VES3D_ARG(n_vec >= 0, "n_vec < 0");
  if (n_vec == 0) return VES3D_OK;
  cudaStream_t st = (cudaStream_t)stream;
  TablesOwner tab;  // rotation blocks and phase tables of order p (freed on return)
  build_tables(p, 2 * p, tab.h);
  int s = tab.upload(st);
  if (!s) s = launch_rotate_all(S, n_vec, tab.d, R, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  if (s) return s;
  VES3D_CK(e);
  return VES3D_OK;
}

int ves3d_move_pole(const double* X, long n_fun, int p, int trg_i, int trg_j, double* Y, void* stream) {
  VES3D_ARG(X && Y, "null pointer");
  VES3D_ARG(p >= 1 && p <= 127, "order must be in [1, 127]");
  VES3D_ARG(n_fun >= 0, "n_fun < 0");
  VES3D_ARG(trg_i >= 0 && trg_i <= p && trg_j >= 0 && trg_j < 2 * p, "target outside the (p + 1) x 2p grid");
  if (n_fun == 0) return VES3D_OK;
  cudaStream_t st = (cudaStream_t)stream;
  TablesOwner tab;  // transforms and rotation tables of order p (freed on return)
  build_tables(p, p, tab.h);
  int s = tab.upload(st);
  const DevTables& T = tab.d;
  const size_t nc = ncoef_(p);
  double* work = nullptr;  // coefficients, then rotated coefficients
  if (!s) s = cuda_status(cudaMallocAsync((void**)&work, 2 * n_fun * nc * sizeof(double), st), "cudaMallocAsync",
                          __FILE__, __LINE__);
  if (!s) s = launch_grid2shc(X, n_fun, p, T.ana_four, T.ana_leg, T.jf_of_coef, work, st);
  if (!s) s = launch_rotate_one(work, n_fun, trg_i, trg_j, T, work + n_fun * nc, st);
  if (!s)
    s = launch_synthesis(work + n_fun * nc, n_fun, p, p, T.syn0_leg, T.syn0_dleg, T.syn0_four, T.syn0_dfour,
                         T.blk_off, Y, nullptr, nullptr, st);
  if (work) cudaFreeAsync(work, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  if (s) return s;
  VES3D_CK(e);
  return VES3D_OK;
}

int ves3d_cuda_stokes_f32(int src_m, int trg_m, int n, int t_head, int t_tail, const float* T, const float* S,
                          const float* D, float* U, const float* Q, void* stream) {
  VES3D_ARG(T && S && D && U, "null pointer");
  VES3D_ARG(src_m >= 0 && trg_m >= 0 && n >= 0, "negative size");
  VES3D_ARG(t_head >= 0 && t_tail <= trg_m && t_head <= t_tail, "target range outside [0, trg_m]");
  return launch_direct_stokes_f32(src_m, trg_m, n, t_head, t_tail, T, S, D, U, Q, (cudaStream_t)stream);
}

int ves3d_sht_backward_d2(const double* S, long n_fun, int p, double* X_uu, double* X_vv, double* X_uv,
                          void* stream) {
  VES3D_ARG(S && (X_uu || X_vv || X_uv), "null pointer");
  VES3D_ARG(p >= 1 && p <= 127, "order must be in [1, 127]");
  VES3D_ARG(n_fun >= 0, "n_fun < 0");
  if (n_fun == 0) return VES3D_OK;
  cudaStream_t st = (cudaStream_t)stream;
  TablesOwner tab;  // order-p synthesis tables with their second derivatives (freed on return)
  build_tables(p, 2 * p, tab.h);
  int s = tab.upload(st);
  const DevTables& T = tab.d;
  double* xu = nullptr;  // X_u, computed alongside X_uv and X_uu (not returned)
  if (!s && (X_uu || X_uv)) {
    s = dalloc(&xu, (size_t)n_fun * ngrid_(p));
    // values from d/du P (X_u), their v-derivative (X_uv), and d2/du2 P (X_uu)
    if (!s)
      s = launch_synthesis(S, n_fun, p, p, T.syn0_dleg, T.syn0_d2leg, T.syn0_four, T.syn0_dfour, T.blk_off, xu, X_uv,
                           X_uu, st);
  }
  if (!s && X_vv)
    s = launch_synthesis(S, n_fun, p, p, T.syn0_leg, T.syn0_leg, T.syn0_d2four, T.syn0_d2four, T.blk_off, X_vv,
                         nullptr, nullptr, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  dfree(xu);
  if (s) return s;
  VES3D_CK(e);
  return VES3D_OK;
}

int ves3d_sht_filter_coeffs(int p, int filter_freq, double exponent, double* coeff) {
  VES3D_ARG(coeff != nullptr, "coeff is null");
  VES3D_ARG(p >= 1 && p <= 128, "order must be in [1, 128]");
  const int freq = filter_freq == -1 ? 2 * p / 3 : filter_freq;
  VES3D_ARG(freq >= 0, "filter frequency must be >= 0 (or -1 for 2p/3)");
  int i = 0;
  for (int jf = 0; jf < 2 * p; jf++) {
    const int m = (jf + 1) / 2;
    for (int n = m; n <= p; n++, i++) {
      if (exponent <= 0)
        coeff[i] = n > freq ? 0.0 : 1.0;  // lowPassFilter: degrees above freq removed
      else
        coeff[i] = n >= freq ? 0.0 : 1.0 - std::pow((double)n / freq, exponent);
    }
  }
  return VES3D_OK;
}

int ves3d_sht_scale_freq(const double* shc_in, long n_fun, int p, const double* scale, double* shc_out,
                         void* stream) {
  VES3D_ARG(shc_in && scale && shc_out, "null pointer");
  VES3D_ARG(p >= 1 && p <= 128, "order must be in [1, 128]");
  VES3D_ARG(n_fun >= 0, "n_fun < 0");
  cudaStream_t st = (cudaStream_t)stream;
  int s = launch_scale_freq(shc_in, n_fun, ncoef_(p), scale, shc_out, st);
  if (s) return s;
  VES3D_CK(cudaStreamSynchronize(st));
  return VES3D_OK;
}

int ves3d_sht_lowpass(const double* in, long n_fun, int p, int filter_freq, double exponent, double* out,
                      void* stream) {
  VES3D_ARG(in && out, "null pointer");
  VES3D_ARG(p >= 1 && p <= 128, "order must be in [1, 128]");
  VES3D_ARG(n_fun >= 0, "n_fun < 0");
  if (n_fun == 0) return VES3D_OK;
  const int nc = ncoef_(p);
  std::vector<double> coeff(nc);
  int s = ves3d_sht_filter_coeffs(p, filter_freq, exponent, coeff.data());
  if (s) return s;
  cudaStream_t st = (cudaStream_t)stream;
  double *dc = nullptr, *shc = nullptr;
  if ((s = dupload(&dc, coeff, st))) return s;
  if ((s = dalloc(&shc, (size_t)n_fun * nc))) {
    dfree(dc);
    return s;
  }
  s = ves3d_sht_forward(in, n_fun, p, p, shc, stream);
  if (!s) s = ves3d_sht_scale_freq(shc, n_fun, p, dc, shc, stream);
  if (!s) s = ves3d_sht_backward(shc, n_fun, p, p, out, nullptr, nullptr, stream);
  cudaStreamSynchronize(st);
  dfree(dc);
  dfree(shc);
  return s;
}

int ves3d_sht_pole(const double* S, long n_fun, int p, double* P, void* stream) {
  VES3D_ARG(S && P, "null pointer");
  VES3D_ARG(p >= 1 && p <= 128, "order must be in [1, 128]");
  VES3D_ARG(n_fun >= 0, "n_fun < 0");
  if (n_fun == 0) return VES3D_OK;
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<double> qp;
  pole_table(p, qp);
  double* dq = nullptr;
  int s = dupload(&dq, qp, st);
  if (!s) s = launch_shc2pole(S, n_fun, p, dq, P, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  dfree(dq);
  if (s) return s;
  VES3D_CK(e);
  return VES3D_OK;
}

int ves3d_tables_export(int p0, int p1, const char* name, double* out, size_t cap, size_t* n) {
  VES3D_ARG(name != nullptr && n != nullptr, "null argument");
  VES3D_ARG(p0 >= 2 && p0 <= 64 && p1 >= p0 && p1 <= 128, "orders out of range");
  ShTables T;
  build_tables(p0, p1, T);
  const std::vector<double>* v = nullptr;
  std::string nm(name);
  if (nm == "nodes0") v = &T.x0;
  else if (nm == "weights0") v = &T.w0;
  else if (nm == "nodes1") v = &T.x1;
  else if (nm == "smooth_w0") v = &T.smooth_w0;
  else if (nm == "sing_w") v = &T.sing_w;
  else if (nm == "mr") v = &T.mr;
  else if (nm == "ana_leg") v = &T.ana.leg;
  else if (nm == "ana_four") v = &T.ana.four;
  else if (nm == "syn1_leg") v = &T.syn1.leg;
  else if (nm == "syn1_dleg") v = &T.syn1.dleg;
  else if (nm == "syn1_four") v = &T.syn1.four;
  else if (nm == "syn1_dfour") v = &T.syn1.dfour;
  else if (nm == "qp") v = &T.qp;
  VES3D_ARG(v != nullptr, "unknown table name");
  *n = v->size();
  if (out) {
    VES3D_ARG(cap >= v->size(), "output capacity too small");
    std::memcpy(out, v->data(), v->size() * sizeof(double));
  }
  return VES3D_OK;
}

int ves3d_cuda_stokes_f64(int src_m, int trg_m, int n, int t_head, int t_tail, const double* T, const double* S,
                          const double* D, double* U, const double* Q, void* stream) {
  VES3D_ARG(T && S && D && U, "null pointer");
  VES3D_ARG(src_m >= 0 && trg_m >= 0 && n >= 0, "negative size");
  VES3D_ARG(t_head >= 0 && t_tail <= trg_m && t_head <= t_tail, "target range outside [0, trg_m]");
  return launch_direct_stokes_f64(src_m, trg_m, n, t_head, t_tail, T, S, D, U, Q, (cudaStream_t)stream);
}

int ves3d_cuda_stokes_double_layer_f64(int src_m, int trg_m, int n, int t_head, int t_tail, const double* T,
                                       const double* S, const double* N, const double* D, double* U, const double* Q,
                                       void* stream) {
  VES3D_ARG(T && S && N && D && U, "null pointer");
  VES3D_ARG(src_m >= 0 && trg_m >= 0 && n >= 0, "negative size");
  VES3D_ARG(t_head >= 0 && t_tail <= trg_m && t_head <= t_tail, "target range outside [0, trg_m]");
  return launch_direct_stokes_dl_f64(src_m, trg_m, n, t_head, t_tail, T, S, N, D, U, Q, (cudaStream_t)stream);
}

int ves3d_stokes_alltoall_device_f64(const double* src, const double* den, size_t np, double* pot, void* stream) {
  VES3D_ARG(src && den && pot, "null pointer");
  return launch_alltoall_f64(src, den, (long)np, pot, (cudaStream_t)stream);
}

struct InteractionWorkspace {
  double* buf = nullptr;
  size_t cap = 0;
  cudaStream_t st = nullptr;
};

void ves3d_stokes_alltoall_f64(const double* src, const double* den, size_t np, double* pot, void** ctx) {
  auto fail = [&](void) {
    for (size_t i = 0; i < 3 * np; i++) pot[i] = __builtin_nan("");
  };
  if (!src || !den || !pot) {
    set_error("invalid argument: null pointer");
    if (pot) fail();
    return;
  }
  if (np == 0) return;  // nothing to compute
  InteractionWorkspace local;
  InteractionWorkspace* ws = &local;
  if (ctx) {
    if (!*ctx) *ctx = new InteractionWorkspace();
    ws = (InteractionWorkspace*)*ctx;
  }
  const size_t need = 9 * np;
  if (ws->cap < need) {
    if (ws->buf) cudaFree(ws->buf);
    ws->buf = nullptr;
    ws->cap = 0;
    if (cudaMalloc((void**)&ws->buf, need * sizeof(double)) != cudaSuccess) {
      set_error("cudaMalloc of %zu bytes failed", need * sizeof(double));
      fail();
      return;
    }
    ws->cap = need;
  }
  if (!ws->st && cudaStreamCreateWithFlags(&ws->st, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("cudaStreamCreate failed");
    fail();
    return;
  }
  double *dsrc = ws->buf, *dden = ws->buf + 3 * np, *dpot = ws->buf + 6 * np;
  int s = VES3D_OK;
  if (cudaMemcpyAsync(dsrc, src, 3 * np * sizeof(double), cudaMemcpyHostToDevice, ws->st) != cudaSuccess ||
      cudaMemcpyAsync(dden, den, 3 * np * sizeof(double), cudaMemcpyHostToDevice, ws->st) != cudaSuccess)
    s = VES3D_ERR_CUDA;
  if (!s) s = launch_alltoall_f64(dsrc, dden, (long)np, dpot, ws->st);
  if (!s && cudaMemcpyAsync(pot, dpot, 3 * np * sizeof(double), cudaMemcpyDeviceToHost, ws->st) != cudaSuccess)
    s = VES3D_ERR_CUDA;
  if (cudaStreamSynchronize(ws->st) != cudaSuccess) s = VES3D_ERR_CUDA;
  if (s) {
    if (!g_err[0]) set_error("all-to-all interaction failed");
    fail();
  }
  if (!ctx) {
    cudaFree(ws->buf);
    cudaStreamDestroy(ws->st);
  }
}

void ves3d_interaction_free(void** ctx) {
  if (!ctx || !*ctx) return;
  InteractionWorkspace* ws = (InteractionWorkspace*)*ctx;
  if (ws->buf) cudaFree(ws->buf);
  if (ws->st) cudaStreamDestroy(ws->st);
  delete ws;
  *ctx = nullptr;
}

}  // extern "C"

// ======================================================================================
// Surface geometry, tractions, implicit step
// ======================================================================================
namespace {

int ensure_implicit_buffers(ves3d_sv* sv) {
  if (sv->geo_cap >= sv->nves) return VES3D_OK;
  sv->free_implicit();
  const size_t ng = ngrid_(sv->p), nc = ncoef_(sv->p), nv = sv->nves;
  int s = 0;
  s |= dalloc(&sv->geo, nv * kGeoComps * ng);
  s |= dalloc(&sv->wc, nv * 3 * nc);
  for (auto& q : sv->w) s |= dalloc(&q, nv * 3 * ng);
  if (s) {
    sv->free_implicit();
    return s;
  }
  sv->geo_cap = sv->nves;
  return VES3D_OK;
}

// coefficient derivatives at order p: which = 0 -> (value, v, u); 1 -> (u, uv, uu); 2 -> vv
int synth_d(ves3d_sv* sv, const double* coef, long nfun, int which, double* a, double* b, double* c) {
  const DevTables& T = sv->tab->d;
  const int p = sv->p;
  if (which == 0)
    return launch_synthesis(coef, nfun, p, p, T.syn0_leg, T.syn0_dleg, T.syn0_four, T.syn0_dfour, T.blk_off, a, b, c,
                            sv->stream);
  if (which == 1)
    return launch_synthesis(coef, nfun, p, p, T.syn0_dleg, T.syn0_d2leg, T.syn0_four, T.syn0_dfour, T.blk_off, a, b,
                            c, sv->stream);
  return launch_synthesis(coef, nfun, p, p, T.syn0_leg, T.syn0_leg, T.syn0_d2four, T.syn0_d2four, T.blk_off, a,
                          nullptr, nullptr, sv->stream);
}

int grid2shc_p(ves3d_sv* sv, const double* in, long nfun, double* out) {
  const DevTables& T = sv->tab->d;
  return launch_grid2shc(in, nfun, sv->p, T.ana_four, T.ana_leg, T.jf_of_coef, out, sv->stream);
}

// The reference Surface's low-pass filter (SHTrans::lowPassFilter at diff_filter_freq,
// src/Surface.cc:310-311, :336, :371, :564) of nfun grid functions in place, through the
// coefficient scratch wc (room for nfun functions); nothing when the filter is off.
int filter_fields(ves3d_sv* sv, double* wc, double* f, long nfun) {
  if (!sv->filter_freq || nfun <= 0) return VES3D_OK;
  int s;
  const int nc = ncoef_(sv->p);
  if ((s = grid2shc_p(sv, f, nfun, wc))) return s;
  if ((s = launch_scale_freq(wc, nfun, nc, sv->filt, wc, sv->stream))) return s;
  return synth_d(sv, wc, nfun, 0, f, nullptr, nullptr);
}

int ensure_geometry(ves3d_sv* sv) {
  int s;
  if ((s = ensure_implicit_buffers(sv))) return s;
  if (sv->geo_valid) return VES3D_OK;
  const long nv = sv->nves, nf = 3 * nv;
  const int ng = ngrid_(sv->p);
  double** w = sv->w;
  // w0 value, w1 v, w2 u, w3 (u again), w4 uv, w5 uu, w6 vv
  if ((s = synth_d(sv, sv->Sx, nf, 0, w[0], w[1], w[2]))) return s;
  if ((s = synth_d(sv, sv->Sx, nf, 1, w[3], w[4], w[5]))) return s;
  if ((s = synth_d(sv, sv->Sx, nf, 2, w[6], nullptr, nullptr))) return s;
  if ((s = launch_geometry(w[2], w[1], w[5], w[4], w[6], nv, ng, sv->geo, sv->stream))) return s;
  if (sv->filter_freq) {
    // H and K (record components 13, 14) filtered as Surface::updateAll does
    const size_t row = ng * sizeof(double), pitch = kGeoComps * row;
    for (int k = 0; k < 2; k++)
      VES3D_CK(cudaMemcpy2DAsync(w[0] + k * nv * ng, row, sv->geo + (13L + k) * ng, pitch, row, (size_t)nv,
                                 cudaMemcpyDeviceToDevice, sv->stream));
    if ((s = filter_fields(sv, sv->wc, w[0], 2 * nv))) return s;
    for (int k = 0; k < 2; k++)
      VES3D_CK(cudaMemcpy2DAsync(sv->geo + (13L + k) * ng, pitch, w[0] + k * nv * ng, row, row, (size_t)nv,
                                 cudaMemcpyDeviceToDevice, sv->stream));
  }
  sv->geo_valid = true;
  return VES3D_OK;
}

// The space the implicit operator acts on: nv field vesicles with their work fields and
// coefficient scratch. Normally the suspension itself; when several operator
// applications are batched (the preconditioner assembly), nv = k nves field vesicles,
// copy q of vesicle v at index q nves + v, which use the geometry record and the self
// matrix of vesicle v.
struct OpSpace {
  long nv = 0;
  double* w[8] = {};
  double* wc = nullptr;
  double* fc = nullptr;  // batched self part: density / velocity coefficients [nv][3 nc]
  double* vc = nullptr;
};

OpSpace base_space(ves3d_sv* sv) {
  OpSpace sp;
  sp.nv = sv->nves;
  for (int k = 0; k < 8; k++) sp.w[k] = sv->w[k];
  sp.wc = sv->wc;
  return sp;
}

// grad of a scalar field (in [nv][ng]) -> out [nv][3][ng]; uses w6, w7 and wc
int op_grad(ves3d_sv* sv, const OpSpace& sp, const double* in, double* out) {
  int s;
  const long nv = sp.nv;
  const int ng = ngrid_(sv->p);
  double *a = sp.w[6], *b = sp.w[7];
  if ((s = grid2shc_p(sv, in, nv, sp.wc))) return s;
  // value into out (overwritten below), v-derivative into a, u-derivative into b
  if ((s = synth_d(sv, sp.wc, nv, 0, out, a, b))) return s;
  if ((s = launch_grad_combine(b, a, sv->geo, nv, ng, out, sv->stream, sv->nves))) return s;
  return filter_fields(sv, sp.wc, out, 3 * nv);
}

// div of a vector field (in [nv][3][ng]) -> out [nv][ng] times scale; uses w5, w6, w7, wc
int op_div(ves3d_sv* sv, const OpSpace& sp, const double* in, double* out, double scale) {
  int s;
  const long nv = sp.nv;
  const int ng = ngrid_(sv->p);
  if ((s = grid2shc_p(sv, in, 3 * nv, sp.wc))) return s;
  if ((s = synth_d(sv, sp.wc, 3 * nv, 0, sp.w[5], sp.w[6], sp.w[7]))) return s;
  if ((s = launch_div_combine(sp.w[7], sp.w[6], sv->geo, nv, ng, scale, out, sv->stream, sv->nves))) return s;
  return filter_fields(sv, sp.wc, out, nv);
}

// linearised mean curvature of a displacement field; uses w4..w7, wc
int op_linH(ves3d_sv* sv, const OpSpace& sp, const double* in, double* out) {
  int s;
  const long nv = sp.nv;
  const int ng = ngrid_(sv->p);
  if ((s = grid2shc_p(sv, in, 3 * nv, sp.wc))) return s;
  if ((s = synth_d(sv, sp.wc, 3 * nv, 1, sp.w[4], sp.w[5], sp.w[6]))) return s;  // u, uv, uu
  if ((s = synth_d(sv, sp.wc, 3 * nv, 2, sp.w[7], nullptr, nullptr))) return s;    // vv
  if ((s = launch_linH_combine(sp.w[6], sp.w[5], sp.w[7], sv->geo, nv, ng, out, sv->stream, sv->nves))) return s;
  return filter_fields(sv, sp.wc, out, nv);
}

// bending traction of a scalar h (the mean curvature or its linearisation), added to add.
// scratch: w3 (gradient), w2 (Laplacian)
int op_bend_of(ves3d_sv* sv, const OpSpace& sp, const double* h, const double* add, double* out) {
  int s;
  const long nv = sp.nv;
  const int ng = ngrid_(sv->p);
  if ((s = op_grad(sv, sp, h, sp.w[3]))) return s;
  if ((s = op_div(sv, sp, sp.w[3], sp.w[2], 1.0))) return s;
  return launch_bend_combine(h, sp.w[2], sv->geo, nv, ng, sv->kappa, add, out, sv->stream, sv->nves);
}

// tension traction of sigma added to add; scratch w3
int op_tension(ves3d_sv* sv, const OpSpace& sp, const double* sigma, const double* add, double* out) {
  int s;
  const long nv = sp.nv;
  const int ng = ngrid_(sv->p);
  if ((s = op_grad(sv, sp, sigma, sp.w[3]))) return s;
  return launch_tension_combine(sigma, sp.w[3], sv->geo, nv, ng, add, out, sv->stream, sv->nves);
}

int op_grad(ves3d_sv* sv, const double* in, double* out) { return op_grad(sv, base_space(sv), in, out); }
int op_div(ves3d_sv* sv, const double* in, double* out, double scale) {
  return op_div(sv, base_space(sv), in, out, scale);
}
int op_linH(ves3d_sv* sv, const double* in, double* out) { return op_linH(sv, base_space(sv), in, out); }
int op_bend_of(ves3d_sv* sv, const double* h, const double* add, double* out) {
  return op_bend_of(sv, base_space(sv), h, add, out);
}
int op_tension(ves3d_sv* sv, const double* sigma, const double* add, double* out) {
  return op_tension(sv, base_space(sv), sigma, add, out);
}

// Self part of the single layer for every field vesicle of a batched space (the isolated
// vesicles' operator; no far field): coefficients, one read of each self matrix for all
// copies, synthesis.
int stokes_self_batch(ves3d_sv* sv, const OpSpace& sp, const double* f, double* out, const double* g = nullptr) {
  int s;
  const DevTables& T = sv->tab->d;
  const int p0 = sv->p, n = 3 * ncoef_(p0);
  if (!sv->sl_valid && (s = run_setup(sv))) return s;
  if (g && !sv->dl_valid && (s = run_setup(sv, true))) return s;
  if ((s = launch_grid2shc(f, sp.nv * 3, p0, T.ana_four, T.ana_leg, T.jf_of_coef, sp.fc, sv->stream))) return s;
  if ((s = launch_self_gemv_multi(sp.fc, sv->SL, sv->nves, (int)(sp.nv / sv->nves), n, sp.vc, sv->stream)))
    return s;
  if (g) {  // the double layer's self part of density g, added in coefficients
    if ((s = launch_grid2shc(g, sp.nv * 3, p0, T.ana_four, T.ana_leg, T.jf_of_coef, sp.fc, sv->stream))) return s;
    if ((s = launch_self_gemv_multi(sp.fc, sv->DL, sv->nves, (int)(sp.nv / sv->nves), n, sp.vc, sv->stream,
                                    /*accumulate=*/true)))
      return s;
  }
  return launch_synthesis(sp.vc, sp.nv * 3, p0, p0, T.syn0_leg, T.syn0_dleg, T.syn0_four, T.syn0_dfour, T.blk_off, out,
                          nullptr, nullptr, sv->stream);
}

// Stokes single layer of a device density f (AxisMajor) -> out (device), through the
// context's cached self matrices and far field.
// With dl, the double layer of the density already in the context's buffer G is added; the
// buffer is the operator's from then on (the context's double-layer density is cleared).
int stokes_apply(ves3d_sv* sv, const double* f, double* out, bool dl = false) {
  int s;
  const size_t n = (size_t)sv->npts() * 3;
  VES3D_CK(cudaMemcpyAsync(sv->F, f, n * sizeof(double), cudaMemcpyDeviceToDevice, sv->stream));
  sv->have_den = true;
  if (dl) sv->have_dl = false;
  if ((s = run_eval(sv, dl))) return s;
  VES3D_CK(cudaMemcpyAsync(out, sv->V, n * sizeof(double), cudaMemcpyDeviceToDevice, sv->stream));
  return VES3D_OK;
}

// work vectors of the implicit operator (beyond w[]): f, Sf [3N], h [N], y [3N], and two
// grid-space [u; sigma] vectors g1, g2 [4N] for the Galerkin form.
struct ImplicitWork {
  double *f, *Sf, *h, *y, *g1, *g2;
};

long sh_unknowns(const ves3d_sv* sv) { return 4L * sv->nves * ncoef_(sv->p); }

int implicit_work(ves3d_sv* sv, ImplicitWork& iw) {
  const size_t N = sv->npts();
  const size_t need = bicgstab_workspace_doubles(sh_unknowns(sv)) + 3 * N + 3 * N + N + 3 * N + 8 * N;
  if (sv->bws_cap < (long)need) {
    dfree(sv->bws);
    sv->bws = nullptr;
    sv->bws_cap = 0;
    int s = dalloc(&sv->bws, need);
    if (s) return s;
    sv->bws_cap = (long)need;
  }
  double* base = sv->bws + bicgstab_workspace_doubles(sh_unknowns(sv));
  iw.f = base;
  iw.Sf = base + 3 * N;
  iw.h = base + 6 * N;
  iw.y = base + 7 * N;
  iw.g1 = base + 10 * N;
  iw.g2 = base + 14 * N;
  return VES3D_OK;
}

// The implicit operator [u; sigma] -> [u - S f ; -div S f] with f = linbend(dt u) +
// gravity(dt u) + tension(sigma), in two phases around the single layer S (so that a
// polydisperse suspension can apply one S over all its order groups):
// forces: iw.f = f(x)
int implicit_forces(ves3d_sv* sv, const OpSpace& sp, const ImplicitWork& iw, const double* x) {
  int s;
  const long N = sp.nv * ngrid_(sv->p);
  const double* u = x;
  const double* sig = x + 3 * N;
  if ((s = lincomb_f64(3 * N, sv->dt, u, 0.0, u, 0.0, nullptr, iw.y, sv->stream))) return s;  // y = dt u
  if ((s = op_linH(sv, sp, iw.y, iw.h))) return s;
  if ((s = op_bend_of(sv, sp, iw.h, nullptr, iw.f))) return s;
  if (sv->drho != 0.0 &&
      (s = launch_gravity_combine(iw.y, sv->geo, sp.nv, ngrid_(sv->p), sv->drho, sv->grav, iw.f, iw.f, sv->stream,
                                  sv->nves)))
    return s;
  return op_tension(sv, sp, sig, iw.f, iw.f);
}

// finish: y = [u - Sf; -div Sf]
int implicit_finish(ves3d_sv* sv, const OpSpace& sp, const double* x, const double* Sf, double* y) {
  int s;
  const long N = sp.nv * ngrid_(sv->p);
  if ((s = lincomb_f64(3 * N, 1.0, x, -1.0, Sf, 0.0, nullptr, y, sv->stream))) return s;
  return op_div(sv, sp, Sf, y + 3 * N, -1.0);
}

// S is the context's full single layer, or the self part alone for a batched space
// (self_batch)
int ensure_contrast(ves3d_sv* sv);

int implicit_matvec(ves3d_sv* sv, const OpSpace& sp, const ImplicitWork& iw, bool self_batch, const double* x,
                    double* y) {
  int s;
  if ((s = implicit_forces(sv, sp, iw, x))) return s;
  if (!sv->contrast) {
    if ((s = self_batch ? stokes_self_batch(sv, sp, iw.f, iw.Sf) : stokes_apply(sv, iw.f, iw.Sf))) return s;
    return implicit_finish(sv, sp, x, iw.Sf, y);
  }
  // viscosity contrast (ImplicitApply, src/InterfacialVelocity.cc:934-966):
  // Sf = S[f] + D[(1 - l) u], y = [(1 + l)/2 u - Sf; -div Sf]. iw.y (dt u) is free after the forces.
  const long N = sp.nv * ngrid_(sv->p), per = 3L * ngrid_(sv->p);
  if ((s = ensure_contrast(sv)) || (s = alloc_dl(sv))) return s;
  if (self_batch) {
    if ((s = launch_scale_vesicles(x, 3 * N, per, sv->dlc, sv->nves, nullptr, 0.0, iw.y, sv->stream))) return s;
    if ((s = stokes_self_batch(sv, sp, iw.f, iw.Sf, iw.y))) return s;
  } else {
    if ((s = launch_scale_vesicles(x, 3 * N, per, sv->dlc, sv->nves, nullptr, 0.0, sv->G, sv->stream))) return s;
    if ((s = stokes_apply(sv, iw.f, iw.Sf, /*dl=*/true))) return s;
  }
  if ((s = launch_scale_vesicles(x, 3 * N, per, sv->velc, sv->nves, iw.Sf, -1.0, y, sv->stream))) return s;
  return op_div(sv, sp, iw.Sf, y + 3 * N, -1.0);
}

// Device coefficients of the viscosity contrast for the current vesicle count.
int ensure_contrast(ves3d_sv* sv) {
  if (sv->contrast_nves == sv->nves && sv->velc) return VES3D_OK;
  const long nv = sv->nves;
  if (sv->lam.size() != 1 && (long)sv->lam.size() != nv) {
    set_error("viscosity contrast was set for %ld vesicles, the surfaces have %ld", (long)sv->lam.size(), nv);
    return VES3D_ERR_STATE;
  }
  std::vector<double> vc(nv), dc(nv);
  for (long v = 0; v < nv; v++) {
    const double l = sv->lam.size() == 1 ? sv->lam[0] : sv->lam[v];
    vc[v] = 0.5 + 0.5 * l;  // VesicleProps.cc:27-32
    dc[v] = 1.0 - l;        // :34-39
  }
  dfree(sv->velc);
  dfree(sv->dlc);
  sv->velc = sv->dlc = nullptr;
  sv->contrast_nves = -1;
  int s = dupload(&sv->velc, vc, sv->stream);
  if (!s) s = dupload(&sv->dlc, dc, sv->stream);
  if (s) return s;
  VES3D_CK(cudaStreamSynchronize(sv->stream));
  sv->contrast_nves = nv;
  return VES3D_OK;
}

int implicit_matvec(ves3d_sv* sv, const double* x, double* y) {
  int s;
  ImplicitWork iw;
  if ((s = implicit_work(sv, iw))) return s;
  return implicit_matvec(sv, base_space(sv), iw, false, x, y);
}

// Galerkin maps: SH coefficients [u (3 nv fun); sigma (nv fun)] <-> grid [u; sigma]
int coef_to_grid(ves3d_sv* sv, long nv, const double* c, double* g) {
  const long N = nv * ngrid_(sv->p);
  const long nc = ncoef_(sv->p);
  int s = synth_d(sv, c, 3 * nv, 0, g, nullptr, nullptr);
  if (s) return s;
  return synth_d(sv, c + 3 * nv * nc, nv, 0, g + 3 * N, nullptr, nullptr);
}

int grid_to_coef(ves3d_sv* sv, long nv, const double* g, double* c) {
  const long N = nv * ngrid_(sv->p);
  const long nc = ncoef_(sv->p);
  int s = grid2shc_p(sv, g, 3 * nv, c);
  if (s) return s;
  return grid2shc_p(sv, g + 3 * N, nv, c + 3 * nv * nc);
}

int coef_to_grid(ves3d_sv* sv, const double* c, double* g) { return coef_to_grid(sv, sv->nves, c, g); }
int grid_to_coef(ves3d_sv* sv, const double* g, double* c) { return grid_to_coef(sv, sv->nves, g, c); }

// ImplicitApply, Galerkin form (src/InterfacialVelocity.cc:982-1052)
int implicit_matvec_sh(ves3d_sv* sv, const double* c, double* y) {
  int s;
  ImplicitWork iw;
  if ((s = implicit_work(sv, iw))) return s;
  if ((s = coef_to_grid(sv, c, iw.g1))) return s;
  if ((s = implicit_matvec(sv, iw.g1, iw.g2))) return s;
  return grid_to_coef(sv, iw.g2, y);
}

// The same on a batched space with the self part only (the isolated-vesicle operator,
// applied to sp.nv / nves coefficient vectors at once)
int implicit_matvec_sh_self_batch(ves3d_sv* sv, const OpSpace& sp, const ImplicitWork& iw, const double* c,
                                  double* y) {
  int s;
  if ((s = coef_to_grid(sv, sp.nv, c, iw.g1))) return s;
  if ((s = implicit_matvec(sv, sp, iw, true, iw.g1, iw.g2))) return s;
  return grid_to_coef(sv, sp.nv, iw.g2, y);
}

// Right-hand side [u_inf + S f_b; div(u_inf + S f_b)] (AssembleRhsVel,
// src/InterfacialVelocity.cc:716-771), again in two phases around S:
// forces: iw.f = f_b = bending traction of H (+ the explicit gravity jump on X)
int rhs_forces(ves3d_sv* sv, const ImplicitWork& iw) {
  int s;
  const int ng = ngrid_(sv->p);
  // H is geometry component 13 of every vesicle's record: one strided copy
  VES3D_CK(cudaMemcpy2DAsync(iw.h, ng * sizeof(double), sv->geo + 13L * ng, kGeoComps * ng * sizeof(double),
                             ng * sizeof(double), (size_t)sv->nves, cudaMemcpyDeviceToDevice, sv->stream));
  if ((s = op_bend_of(sv, iw.h, nullptr, iw.f))) return s;
  if (sv->drho != 0.0 &&
      (s = launch_gravity_combine(sv->X, sv->geo, sv->nves, ng, sv->drho, sv->grav, iw.f, iw.f, sv->stream)))
    return s;
  return VES3D_OK;
}

// finish: y = [u_inf + Sf; div(u_inf + Sf)]
int rhs_finish(ves3d_sv* sv, const double* Sf, double* y) {
  int s;
  const long N = sv->npts();
  if ((s = launch_shear(sv->X, sv->nves, ngrid_(sv->p), sv->shear, y, sv->stream))) return s;
  if ((s = lincomb_f64(3 * N, 1.0, y, 1.0, Sf, 0.0, nullptr, y, sv->stream))) return s;
  return op_div(sv, y, y + 3 * N, 1.0);
}

int implicit_rhs(ves3d_sv* sv, double* y) {
  int s;
  ImplicitWork iw;
  if ((s = implicit_work(sv, iw))) return s;
  if ((s = rhs_forces(sv, iw))) return s;
  if ((s = stokes_apply(sv, iw.f, iw.Sf))) return s;
  return rhs_finish(sv, iw.Sf, y);
}

int implicit_matvec_cb(void* ctx, const double* x, double* y) { return implicit_matvec_sh((ves3d_sv*)ctx, x, y); }

int implicit_matvec_fp64_cb(void* ctx, const double* x, double* y) {
  ves3d_sv* sv = (ves3d_sv*)ctx;
  sv->far_force_fp64 = 1;
  int s = implicit_matvec_sh(sv, x, y);
  sv->far_force_fp64 = 0;
  return s;
}

unsigned grid_1d(long n) {
  long b = (n + 255) / 256;
  return (unsigned)(b < 4096 ? (b < 1 ? 1 : b) : 4096);
}

// ---- preconditioners of the implicit solve -------------------------------------------
// Unknowns of the Galerkin system: [u coefficients (3 nv functions of nc); sigma
// coefficients (nv functions of nc)]. Vesicle v's unknowns, local index i in [0, 4 nc):
// i < 3 nc -> v 3 nc + i; else 3 nv nc + v nc + (i - 3 nc).
__device__ __forceinline__ long sh_global(long v, long i, long nv, int nc) {
  return i < 3 * nc ? v * 3 * nc + i : 3 * nv * nc + v * nc + (i - 3 * nc);
}

// Batched assembly: k copies of the suspension, copy q carries the unit vector of column
// j0 + q of every vesicle (field vesicle q nv + v of a space of k nv vesicles)
__device__ __forceinline__ long sh_global_b(long w, long i, long NV, int nc) {
  return i < 3 * nc ? w * 3 * nc + i : 3 * NV * nc + w * nc + (i - 3 * nc);
}

__global__ void k_unit_columns_batch(double* __restrict__ e, long nv, int k, int nc, int j0, int kq) {
  const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (long)kq * nv) return;
  const long q = g / nv, v = g - q * nv;
  e[sh_global_b(q * nv + v, j0 + q, (long)k * nv, nc)] = 1.0;
}

__global__ void k_store_columns_batch(const double* __restrict__ y, long nv, int k, int nc, int j0, int kq,
                                      double* __restrict__ A) {
  const long n = 4L * nc;
  for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < (long)kq * nv * n; g += (long)gridDim.x * blockDim.x) {
    const long i = g % n, qv = g / n;
    const long q = qv / nv, v = qv - q * nv;
    A[v * n * n + (j0 + q) * n + i] = y[sh_global_b(q * nv + v, i, (long)k * nv, nc)];
  }
}


// Constant tension is (up to quadrature error) a null mode of an isolated vesicle: the
// single layer of 2 H n over a closed surface vanishes. Shift the sigma degree-0 diagonal
// entry by the mean |diagonal| of the tension block so the block factors stably; the
// preconditioner only steers the iteration along that mode.
__global__ void k_shift_null_mode(double* __restrict__ A, long nv, int nc) {
  const long v = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const long n = 4L * nc;
  double* Av = A + v * n * n;
  double m = 0;
  for (long i = 3L * nc; i < n; i++) m += fabs(Av[i * n + i]);
  m /= nc;
  const long i0 = 3L * nc;
  Av[i0 * n + i0] += m > 0 ? m : 1.0;
}

__global__ void k_identity_blocks(double* __restrict__ A, long nv, long n) {
  for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < nv * n * n; g += (long)gridDim.x * blockDim.x) {
    const long r = g % (n * n);
    A[g] = (r % n) == (r / n) ? 1.0 : 0.0;
  }
}

__global__ void k_to_f32(const double* __restrict__ a, long n, float* __restrict__ b) {
  for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (long)gridDim.x * blockDim.x)
    b[g] = (float)a[g];
}

// y_v = M_v x_v for every vesicle (M_v column-major FP32, n x n; x, y in the global
// layout). Block (row tile of 256, vesicle): x_v staged in shared memory, each thread
// walks the columns for its row, so every column read is one coalesced 1 KB segment.
constexpr int kPcRows = 256;
__global__ void __launch_bounds__(kPcRows) k_block_gemv(const float* __restrict__ M, const double* __restrict__ x,
                                                        long nv, int nc, double* __restrict__ y) {
  extern __shared__ double xs[];
  const int n = 4 * nc;
  const long v = blockIdx.y;
  for (int i = threadIdx.x; i < n; i += blockDim.x) xs[i] = x[sh_global(v, i, nv, nc)];
  __syncthreads();
  const int row = blockIdx.x * kPcRows + threadIdx.x;
  if (row >= n) return;
  const float* Mv = M + v * (long)n * n + row;
  double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  int j = 0;
  for (; j + 4 <= n; j += 4) {
    a0 = fma((double)Mv[(long)j * n], xs[j], a0);
    a1 = fma((double)Mv[(long)(j + 1) * n], xs[j + 1], a1);
    a2 = fma((double)Mv[(long)(j + 2) * n], xs[j + 2], a2);
    a3 = fma((double)Mv[(long)(j + 3) * n], xs[j + 3], a3);
  }
  for (; j < n; j++) a0 = fma((double)Mv[(long)j * n], xs[j], a0);
  y[sh_global(v, row, nv, nc)] = (a0 + a1) + (a2 + a3);
}

// Diagonal spectral scales of the reference (InterfacialVelocity::ConfigurePrecond,
// src/InterfacialVelocity.cc:665-713), per coefficient of degree n:
//   velocity: 1 / |1 - dt n^3| (1 where that is >= 1e3 or <= 1e-10)
//   tension : (4n^2 - 1)(2n + 3) / ((n + 1)(2n^2 + 2n - 1) n)  (1 for n = 0 or ~0)
__global__ void k_diag_precond(const double* __restrict__ x, long nv, int nc, const int* __restrict__ n_of_coef,
                               double dt, double* __restrict__ y) {
  const long tot = 4 * nv * nc;
  for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < tot; g += (long)gridDim.x * blockDim.x) {
    const bool vel = g < 3 * nv * nc;
    const double n = (double)n_of_coef[g % nc];
    double sc;
    if (vel) {
      double b = 1.0 / fabs(1.0 - dt * n * n * n);
      b = fabs(b) < 1e3 ? b : 1.0;
      sc = fabs(b) > 1e-10 ? b : 1.0;
    } else {
      double e = (4 * n * n - 1) * (2 * n + 3) / (n + 1) / (2 * n * n + 2 * n - 1);
      e = n == 0 ? 1.0 : e / n;
      sc = fabs(e) > 1e-10 ? e : 1.0;
    }
    y[g] = sc * x[g];
  }
}

int precond_apply(void* ctx, const double* x, double* y) {
  ves3d_sv* sv = (ves3d_sv*)ctx;
  const int nc = ncoef_(sv->p);
  const long nv = sv->nves;
  if (sv->precond == VES3D_PRECOND_DIAG_SPECTRAL) {
    k_diag_precond<<<grid_1d(4 * nv * nc), 256, 0, sv->stream>>>(x, nv, nc, sv->tab->d.n_of_coef, sv->dt, y);
    VES3D_LAUNCHED();
    return VES3D_OK;
  }
  const int n = 4 * nc;
  dim3 grid((n + kPcRows - 1) / kPcRows, (unsigned)nv);
  k_block_gemv<<<grid, kPcRows, n * sizeof(double), sv->stream>>>(sv->pc_inv, x, nv, nc, y);
  VES3D_LAUNCHED();
  return VES3D_OK;
}

// Per-vesicle inverse of the isolated-vesicle Galerkin operator (the implicit operator
// with the self part of the single layer only): columns by applying that operator to
// unit vectors in FP64 (one column of every vesicle per application), LU with partial
// pivoting (cuSOLVER getrf) and solves against the identity (getrs) in FP64, stored in
// FP32 -- the preconditioner only steers the iteration; the tests on the true residual
// fix the accuracy of the solution.
// Streams and cuSOLVER handles of the preconditioner factorisation: one process-wide set
// per device, created on first use and kept until exit (creating 32 handles costs ~0.1 s,
// which every new operator context would otherwise pay); a mutex serialises their use.
struct SolverPool {
  std::mutex mu;
  bool ready = false;
  cudaStream_t st[kPcStreams] = {};
  cusolverDnHandle_t h[kPcStreams] = {};
};

SolverPool& solver_pool(int device) {
  static SolverPool* pools[64] = {};
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  SolverPool*& p = pools[(unsigned)device % 64];
  if (!p) p = new SolverPool();  // intentionally never freed: handles live until exit
  return *p;
}

int build_self_block_precond(ves3d_sv* sv) {
  NvtxRange nvtx("ves3d precond");
  int s;
  const int nc = ncoef_(sv->p), n = 4 * nc;
  const long nv = sv->nves, nn = (long)n * n;
  if (sv->pc_cap < nv * nn) {
    if (sv->pc_inv) cudaFree(sv->pc_inv);
    sv->pc_inv = nullptr;
    sv->pc_cap = 0;
    VES3D_CK(cudaMalloc((void**)&sv->pc_inv, sizeof(float) * nv * nn));
    sv->pc_cap = nv * nn;
  }
  if (!sv->pc_ev[0])
    for (auto& ev : sv->pc_ev) VES3D_CK(cudaEventCreate(&ev));
  SolverPool& pool = solver_pool(sv->device);
  std::lock_guard<std::mutex> pool_lock(pool.mu);
  if (!pool.ready) {
    for (int k = 0; k < kPcStreams; k++) {
      if (!pool.st[k]) VES3D_CK(cudaStreamCreateWithFlags(&pool.st[k], cudaStreamNonBlocking));
      if (!pool.h[k]) {
        if (cusolverDnCreate(&pool.h[k]) != CUSOLVER_STATUS_SUCCESS) {
          pool.h[k] = nullptr;
          set_error("cusolverDnCreate failed");
          return VES3D_ERR_CUDA;
        }
        if (cusolverDnSetStream(pool.h[k], pool.st[k]) != CUSOLVER_STATUS_SUCCESS) {
          set_error("cusolverDnSetStream failed");
          return VES3D_ERR_CUDA;
        }
      }
    }
    pool.ready = true;
  }
  cudaStream_t* pc_stream = pool.st;
  cusolverDnHandle_t* pc_solver = pool.h;
  double *A = nullptr, *B = nullptr;
  int *piv = nullptr, *info = nullptr;
  if ((s = dalloc(&A, nv * nn))) return s;
  if ((s = dalloc(&B, nv * nn)) || (s = dalloc(&piv, nv * (long)n)) || (s = dalloc(&info, nv))) {
    dfree(A); dfree(B); dfree(piv);
    return s;
  }
  VES3D_CK(cudaEventRecord(sv->pc_ev[0], sv->stream));
  // columns of the isolated-vesicle operator, kPcBatch per application: kPcBatch copies
  // of the suspension (geometry and self matrices shared), copy q carrying the unit
  // vector of column j0 + q of every vesicle; each self matrix is read once per batch
  {
    const int K = std::min(kPcBatch, n);
    const int ng = ngrid_(sv->p);
    OpSpace sp;
    sp.nv = (long)K * nv;
    const long Nv = sp.nv * ng, nshb = 4L * nc * sp.nv;
    double* bb = nullptr;
    const size_t need = (size_t)8 * 3 * Nv + 3 * (size_t)3 * nc * sp.nv + 18 * (size_t)Nv + 2 * (size_t)nshb;
    if (!s) s = dalloc(&bb, need);
    if (!s) {
      double* q = bb;
      for (int k = 0; k < 8; k++, q += 3 * Nv) sp.w[k] = q;
      sp.wc = q;
      q += 3L * nc * sp.nv;
      sp.fc = q;
      q += 3L * nc * sp.nv;
      sp.vc = q;
      q += 3L * nc * sp.nv;
      ImplicitWork bw;
      bw.f = q;
      bw.Sf = q + 3 * Nv;
      bw.h = q + 6 * Nv;
      bw.y = q + 7 * Nv;
      bw.g1 = q + 10 * Nv;
      bw.g2 = q + 14 * Nv;
      q += 18 * Nv;
      double* eb = q;
      double* yb = q + nshb;
      for (int j0 = 0; j0 < n && !s; j0 += K) {
        const int kq = std::min(K, n - j0);
        s = cuda_status(cudaMemsetAsync(eb, 0, nshb * sizeof(double), sv->stream), "memset", __FILE__, __LINE__);
        if (!s) {
          k_unit_columns_batch<<<grid_1d((long)kq * nv), 256, 0, sv->stream>>>(eb, nv, K, nc, j0, kq);
          s = cuda_status(cudaGetLastError(), "k_unit_columns_batch", __FILE__, __LINE__);
          if (!s) launch_counter()++;
        }
        if (!s) s = implicit_matvec_sh_self_batch(sv, sp, bw, eb, yb);
        if (!s) {
          k_store_columns_batch<<<grid_1d((long)kq * nv * n), 256, 0, sv->stream>>>(yb, nv, K, nc, j0, kq, A);
          s = cuda_status(cudaGetLastError(), "k_store_columns_batch", __FILE__, __LINE__);
          if (!s) launch_counter()++;
        }
      }
    }
    // the batch buffers are released after the stream's work (the factorisation follows)
    cudaStreamSynchronize(sv->stream);
    dfree(bb);
  }
  if (!s) {
    k_shift_null_mode<<<(unsigned)((nv + 127) / 128), 128, 0, sv->stream>>>(A, nv, nc);
    s = cuda_status(cudaGetLastError(), "k_shift_null_mode", __FILE__, __LINE__);
    if (!s) launch_counter()++;
  }
  if (!s) {
    k_identity_blocks<<<grid_1d(nv * nn), 256, 0, sv->stream>>>(B, nv, n);
    s = cuda_status(cudaGetLastError(), "k_identity_blocks", __FILE__, __LINE__);
    if (!s) launch_counter()++;
  }
  int lwork = 0;
  if (!s && cusolverDnDgetrf_bufferSize(pc_solver[0], n, n, A, n, &lwork) != CUSOLVER_STATUS_SUCCESS) {
    set_error("cusolverDnDgetrf_bufferSize failed");
    s = VES3D_ERR_CUDA;
  }
  lwork = std::max(lwork, 1);
  double* work = nullptr;
  if (!s) s = dalloc(&work, (size_t)lwork * kPcStreams);
  // dense LU + solve against the identity in FP64, vesicles spread over kPcStreams streams
  // (one factorisation of n ~ 10^3 is latency-bound and does not fill the GPU)
  if (!s) s = cuda_status(cudaEventRecord(sv->pc_ev[1], sv->stream), "event", __FILE__, __LINE__);
  for (int k = 0; k < kPcStreams && !s; k++)
    s = cuda_status(cudaStreamWaitEvent(pc_stream[k], sv->pc_ev[1], 0), "wait", __FILE__, __LINE__);
  for (long v = 0; v < nv && !s; v++) {
    const int k = (int)(v % kPcStreams);
    if (cusolverDnDgetrf(pc_solver[k], n, n, A + v * nn, n, work + (long)k * lwork, piv + v * n, info + v) !=
            CUSOLVER_STATUS_SUCCESS ||
        cusolverDnDgetrs(pc_solver[k], CUBLAS_OP_N, n, n, A + v * nn, n, piv + v * n, B + v * nn, n, info + v) !=
            CUSOLVER_STATUS_SUCCESS) {
      set_error("cuSOLVER getrf/getrs failed for vesicle %ld", v);
      s = VES3D_ERR_CUDA;
    }
  }
  // join (also after an error, so nothing is left running on the side streams)
  for (int k = 0; k < kPcStreams; k++) {
    cudaEventRecord(sv->pc_ev[3 + k], pc_stream[k]);
    cudaStreamWaitEvent(sv->stream, sv->pc_ev[3 + k], 0);
  }
  if (!s) {
    k_to_f32<<<grid_1d(nv * nn), 256, 0, sv->stream>>>(B, nv * nn, sv->pc_inv);
    s = cuda_status(cudaGetLastError(), "k_to_f32", __FILE__, __LINE__);
    if (!s) launch_counter()++;
  }
  std::vector<int> hinfo(nv, 0);
  if (!s)
    s = cuda_status(cudaMemcpyAsync(hinfo.data(), info, nv * sizeof(int), cudaMemcpyDeviceToHost, sv->stream), "copy",
                    __FILE__, __LINE__);
  if (!s) s = cuda_status(cudaEventRecord(sv->pc_ev[2], sv->stream), "event", __FILE__, __LINE__);
  cudaStreamSynchronize(sv->stream);
  for (long v = 0; v < nv && !s; v++)
    if (hinfo[v] != 0) {
      set_error("self-block preconditioner: vesicle %ld has a singular isolated operator (info %d)", v, hinfo[v]);
      s = VES3D_ERR_NUMERIC;
    }
  if (!s) {
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, sv->pc_ev[0], sv->pc_ev[1]);
    cudaEventElapsedTime(&b, sv->pc_ev[1], sv->pc_ev[2]);
    sv->pc_ms[0] = a + b;
    sv->pc_ms[1] = a;
    sv->pc_ms[2] = b;
    sv->pc_valid = true;
    sv->pc_age = 0;
    sv->pc_nves = nv;
  }
  dfree(A);
  dfree(B);
  dfree(work);
  dfree(piv);
  dfree(info);
  return s;
}

int ensure_precond(ves3d_sv* sv) {
  if (sv->precond == VES3D_PRECOND_NONE || sv->pc_valid) return VES3D_OK;
  if (sv->precond == VES3D_PRECOND_DIAG_SPECTRAL) {
    sv->pc_ms[0] = sv->pc_ms[1] = sv->pc_ms[2] = 0;
    sv->pc_valid = true;
    sv->pc_age = 0;
    sv->pc_nves = sv->nves;
    return VES3D_OK;
  }
  return build_self_block_precond(sv);
}

MatVecFn precond_fn(ves3d_sv* sv) { return sv->precond == VES3D_PRECOND_NONE ? nullptr : precond_apply; }

// The operators of one implicit system: the inner-solve operator in the context's
// precision, the same operator with the FP64 far field (outer residuals) and the right
// preconditioner (may be null), all on one context and stream.
struct SolveOps {
  MatVecFn mixed = nullptr;
  MatVecFn fp64 = nullptr;
  MatVecFn P = nullptr;
  void* ctx = nullptr;
  cudaStream_t st = nullptr;
};

// VES3D_SOLVER_TRACE=1 in the environment: one line per refinement step on stderr
bool solver_trace() {
  static const bool on = [] {
    const char* e = std::getenv("VES3D_SOLVER_TRACE");
    return e && *e && *e != '0';
  }();
  return on;
}

// Mixed-precision iterative refinement: outer residuals r = b - A x with the FP64
// operator; inner BiCGStab with the mixed operator on A d = r to a relative tolerance of
// 1e-2 (at most 150 iterations per correction); x += d. A correction that does not reduce
// the FP64 residual is undone (the residual before it is kept, so undoing costs no
// operator application) and retried once with the mixed operator to 1e-3; a second
// failure in a row switches to FP64 inner solves of at most 50 iterations each.
// *tol in: target relative residual; out: achieved. *max_iter in: bound on inner
// iterations in total; out: inner iterations used; outer refinements (FP64 matvecs) go to
// *outer_out.
int mixed_refinement(const SolveOps& ops, double* x, const double* b, long n, double* tol, int* max_iter, int* code,
                     int* outer_out, int* inner_out) {
  int s;
  const double target = *tol;
  const int budget = *max_iter;
  cudaStream_t st = ops.st;
  double *r = nullptr, *rp = nullptr, *d = nullptr, *ax = nullptr, *ws = nullptr;
  if ((s = dalloc(&r, n))) return s;
  if ((s = dalloc(&rp, n)) || (s = dalloc(&d, n)) || (s = dalloc(&ax, n)) ||
      (s = dalloc(&ws, bicgstab_workspace_doubles(n)))) {
    dfree(r); dfree(rp); dfree(d); dfree(ax);
    return s;
  }
  double nb2 = 0;
  s = dot_f64(b, b, n, bicgstab_dot_scratch(ws, n), &nb2, st);
  const double normb = nb2 > 0 ? std::sqrt(nb2) : 1.0;
  int used = 0, outer = 0, fails = 0;
  double relres = 1e300;
  *code = 101;
  while (!s && outer < 30) {
    NvtxRange nvtx("ves3d refine");
    // FP64 residual
    if ((s = ops.fp64(ops.ctx, x, ax))) break;
    if ((s = lincomb_f64(n, 1.0, b, -1.0, ax, 0.0, nullptr, r, st))) break;
    double rr = 0;
    if ((s = dot_f64(r, r, n, bicgstab_dot_scratch(ws, n), &rr, st))) break;
    const double cur = std::sqrt(rr) / normb;
    outer++;
    if (solver_trace())
      std::fprintf(stderr, "[ves3d refine] outer %d FP64 relres %.3e (inner iterations so far %d)\n", outer, cur,
                   used);
    if (cur != cur) {  // non-finite residual (BiCGSReturn RelresIsNan)
      relres = cur;
      *code = 104;
      break;
    }
    if (cur > relres) {
      // the last correction made things worse: undo it and restore the residual before it
      if ((s = lincomb_f64(n, 1.0, x, -1.0, d, 0.0, nullptr, x, st))) break;
      VES3D_CK(cudaMemcpyAsync(r, rp, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
      fails++;
    } else {
      relres = cur;
      fails = 0;
      if (relres < target) {
        *code = 100;
        break;
      }
      VES3D_CK(cudaMemcpyAsync(rp, r, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    if (used >= budget) break;
    // inner solve for the correction, from zero, to 1e-2 of the current residual (or the
    // target): the FP32 far field is accurate to ~1e-5 for dipole-dominated densities, so
    // each correction only has to make a modest, reliable reduction
    VES3D_CK(cudaMemsetAsync(d, 0, n * sizeof(double), st));
    const bool fp64_inner = fails >= 2;
    double itol = std::max(fails == 1 ? 1e-3 : 1e-2, 0.5 * target / relres);
    int imax = std::min(budget - used, fp64_inner ? 50 : 150), icode = 0;
    if ((s = bicgstab_run(fp64_inner ? ops.fp64 : ops.mixed, ops.ctx, d, r, n, &itol, &imax, &icode, ws, st, ops.P,
                          ops.ctx)))
      break;
    if (solver_trace())
      std::fprintf(stderr, "[ves3d refine]   inner (%s) %d iterations, code %d, relres %.3e\n",
                   fp64_inner ? "FP64" : "mixed", imax, icode, itol);
    used += imax;
    if ((s = lincomb_f64(n, 1.0, x, 1.0, d, 0.0, nullptr, x, st))) break;
  }
  *tol = relres;
  *max_iter = used;
  if (outer_out) *outer_out = outer;
  if (inner_out) *inner_out = used;
  dfree(r);
  dfree(rp);
  dfree(d);
  dfree(ax);
  dfree(ws);
  return s;
}

int mixed_refinement(ves3d_sv* sv, double* x, const double* b, long n, double* tol, int* max_iter, int* code) {
  SolveOps ops;
  ops.mixed = implicit_matvec_cb;
  ops.fp64 = implicit_matvec_fp64_cb;
  ops.P = precond_fn(sv);
  ops.ctx = sv;
  ops.st = sv->stream;
  return mixed_refinement(ops, x, b, n, tol, max_iter, code, &sv->ir_outer, &sv->ir_inner);
}

}  // namespace

extern "C" {

int ves3d_sv_solver_stats(ves3d_sv* sv, int* outer, int* inner) {
  VES3D_ARG(sv && outer && inner, "null argument");
  *outer = sv->ir_outer;
  *inner = sv->ir_inner;
  return VES3D_OK;
}

int ves3d_sv_integrals(ves3d_sv* sv, double* area, double* volume, double* centers, int is_device) {
  int s = check_sv(sv);
  if (s) return s;
  if (!sv->have_src) {
    set_error("no surfaces set");
    return VES3D_ERR_STATE;
  }
  const long nv = sv->nves;
  double* d = nullptr;
  if ((s = dalloc(&d, 5 * nv))) return s;
  s = launch_integrals(sv->X, sv->Xp, sv->Xt, sv->tab->d.smooth_w0, nv, sv->p, d, sv->stream);
  std::vector<double> h(5 * nv);
  if (!s)
    s = cuda_status(cudaMemcpyAsync(h.data(), d, 5 * nv * sizeof(double), cudaMemcpyDeviceToHost, sv->stream),
                    "copy", __FILE__, __LINE__);
  if (!s) s = cuda_status(cudaStreamSynchronize(sv->stream), "sync", __FILE__, __LINE__);
  dfree(d);
  if (s) return s;
  std::vector<double> a(nv), vo(nv), c(3 * nv);
  for (long v = 0; v < nv; v++) {
    a[v] = h[5 * v];
    vo[v] = h[5 * v + 1];
    for (int k = 0; k < 3; k++) c[3 * v + k] = h[5 * v + 2 + k];
  }
  const cudaMemcpyKind kind = is_device ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost;
  if (area) VES3D_CK(cudaMemcpy(area, a.data(), nv * sizeof(double), kind));
  if (volume) VES3D_CK(cudaMemcpy(volume, vo.data(), nv * sizeof(double), kind));
  if (centers) VES3D_CK(cudaMemcpy(centers, c.data(), 3 * nv * sizeof(double), kind));
  return VES3D_OK;
}

int ves3d_sv_set_implicit_params(ves3d_sv* sv, double dt, double kappa, double shear_rate) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(dt > 0 && kappa >= 0, "dt must be > 0 and kappa >= 0");
  if (dt != sv->dt || kappa != sv->kappa) sv->pc_valid = false;
  mark_implicit(sv);
  sv->dt = dt;
  sv->kappa = kappa;
  sv->shear = shear_rate;
  return VES3D_OK;
}

int ves3d_sv_set_surface_filter(ves3d_sv* sv, int filter_freq) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(filter_freq >= -1, "filter frequency: 0 (off), -1 (2p/3) or the highest degree kept");
  const int f = filter_freq == -1 ? 2 * sv->p / 3 : filter_freq;
  if (f == sv->filter_freq) return VES3D_OK;
  if (f) {
    const int nc = ncoef_(sv->p);
    std::vector<double> c(nc);
    if ((s = ves3d_sht_filter_coeffs(sv->p, f, 0.0, c.data()))) return s;
    dfree(sv->filt);
    sv->filt = nullptr;
    if ((s = dupload(&sv->filt, c, sv->stream))) return s;
    VES3D_CK(cudaStreamSynchronize(sv->stream));
  }
  sv->filter_freq = f;
  sv->geo_valid = false;
  sv->pc_valid = false;
  return VES3D_OK;
}

int ves3d_sv_set_gravity(ves3d_sv* sv, double excess_density, double gx, double gy, double gz) {
  int s = check_sv(sv);
  if (s) return s;
  if (excess_density != sv->drho || gx != sv->grav[0] || gy != sv->grav[1] || gz != sv->grav[2])
    sv->pc_valid = false;
  sv->drho = excess_density;
  sv->grav[0] = gx;
  sv->grav[1] = gy;
  sv->grav[2] = gz;
  return VES3D_OK;
}

int ves3d_sv_set_viscosity_contrast(ves3d_sv* sv, const double* lambda, long n) {
  int s = check_sv(sv);
  if (s) return s;
  if (!lambda || n == 0) {
    sv->lam.clear();
    sv->contrast = false;
    sv->pc_valid = false;
    return VES3D_OK;
  }
  VES3D_ARG(n == 1 || (sv->have_src && n == sv->nves), "n must be 1 or the number of vesicles");
  for (long i = 0; i < n; i++) VES3D_ARG(std::isfinite(lambda[i]) && lambda[i] > 0.0, "contrast must be positive");
  sv->lam.assign(lambda, lambda + n);
  bool any = false;
  for (double l : sv->lam) any |= std::fabs(l - 1.0) > 1e-12;  // has_contrast, VesicleProps.cc:45-49
  sv->contrast = any;
  sv->contrast_nves = -1;
  sv->pc_valid = false;  // the self-block preconditioner is built from the operator
  return VES3D_OK;
}

int ves3d_sv_set_precond(ves3d_sv* sv, int scheme) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(scheme >= VES3D_PRECOND_NONE && scheme <= VES3D_PRECOND_SELF_BLOCK, "unknown preconditioner");
  if (scheme != sv->precond) sv->pc_valid = false;
  sv->precond = scheme;
  return VES3D_OK;
}

int ves3d_sv_set_precond_refresh(ves3d_sv* sv, int every) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(every >= 1, "refresh interval must be >= 1");
  sv->pc_refresh = every;
  return VES3D_OK;
}

int ves3d_sv_precond_info(ves3d_sv* sv, double* ms, size_t* bytes, int* age) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(ms && bytes, "null argument");
  if (age) *age = sv->pc_valid ? sv->pc_age : -1;
  for (int k = 0; k < 3; k++) ms[k] = sv->pc_ms[k];
  *bytes = sv->precond == VES3D_PRECOND_SELF_BLOCK ? (size_t)sv->pc_cap * sizeof(float) : 0;
  return VES3D_OK;
}

int ves3d_sv_surface_op(ves3d_sv* sv, int op, const double* in, double* out, int is_device) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(out != nullptr, "out is null");
  if (!sv->have_src) {
    set_error("no surfaces set");
    return VES3D_ERR_STATE;
  }
  if ((s = ensure_geometry(sv))) return s;
  const long N = sv->npts();
  const int ng = ngrid_(sv->p);
  size_t nin = 0, nout = 0;
  switch (op) {
    case VES3D_OP_GEOMETRY: nout = (size_t)sv->nves * kGeoComps * ng; break;
    case VES3D_OP_GRAD: nin = N; nout = 3 * N; break;
    case VES3D_OP_DIV: nin = 3 * N; nout = N; break;
    case VES3D_OP_LIN_MEANCURV: nin = 3 * N; nout = N; break;
    case VES3D_OP_LIN_BENDING: nin = 3 * N; nout = 3 * N; break;
    case VES3D_OP_BENDING: nout = 3 * N; break;
    case VES3D_OP_TENSION: nin = N; nout = 3 * N; break;
    case VES3D_OP_IMPLICIT_MATVEC: nin = 4 * N; nout = 4 * N; break;
    case VES3D_OP_IMPLICIT_RHS: nout = 4 * N; break;
    case VES3D_OP_GRAVITY: nin = 3 * N; nout = 3 * N; break;
    default: VES3D_ARG(false, "unknown surface op");
  }
  VES3D_ARG(nin == 0 || in != nullptr, "in is null");
  double *din = nullptr, *dout = nullptr;
  int st = VES3D_OK;
  if (nin && (st = dalloc(&din, nin))) return st;
  if ((st = dalloc(&dout, nout))) {
    dfree(din);
    return st;
  }
  if (nin) st = copy_in(din, in, nin, is_device, sv->stream);
  ImplicitWork iw;
  if (!st) st = implicit_work(sv, iw);
  if (!st) {
    switch (op) {
      case VES3D_OP_GEOMETRY:
        st = cuda_status(cudaMemcpyAsync(dout, sv->geo, nout * sizeof(double), cudaMemcpyDeviceToDevice, sv->stream),
                         "copy", __FILE__, __LINE__);
        break;
      case VES3D_OP_GRAD: st = op_grad(sv, din, dout); break;
      case VES3D_OP_DIV: st = op_div(sv, din, dout, 1.0); break;
      case VES3D_OP_LIN_MEANCURV: st = op_linH(sv, din, dout); break;
      case VES3D_OP_LIN_BENDING:
        st = op_linH(sv, din, iw.h);
        if (!st) st = op_bend_of(sv, iw.h, nullptr, dout);
        break;
      case VES3D_OP_BENDING:
        for (long v = 0; v < sv->nves && !st; v++)
          st = cuda_status(cudaMemcpyAsync(iw.h + v * ng, sv->geo + (v * kGeoComps + 13) * (long)ng,
                                           ng * sizeof(double), cudaMemcpyDeviceToDevice, sv->stream),
                           "copy", __FILE__, __LINE__);
        if (!st) st = op_bend_of(sv, iw.h, nullptr, dout);
        break;
      case VES3D_OP_TENSION: st = op_tension(sv, din, nullptr, dout); break;
      case VES3D_OP_IMPLICIT_MATVEC: st = implicit_matvec(sv, din, dout); break;
      case VES3D_OP_IMPLICIT_RHS: st = implicit_rhs(sv, dout); break;
      case VES3D_OP_GRAVITY:
        st = launch_gravity_combine(din, sv->geo, sv->nves, ng, sv->drho, sv->grav, nullptr, dout, sv->stream);
        break;
    }
  }
  if (!st) st = copy_out(out, dout, nout, is_device, sv->stream);
  cudaStreamSynchronize(sv->stream);
  dfree(din);
  dfree(dout);
  return st;
}

int ves3d_sv_implicit_solve(ves3d_sv* sv, const double* x0, double* x, double* tol, int* max_iter, int* code,
                            int is_device) {
  NvtxRange nvtx("ves3d implicit_solve");
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(x && tol && max_iter && code, "null argument");
  if (!sv->have_src) {
    set_error("no surfaces set");
    return VES3D_ERR_STATE;
  }
  if ((s = ensure_geometry(sv))) return s;
  ImplicitWork iw;
  if ((s = implicit_work(sv, iw))) return s;
  const long ng4 = 4 * sv->npts(), nsh = sh_unknowns(sv);
  double *dc = nullptr, *db = nullptr, *dg = nullptr;
  if ((s = dalloc(&dc, nsh))) return s;
  if ((s = dalloc(&db, nsh))) {
    dfree(dc);
    return s;
  }
  if ((s = dalloc(&dg, ng4))) {
    dfree(dc);
    dfree(db);
    return s;
  }
  if (x0) {
    s = copy_in(dg, x0, ng4, is_device, sv->stream);
    if (!s) s = grid_to_coef(sv, dg, dc);
  } else {
    s = cuda_status(cudaMemsetAsync(dc, 0, nsh * sizeof(double), sv->stream), "memset", __FILE__, __LINE__);
  }
  // right-hand side always with the FP64 far field
  sv->far_force_fp64 = 1;
  if (!s) s = implicit_rhs(sv, dg);
  sv->far_force_fp64 = 0;
  if (!s) s = grid_to_coef(sv, dg, db);
  if (!s) s = ensure_precond(sv);
  if (!s) {
    if (sv->prec == VES3D_PREC_FP64)
      s = bicgstab_run(implicit_matvec_cb, sv, dc, db, nsh, tol, max_iter, code, sv->bws, sv->stream,
                       precond_fn(sv), sv);
    else
      s = mixed_refinement(sv, dc, db, nsh, tol, max_iter, code);
  }
  if (!s) s = coef_to_grid(sv, dc, dg);
  if (!s) s = copy_out(x, dg, ng4, is_device, sv->stream);
  cudaStreamSynchronize(sv->stream);
  dfree(dc);
  dfree(db);
  dfree(dg);
  return s;
}

// ---- initial guesses of the implicit solve ------------------------------------------
// Per-vesicle features and targets of the learned guess, and the residual-minimising
// combination of candidate guesses (the true residual of the solver's own system decides
// how much of each candidate is used; a useless candidate gets weight ~0).

}  // extern "C"

namespace {

// feat[v][j] = coef[v][j] (3 nc per vesicle) with every degree-0 coefficient set to 0
__global__ void k_pack_features(const double* __restrict__ coef, long n, int nc, float* __restrict__ feat) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    feat[i] = (i % nc) == 0 ? 0.f : (float)coef[i];
}

// tgt[v] = [cu[v] (3 nc); cs[v] (nc)]  <->  (cu, cs)
__global__ void k_pack_targets(const double* __restrict__ cu, const double* __restrict__ cs, long nv, int nc,
                               float* __restrict__ tgt, double* __restrict__ ou, double* __restrict__ os,
                               const float* __restrict__ in) {
  const long n = nv * 4 * nc;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const long v = i / (4 * nc);
    const int j = (int)(i - v * 4 * nc);
    if (in) {
      const double x = (double)in[i];
      if (j < 3 * nc) ou[v * 3 * nc + j] = x;
      else os[v * nc + j - 3 * nc] = x;
    } else {
      tgt[i] = (float)(j < 3 * nc ? cu[v * 3 * nc + j] : cs[v * nc + j - 3 * nc]);
    }
  }
}

// Solve the n x n normal equations G a = h (n <= 8) by Gaussian elimination with partial
// pivoting, after Jacobi scaling (unit diagonal, so candidates of very different size are
// treated alike); a ridge of 1e-13 keeps dependent candidates from blowing the weights up.
void small_solve(int n, std::vector<double> G, std::vector<double> h, std::vector<double>& a) {
  std::vector<double> d(n);
  for (int i = 0; i < n; i++) d[i] = G[i * n + i] > 0 ? 1.0 / std::sqrt(G[i * n + i]) : 0.0;
  for (int i = 0; i < n; i++) {
    h[i] *= d[i];
    for (int j = 0; j < n; j++) G[i * n + j] *= d[i] * d[j];
    G[i * n + i] += 1e-13;
  }
  for (int k = 0; k < n; k++) {
    int piv = k;
    for (int i = k + 1; i < n; i++)
      if (std::fabs(G[i * n + k]) > std::fabs(G[piv * n + k])) piv = i;
    if (piv != k) {
      for (int j = 0; j < n; j++) std::swap(G[k * n + j], G[piv * n + j]);
      std::swap(h[k], h[piv]);
    }
    const double d = G[k * n + k];
    if (d == 0) continue;
    for (int i = k + 1; i < n; i++) {
      const double f = G[i * n + k] / d;
      for (int j = k; j < n; j++) G[i * n + j] -= f * G[k * n + j];
      h[i] -= f * h[k];
    }
  }
  a.assign(n, 0.0);
  for (int k = n - 1; k >= 0; k--) {
    double t = h[k];
    for (int j = k + 1; j < n; j++) t -= G[k * n + j] * a[j];
    a[k] = G[k * n + k] != 0 ? t / G[k * n + k] : 0.0;
  }
  for (int i = 0; i < n; i++) a[i] *= d[i];
}

}  // namespace

extern "C" {

int ves3d_sv_guess_features(ves3d_sv* sv, float* feat, int is_device) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(feat != nullptr, "feat is null");
  if (!sv->have_src) {
    set_error("no surfaces set");
    return VES3D_ERR_STATE;
  }
  const long nv = sv->nves, nc = ncoef_(sv->p), n = nv * 3 * nc;
  double* c = nullptr;
  float* f = nullptr;
  if ((s = dalloc(&c, n))) return s;
  if ((s = dalloc(&f, n))) {
    dfree(c);
    return s;
  }
  s = grid2shc_p(sv, sv->X, 3 * nv, c);
  if (!s) {
    k_pack_features<<<grid_1d(n), 256, 0, sv->stream>>>(c, n, (int)nc, f);
    s = cuda_status(cudaGetLastError(), "k_pack_features", __FILE__, __LINE__);
    if (!s) launch_counter()++;
  }
  if (!s)
    s = cuda_status(cudaMemcpyAsync(feat, f, n * sizeof(float),
                                    is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, sv->stream),
                    "copy", __FILE__, __LINE__);
  cudaStreamSynchronize(sv->stream);
  dfree(c);
  dfree(f);
  return s;
}

int ves3d_sv_guess_targets(ves3d_sv* sv, const double* x, float* tgt, int is_device) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(x && tgt, "null argument");
  if (!sv->have_src) {
    set_error("no surfaces set");
    return VES3D_ERR_STATE;
  }
  const long nv = sv->nves, nc = ncoef_(sv->p), N = sv->npts();
  const int ng = ngrid_(sv->p);
  double *g = nullptr, *ui = nullptr, *cu = nullptr;
  float* t = nullptr;
  if ((s = dalloc(&g, 4 * N))) return s;
  if ((s = dalloc(&ui, 3 * N)) || (s = dalloc(&cu, 4 * nv * nc)) || (s = dalloc(&t, 4 * nv * nc))) {
    dfree(g); dfree(ui); dfree(cu);
    return s;
  }
  s = copy_in(g, x, 4 * N, is_device, sv->stream);
  if (!s) s = launch_shear(sv->X, nv, ng, sv->shear, ui, sv->stream);
  if (!s) s = lincomb_f64(3 * N, 1.0, g, -1.0, ui, 0.0, nullptr, g, sv->stream);
  if (!s) s = grid2shc_p(sv, g, 3 * nv, cu);
  if (!s) s = grid2shc_p(sv, g + 3 * N, nv, cu + 3 * nv * nc);
  if (!s) {
    k_pack_targets<<<grid_1d(4 * nv * nc), 256, 0, sv->stream>>>(cu, cu + 3 * nv * nc, nv, (int)nc, t, nullptr,
                                                                  nullptr, nullptr);
    s = cuda_status(cudaGetLastError(), "k_pack_targets", __FILE__, __LINE__);
    if (!s) launch_counter()++;
  }
  if (!s)
    s = cuda_status(cudaMemcpyAsync(tgt, t, 4 * nv * nc * sizeof(float),
                                    is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, sv->stream),
                    "copy", __FILE__, __LINE__);
  cudaStreamSynchronize(sv->stream);
  dfree(g);
  dfree(ui);
  dfree(cu);
  dfree(t);
  return s;
}

int ves3d_sv_guess_from_targets(ves3d_sv* sv, const float* tgt, double* x0, int is_device) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(x0 && tgt, "null argument");
  if (!sv->have_src) {
    set_error("no surfaces set");
    return VES3D_ERR_STATE;
  }
  const long nv = sv->nves, nc = ncoef_(sv->p), N = sv->npts();
  const int ng = ngrid_(sv->p);
  double *g = nullptr, *ui = nullptr, *cu = nullptr;
  float* t = nullptr;
  if ((s = dalloc(&g, 4 * N))) return s;
  if ((s = dalloc(&ui, 3 * N)) || (s = dalloc(&cu, 4 * nv * nc)) || (s = dalloc(&t, 4 * nv * nc))) {
    dfree(g); dfree(ui); dfree(cu);
    return s;
  }
  s = cuda_status(cudaMemcpyAsync(t, tgt, 4 * nv * nc * sizeof(float),
                                  is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, sv->stream),
                  "copy", __FILE__, __LINE__);
  if (!s) {
    k_pack_targets<<<grid_1d(4 * nv * nc), 256, 0, sv->stream>>>(nullptr, nullptr, nv, (int)nc, nullptr, cu,
                                                                  cu + 3 * nv * nc, t);
    s = cuda_status(cudaGetLastError(), "k_pack_targets", __FILE__, __LINE__);
    if (!s) launch_counter()++;
  }
  if (!s) s = coef_to_grid(sv, cu, g);
  if (!s) s = launch_shear(sv->X, nv, ng, sv->shear, ui, sv->stream);
  if (!s) s = lincomb_f64(3 * N, 1.0, g, 1.0, ui, 0.0, nullptr, g, sv->stream);
  if (!s) s = copy_out(x0, g, 4 * N, is_device, sv->stream);
  cudaStreamSynchronize(sv->stream);
  dfree(g);
  dfree(ui);
  dfree(cu);
  dfree(t);
  return s;
}

int ves3d_sv_implicit_combine(ves3d_sv* sv, int n_cand, const double* const* cand, double* x0, double* weights,
                              double* relres, int is_device) {
  int s = check_sv(sv);
  if (s) return s;
  VES3D_ARG(n_cand >= 1 && n_cand <= 8, "n_cand must be in [1, 8]");
  VES3D_ARG(cand && x0 && weights && relres, "null argument");
  for (int i = 0; i < n_cand; i++) VES3D_ARG(cand[i] != nullptr, "null candidate");
  if (!sv->have_src) {
    set_error("no surfaces set");
    return VES3D_ERR_STATE;
  }
  if ((s = ensure_geometry(sv))) return s;
  ImplicitWork iw;
  if ((s = implicit_work(sv, iw))) return s;
  const long ng4 = 4 * sv->npts(), nsh = sh_unknowns(sv);
  double *b = nullptr, *C = nullptr, *Y = nullptr, *dg = nullptr, *r = nullptr, *scr = nullptr;
  if ((s = dalloc(&b, nsh))) return s;
  if ((s = dalloc(&C, nsh * n_cand)) || (s = dalloc(&Y, nsh * n_cand)) || (s = dalloc(&dg, ng4)) ||
      (s = dalloc(&r, nsh)) || (s = dalloc(&scr, 1024))) {
    dfree(b); dfree(C); dfree(Y); dfree(dg); dfree(r);
    return s;
  }
  // right-hand side and the candidates' images under the FP64 operator
  sv->far_force_fp64 = 1;
  s = implicit_rhs(sv, dg);
  if (!s) s = grid_to_coef(sv, dg, b);
  for (int i = 0; i < n_cand && !s; i++) {
    s = copy_in(dg, cand[i], ng4, is_device, sv->stream);
    if (!s) s = grid_to_coef(sv, dg, C + i * nsh);
    if (!s) s = implicit_matvec_sh(sv, C + i * nsh, Y + i * nsh);
  }
  sv->far_force_fp64 = 0;
  std::vector<double> G(n_cand * n_cand, 0.0), h(n_cand, 0.0), a;
  std::vector<char> ok(n_cand, 1);
  double bb = 0;
  if (!s) s = dot_f64(b, b, nsh, scr, &bb, sv->stream);
  const double nb = bb > 0 ? std::sqrt(bb) : 1.0;
  for (int i = 0; i < n_cand && !s; i++) {
    // residual of the candidate as given
    s = lincomb_f64(nsh, 1.0, b, -1.0, Y + i * nsh, 0.0, nullptr, r, sv->stream);
    double rr = 0;
    if (!s) s = dot_f64(r, r, nsh, scr, &rr, sv->stream);
    relres[i] = std::sqrt(rr) / nb;
    if (!s) s = dot_f64(Y + i * nsh, b, nsh, scr, &h[i], sv->stream);
    for (int j = 0; j <= i && !s; j++) {
      s = dot_f64(Y + i * nsh, Y + j * nsh, nsh, scr, &G[i * n_cand + j], sv->stream);
      G[j * n_cand + i] = G[i * n_cand + j];
    }
    if (!std::isfinite(G[i * n_cand + i]) || !std::isfinite(h[i])) ok[i] = 0;
  }
  if (!s) {
    // drop non-finite candidates, solve the normal equations of the rest
    std::vector<int> idx;
    for (int i = 0; i < n_cand; i++)
      if (ok[i] && G[i * n_cand + i] > 0) idx.push_back(i);
    const int m = (int)idx.size();
    std::vector<double> Gm(m * m), hm(m), am;
    for (int i = 0; i < m; i++) {
      hm[i] = h[idx[i]];
      for (int j = 0; j < m; j++) Gm[i * m + j] = G[idx[i] * n_cand + idx[j]];
    }
    if (m) small_solve(m, Gm, hm, am);
    for (int i = 0; i < n_cand; i++) weights[i] = 0.0;
    for (int i = 0; i < m; i++) weights[idx[i]] = am[i];
    // combined coefficients and their true residual
    s = cuda_status(cudaMemsetAsync(dg, 0, nsh * sizeof(double), sv->stream), "memset", __FILE__, __LINE__);
    if (!s) s = copy_in(r, b, nsh, 1, sv->stream);
    for (int i = 0; i < m && !s; i++) {
      s = lincomb_f64(nsh, 1.0, dg, am[i], C + idx[i] * nsh, 0.0, nullptr, dg, sv->stream);
      if (!s) s = lincomb_f64(nsh, 1.0, r, -am[i], Y + idx[i] * nsh, 0.0, nullptr, r, sv->stream);
    }
    double rr = 0;
    if (!s) s = dot_f64(r, r, nsh, scr, &rr, sv->stream);
    relres[n_cand] = std::sqrt(rr) / nb;
    if (!s) {
      // dg holds coefficients; map to the grid through b's storage
      s = copy_in(b, dg, nsh, 1, sv->stream);
      if (!s) s = coef_to_grid(sv, b, dg);
      if (!s) s = copy_out(x0, dg, ng4, is_device, sv->stream);
    }
  }
  cudaStreamSynchronize(sv->stream);
  dfree(b);
  dfree(C);
  dfree(Y);
  dfree(dg);
  dfree(r);
  dfree(scr);
  return s;
}

}  // extern "C"

// ======================================================================================
// Polydisperse suspensions: vesicles of different SH orders in one evaluation
// ======================================================================================
struct ves3d_svp {
  int prec = 0, device = 0;
  bool far_dl_f32 = false;  // the mixed form's far double layer in FP32 pairs (opt-in, VES3D_FAR_DL_F32=1)
  cudaStream_t stream = nullptr;
  std::vector<ves3d_sv*> grp;          // one operator per run of equal order
  std::vector<int> gp;                 // order of each run
  std::vector<long> gnv, gpt0;         // vesicles and first point of each run
  long nves = 0, N = 0;
  int max_nt = 0;
  double *pos = nullptr, *den = nullptr, *vself = nullptr, *V = nullptr, *Vfar = nullptr, *part = nullptr;
  long* off = nullptr;
  long capN = 0, capV = 0;
  bool have_den = false;
  // double layer: a density set by ves3d_svp_set_density_dl (in the groups' G buffers), or
  // the implicit step's (1 - lambda) u under a viscosity contrast; unit normals, weighted
  // densities and far partials over all points
  bool have_dl = false;
  double *nrm = nullptr, *dden = nullptr, *part_dl = nullptr;
  std::vector<double> lam;  // viscosity contrast: one value, or one per vesicle
  bool contrast = false;
  cudaEvent_t ev[4] = {};
  float ms[4] = {0, 0, 0, 0};
  cudaGraph_t graph = nullptr;  // captured evaluation (self parts of every group + far field)
  cudaGraphExec_t graph_exec = nullptr;
  // implicit step: parameters pushed to every order group before a solve
  double dt = 0.01, kappa = 0.05, shear = 1.0, drho = 0.0, grav[3] = {0.0, 0.0, -1.0};
  int precond = 0, pc_refresh = 1, filter_freq = 0;
  int far_force_fp64 = 0, ir_outer = 0, ir_inner = 0;
  std::vector<long> coff;  // first SH unknown of each group's [u; sigma] coefficients
  double* sws = nullptr;   // solve workspace: BiCGStab, coefficients, right-hand side, grid
  long sws_cap = 0;
  // right-hand side (coefficients) of the current surfaces and parameters, kept between a
  // guess combination and the solve that follows it
  double* rhs = nullptr;
  long rhs_cap = 0;
  bool rhs_valid = false;
  void drop_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    graph_exec = nullptr;
    graph = nullptr;
  }
  void free_global() {
    double* ps[] = {pos, den, vself, V, Vfar, part, nrm, dden, part_dl};
    for (double* q : ps) dfree(q);
    dfree(off);
    pos = den = vself = V = Vfar = part = nrm = dden = part_dl = nullptr;
    off = nullptr;
    capN = capV = 0;
  }
  void free_groups() {
    for (ves3d_sv* g : grp) ves3d_sv_destroy(g);
    grp.clear();
    gp.clear();
  }
  ~ves3d_svp() {
    drop_graph();
    free_groups();
    free_global();
    dfree(sws);
    dfree(rhs);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
  }
};

extern "C" {

int ves3d_svp_create(int precision, int device, ves3d_svp** out) {
  VES3D_ARG(out != nullptr, "out is null");
  *out = nullptr;
  VES3D_ARG(precision == VES3D_PREC_FP64 || precision == VES3D_PREC_MIXED, "unknown precision");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_error("no CUDA device");
    return VES3D_ERR_NODEV;
  }
  if (device < 0) VES3D_CK(cudaGetDevice(&device));
  VES3D_ARG(device < ndev, "device index out of range");
  VES3D_CK(cudaSetDevice(device));
  std::unique_ptr<ves3d_svp> g(new ves3d_svp());
  g->prec = precision;
  g->device = device;
  {
    const char* d = getenv("VES3D_FAR_DL_F32");
    g->far_dl_f32 = d && d[0] == '1';
  }
  VES3D_CK(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
  for (auto& e : g->ev) VES3D_CK(cudaEventCreate(&e));
  *out = g.release();
  return VES3D_OK;
}

int ves3d_svp_destroy(ves3d_svp* g) {
  if (!g) return VES3D_OK;
  cudaSetDevice(g->device);
  cudaStreamSynchronize(g->stream);
  delete g;
  return VES3D_OK;
}

int ves3d_svp_set_src_coord(ves3d_svp* g, const double* S, const int* orders, long n_ves, int is_device) {
  if (g) {
    g->drop_graph();
    g->rhs_valid = false;
  }
  VES3D_ARG(g && S && orders && n_ves >= 1, "bad arguments");
  VES3D_CK(cudaSetDevice(g->device));
  // runs of equal order
  std::vector<int> rp;
  std::vector<long> rnv;
  for (long v = 0; v < n_ves; v++) {
    VES3D_ARG(orders[v] >= 2 && orders[v] <= 64, "order out of range");
    if (rp.empty() || rp.back() != orders[v]) {
      rp.push_back(orders[v]);
      rnv.push_back(0);
    }
    rnv.back()++;
  }
  if (rp != g->gp) {
    g->free_groups();
    for (int p : rp) {
      ves3d_sv* sv = nullptr;
      int s = ves3d_sv_create(p, 2 * p, g->prec, g->device, &sv);
      if (s) return s;
      ves3d_sv_set_stream(sv, g->stream);
      g->grp.push_back(sv);
    }
    g->gp = rp;
  }
  g->gnv = rnv;
  g->gpt0.assign(rp.size(), 0);
  std::vector<long> off(n_ves + 1, 0);
  long pt = 0, v = 0;
  int max_nt = 0;
  for (size_t r = 0; r < rp.size(); r++) {
    g->gpt0[r] = pt;
    const int ng = ngrid_(rp[r]);
    max_nt = std::max(max_nt, ng);
    for (long k = 0; k < rnv[r]; k++, v++) {
      off[v] = pt;
      pt += ng;
    }
  }
  off[n_ves] = pt;
  g->nves = n_ves;
  g->N = pt;
  g->max_nt = max_nt;
  if (g->capN < pt || g->capV < n_ves) {
    g->free_global();
    int s = 0;
    s |= dalloc(&g->pos, 3 * (size_t)pt);
    s |= dalloc(&g->den, 3 * (size_t)pt);
    s |= dalloc(&g->vself, 3 * (size_t)pt);
    s |= dalloc(&g->V, 3 * (size_t)pt);
    s |= dalloc(&g->Vfar, 3 * (size_t)pt);
    s |= dalloc(&g->part, (size_t)kFarMaxSegments * 3 * pt);
    s |= dalloc(&g->off, (size_t)n_ves + 1);
    if (s) {
      g->free_global();
      return s;
    }
    g->capN = pt;
    g->capV = n_ves;
  }
  VES3D_CK(cudaMemcpyAsync(g->off, off.data(), off.size() * sizeof(long), cudaMemcpyHostToDevice, g->stream));
  for (size_t r = 0; r < rp.size(); r++) {
    int s = ves3d_sv_set_src_coord(g->grp[r], S + 3 * g->gpt0[r], rnv[r], is_device);
    if (s) return s;
    VES3D_CK(cudaMemcpyAsync(g->pos + 3 * g->gpt0[r], g->grp[r]->pos, 3 * (size_t)g->grp[r]->npts() * sizeof(double),
                             cudaMemcpyDeviceToDevice, g->stream));
  }
  VES3D_CK(cudaStreamSynchronize(g->stream));
  g->have_den = false;
  g->have_dl = false;
  return VES3D_OK;
}

int ves3d_svp_set_density_sl(ves3d_svp* g, const double* f, int is_device) {
  VES3D_ARG(g && f, "null argument");
  VES3D_ARG(!g->grp.empty(), "set_src_coord first");
  for (size_t r = 0; r < g->grp.size(); r++) {
    int s = ves3d_sv_set_density_sl(g->grp[r], f + 3 * g->gpt0[r], is_device);
    if (s) return s;
  }
  g->have_den = true;
  return VES3D_OK;
}

// Double-layer buffers of the suspension (normals, weighted densities, far partials) and of
// every group (density, coefficients, self matrices).
static int svp_alloc_dl(ves3d_svp* g) {
  int s = 0;
  for (ves3d_sv* sv : g->grp)
    if ((s = alloc_dl(sv))) return s;
  if (g->nrm) return VES3D_OK;
  s |= dalloc(&g->nrm, 3 * (size_t)g->capN);
  s |= dalloc(&g->dden, 3 * (size_t)g->capN);
  s |= dalloc(&g->part_dl, (size_t)kFarMaxSegments * 3 * g->capN);
  if (s) {
    dfree(g->nrm);
    dfree(g->dden);
    dfree(g->part_dl);
    g->nrm = g->dden = g->part_dl = nullptr;
  }
  return s;
}

int ves3d_svp_set_density_dl(ves3d_svp* g, const double* gdl, int is_device) {
  VES3D_ARG(g != nullptr, "null context");
  VES3D_ARG(!g->grp.empty(), "set_src_coord first");
  int s;
  if (!gdl) {  // SetDensityDL(NULL): the double layer off
    for (ves3d_sv* sv : g->grp)
      if ((s = ves3d_sv_set_density_dl(sv, nullptr, 0))) return s;
    if (g->have_dl) g->drop_graph();
    g->have_dl = false;
    return VES3D_OK;
  }
  if ((s = svp_alloc_dl(g))) return s;
  // each group's own SetDensityDL: its G buffer, and the stage buffers its DL build needs
  for (size_t r = 0; r < g->grp.size(); r++)
    if ((s = ves3d_sv_set_density_dl(g->grp[r], gdl + 3 * g->gpt0[r], is_device))) return s;
  if (!g->have_dl) g->drop_graph();  // a captured evaluation without the double layer
  g->have_dl = true;
  return VES3D_OK;
}

int ves3d_svp_set_viscosity_contrast(ves3d_svp* g, const double* lambda, long n) {
  VES3D_ARG(g != nullptr, "null context");
  g->rhs_valid = false;
  if (!lambda || n == 0) {
    g->lam.clear();
    g->contrast = false;
    return VES3D_OK;
  }
  VES3D_ARG(n == 1 || (!g->grp.empty() && n == g->nves), "n must be 1 or the number of vesicles");
  for (long i = 0; i < n; i++) VES3D_ARG(std::isfinite(lambda[i]) && lambda[i] > 0.0, "contrast must be positive");
  g->lam.assign(lambda, lambda + n);
  bool any = false;
  for (double l : g->lam) any |= std::fabs(l - 1.0) > 1e-12;  // has_contrast, VesicleProps.cc:45-49
  g->contrast = any;
  return VES3D_OK;
}

int ves3d_svp_setup(ves3d_svp* g) {
  VES3D_ARG(g != nullptr, "null context");
  VES3D_ARG(!g->grp.empty(), "set_src_coord first");
  for (ves3d_sv* sv : g->grp) {
    int s;
    if (!sv->sl_valid && (s = run_setup(sv))) return s;
    if (g->have_dl && !sv->dl_valid && (s = run_setup(sv, true))) return s;
  }
  return VES3D_OK;
}

// every group's self part (with dl, of both layers: the DL matrices are built on first use)
static int svp_self_parts(ves3d_svp* g, bool dl) {
  for (size_t r = 0; r < g->grp.size(); r++) {
    ves3d_sv* sv = g->grp[r];
    int s;
    if (dl && !sv->dl_valid && (s = run_setup(sv, true))) return s;
    const long o = 3 * g->gpt0[r];
    if ((s = run_self(sv, g->vself + o, g->den + o, dl ? g->nrm + o : nullptr, dl ? g->dden + o : nullptr)))
      return s;
  }
  return VES3D_OK;
}

// one far-field pass over every point, launched per order group (block shape per group);
// with dl the far double layer (FP64) as a second set of partials of the same reduce
static int svp_far(ves3d_svp* g, bool dl) {
  NvtxRange nvtx("ves3d far");
  const bool mixed = g->prec == VES3D_PREC_MIXED && !g->far_force_fp64;
  std::vector<FarGroup> fg;
  long v0 = 0;
  for (size_t r = 0; r < g->grp.size(); r++) {
    fg.push_back(FarGroup{v0, g->gnv[r], ngrid_(g->gp[r])});
    v0 += g->gnv[r];
  }
  if (!dl)
    return launch_far_groups(mixed, g->pos, g->den, g->off, g->nves, g->N, fg.data(), (int)fg.size(), g->vself, g->V,
                             g->Vfar, g->part, kFarMaxSegments, g->stream);
  int s, nseg = 0, nseg_dl = 0;
  if ((s = launch_far_groups(mixed, g->pos, g->den, g->off, g->nves, g->N, fg.data(), (int)fg.size(), nullptr,
                             nullptr, nullptr, g->part, kFarMaxSegments, g->stream, &nseg)))
    return s;
  if ((s = launch_far_dl_groups(mixed && g->far_dl_f32, g->pos, g->nrm, g->dden, g->off, g->nves, g->N, fg.data(),
                                (int)fg.size(), g->part_dl, kFarMaxSegments, g->stream, &nseg_dl)))
    return s;
  return launch_far_reduce(g->part, nseg, g->off, g->nves, g->N, g->vself, g->V, g->Vfar, g->stream, g->part_dl,
                           nseg_dl, kDl);
}

int ves3d_svp_capture_eval(ves3d_svp* g) {
  VES3D_ARG(g != nullptr, "null context");
  if (g->grp.empty() || !g->have_den) {
    set_error("capture before set_src_coord / set_density_sl");
    return VES3D_ERR_STATE;
  }
  VES3D_CK(cudaSetDevice(g->device));
  g->drop_graph();
  int s;
  if ((s = ves3d_svp_setup(g))) return s;
  // one eager pass first: kernel attributes are set outside the capture
  if ((s = svp_self_parts(g, g->have_dl)) || (s = svp_far(g, g->have_dl))) return s;
  VES3D_CK(cudaStreamSynchronize(g->stream));
  VES3D_CK(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
  s = svp_self_parts(g, g->have_dl);
  if (!s) s = svp_far(g, g->have_dl);
  cudaGraph_t gr = nullptr;
  const cudaError_t e = cudaStreamEndCapture(g->stream, &gr);
  if (!s && e != cudaSuccess) s = cuda_status(e, "cudaStreamEndCapture", __FILE__, __LINE__);
  if (s) {
    if (gr) cudaGraphDestroy(gr);
    return s;
  }
  g->graph = gr;
  const cudaError_t ei = cudaGraphInstantiate(&g->graph_exec, gr, 0);
  if (ei != cudaSuccess) {
    g->drop_graph();
    return cuda_status(ei, "cudaGraphInstantiate", __FILE__, __LINE__);
  }
  return VES3D_OK;
}

int ves3d_svp_launch_eval_graph(ves3d_svp* g, double* vel, int is_device) {
  VES3D_ARG(g != nullptr, "null context");
  if (!g->graph_exec) {
    set_error("no captured evaluation (call ves3d_svp_capture_eval after setting surfaces and densities)");
    return VES3D_ERR_STATE;
  }
  VES3D_CK(cudaSetDevice(g->device));
  VES3D_CK(cudaGraphLaunch(g->graph_exec, g->stream));
  VES3D_LAUNCHED();
  return vel ? copy_out(vel, g->V, 3 * (size_t)g->N, is_device, g->stream) : VES3D_OK;
}

int ves3d_svp_eval(ves3d_svp* g, double* vel, int is_device) {
  VES3D_ARG(g && vel, "null argument");
  if (g->grp.empty() || !g->have_den) {
    set_error("eval before set_src_coord / set_density_sl");
    return VES3D_ERR_STATE;
  }
  VES3D_CK(cudaSetDevice(g->device));
  int s;
  VES3D_CK(cudaEventRecord(g->ev[0], g->stream));
  if ((s = ves3d_svp_setup(g))) return s;
  VES3D_CK(cudaEventRecord(g->ev[1], g->stream));
  if ((s = svp_self_parts(g, g->have_dl))) return s;
  VES3D_CK(cudaEventRecord(g->ev[2], g->stream));
  if ((s = svp_far(g, g->have_dl))) return s;
  VES3D_CK(cudaEventRecord(g->ev[3], g->stream));
  VES3D_CK(cudaEventSynchronize(g->ev[3]));
  VES3D_CK(cudaEventElapsedTime(&g->ms[0], g->ev[0], g->ev[1]));
  VES3D_CK(cudaEventElapsedTime(&g->ms[1], g->ev[1], g->ev[2]));
  VES3D_CK(cudaEventElapsedTime(&g->ms[2], g->ev[2], g->ev[3]));
  VES3D_CK(cudaEventElapsedTime(&g->ms[3], g->ev[0], g->ev[3]));
  return copy_out(vel, g->V, 3 * (size_t)g->N, is_device, g->stream);
}

int ves3d_svp_stage_times(ves3d_svp* g, float* ms) {
  VES3D_ARG(g && ms, "null argument");
  for (int i = 0; i < 4; i++) ms[i] = g->ms[i];
  return VES3D_OK;
}

}  // extern "C"


// ---- implicit step of a polydisperse suspension -------------------------------------
// Every order group keeps its own geometry, tractions, self matrices and preconditioner;
// the single layer between the force and finish phases is one evaluation over all points
// (each group's self part plus the far field across groups). Unknowns: the groups' SH
// coefficient vectors [u; sigma] one after another (group r at coff[r]); grid vectors
// [u (per-vesicle [3][ng] blocks, all points); sigma (all points)].
namespace {

int svp_prepare_implicit(ves3d_svp* g) {
  int s;
  if (g->contrast && g->lam.size() != 1 && (long)g->lam.size() != g->nves) {
    set_error("viscosity contrast was set for %ld vesicles, the surfaces have %ld", (long)g->lam.size(), g->nves);
    return VES3D_ERR_STATE;
  }
  for (ves3d_sv* sv : g->grp) mark_implicit(sv);  // FP64 self matrices before the setup
  if ((s = ves3d_svp_setup(g))) return s;
  g->coff.assign(g->grp.size() + 1, 0);
  for (size_t r = 0; r < g->grp.size(); r++) {
    ves3d_sv* sv = g->grp[r];
    if ((s = ves3d_sv_set_implicit_params(sv, g->dt, g->kappa, g->shear))) return s;
    if ((s = ves3d_sv_set_gravity(sv, g->drho, g->grav[0], g->grav[1], g->grav[2]))) return s;
    if ((s = ves3d_sv_set_precond(sv, g->precond))) return s;
    if ((s = ves3d_sv_set_precond_refresh(sv, g->pc_refresh))) return s;
    if ((s = ves3d_sv_set_surface_filter(sv, g->filter_freq))) return s;
    // the suspension's viscosity contrast for this group's vesicles (one value: all of
    // them), pushed only when it changed (a change rebuilds the group's preconditioner)
    std::vector<double> want;
    if (g->contrast && g->lam.size() == 1) {
      want = g->lam;
    } else if (g->contrast) {
      long first = 0;
      for (size_t q = 0; q < r; q++) first += g->gnv[q];
      want.assign(g->lam.begin() + first, g->lam.begin() + first + g->gnv[r]);
    }
    if (want != sv->lam &&
        (s = ves3d_sv_set_viscosity_contrast(sv, want.empty() ? nullptr : want.data(), (long)want.size())))
      return s;
    if ((s = ensure_geometry(sv))) return s;
    ImplicitWork iw;
    if ((s = implicit_work(sv, iw))) return s;
    g->coff[r + 1] = g->coff[r] + sh_unknowns(sv);
  }
  return VES3D_OK;
}

// g->V = S[f] over the whole suspension, f = every group's iw.f; with dl plus D[G], G the
// density in every group's G buffer
int svp_stokes(ves3d_svp* g, bool dl = false) {
  int s;
  for (ves3d_sv* sv : g->grp) {
    ImplicitWork iw;
    if ((s = implicit_work(sv, iw))) return s;
    VES3D_CK(cudaMemcpyAsync(sv->F, iw.f, 3 * (size_t)sv->npts() * sizeof(double), cudaMemcpyDeviceToDevice,
                             g->stream));
    sv->have_den = true;
  }
  if ((s = svp_self_parts(g, dl))) return s;
  return svp_far(g, dl);
}

// The suspension's implicit operator on SH coefficients c (ImplicitApply,
// src/InterfacialVelocity.cc:878-966): every group's forces, one evaluation over all points,
// every group's finish. Under a viscosity contrast the evaluation adds the double layer of
// (1 - lambda) u and the finish takes (1 + lambda)/2 u - Sf (the groups' own contrast
// coefficients); the groups' G buffers then belong to the operator.
int svp_matvec_sh(ves3d_svp* g, const double* c, double* y) {
  int s;
  const bool con = g->contrast;
  if (con) {
    if ((s = svp_alloc_dl(g))) return s;
    g->have_dl = false;  // the G buffers hold the operator's densities from here on
    g->drop_graph();
  }
  for (size_t r = 0; r < g->grp.size(); r++) {
    ves3d_sv* sv = g->grp[r];
    ImplicitWork iw;
    if ((s = implicit_work(sv, iw))) return s;
    if ((s = coef_to_grid(sv, c + g->coff[r], iw.g1))) return s;
    if ((s = implicit_forces(sv, base_space(sv), iw, iw.g1))) return s;
    if (con) {
      const long N = sv->npts(), per = 3L * ngrid_(sv->p);
      if ((s = ensure_contrast(sv))) return s;
      if ((s = launch_scale_vesicles(iw.g1, 3 * N, per, sv->dlc, sv->nves, nullptr, 0.0, sv->G, g->stream))) return s;
    }
  }
  if ((s = svp_stokes(g, con))) return s;
  for (size_t r = 0; r < g->grp.size(); r++) {
    ves3d_sv* sv = g->grp[r];
    ImplicitWork iw;
    if ((s = implicit_work(sv, iw))) return s;
    const double* Sf = g->V + 3 * g->gpt0[r];
    if (!con) {
      if ((s = implicit_finish(sv, base_space(sv), iw.g1, Sf, iw.g2))) return s;
    } else {
      const long N = sv->npts(), per = 3L * ngrid_(sv->p);
      if ((s = launch_scale_vesicles(iw.g1, 3 * N, per, sv->velc, sv->nves, Sf, -1.0, iw.g2, g->stream))) return s;
      if ((s = op_div(sv, base_space(sv), Sf, iw.g2 + 3 * N, -1.0))) return s;
    }
    if ((s = grid_to_coef(sv, iw.g2, y + g->coff[r]))) return s;
  }
  return VES3D_OK;
}

int svp_matvec_cb(void* ctx, const double* x, double* y) { return svp_matvec_sh((ves3d_svp*)ctx, x, y); }

int svp_matvec_fp64_cb(void* ctx, const double* x, double* y) {
  ves3d_svp* g = (ves3d_svp*)ctx;
  g->far_force_fp64 = 1;
  const int s = svp_matvec_sh(g, x, y);
  g->far_force_fp64 = 0;
  return s;
}

int svp_precond_cb(void* ctx, const double* x, double* y) {
  ves3d_svp* g = (ves3d_svp*)ctx;
  for (size_t r = 0; r < g->grp.size(); r++) {
    const int s = precond_apply(g->grp[r], x + g->coff[r], y + g->coff[r]);
    if (s) return s;
  }
  return VES3D_OK;
}

// right-hand side in coefficients (FP64 far field), from the cache when the surfaces and
// parameters are unchanged since it was computed
int svp_rhs_compute(ves3d_svp* g, double* b);
int svp_rhs(ves3d_svp* g, double* b) {
  int s;
  const long nsh = g->coff.back();
  if (g->rhs_valid && g->rhs_cap >= nsh) {
    VES3D_CK(cudaMemcpyAsync(b, g->rhs, nsh * sizeof(double), cudaMemcpyDeviceToDevice, g->stream));
    return VES3D_OK;
  }
  if ((s = svp_rhs_compute(g, b))) return s;
  if (g->rhs_cap < nsh) {
    dfree(g->rhs);
    g->rhs = nullptr;
    g->rhs_cap = 0;
    if ((s = dalloc(&g->rhs, nsh))) return s;
    g->rhs_cap = nsh;
  }
  VES3D_CK(cudaMemcpyAsync(g->rhs, b, nsh * sizeof(double), cudaMemcpyDeviceToDevice, g->stream));
  g->rhs_valid = true;
  return VES3D_OK;
}

int svp_rhs_compute(ves3d_svp* g, double* b) {
  int s;
  for (ves3d_sv* sv : g->grp) {
    ImplicitWork iw;
    if ((s = implicit_work(sv, iw))) return s;
    if ((s = rhs_forces(sv, iw))) return s;
  }
  g->far_force_fp64 = 1;
  s = svp_stokes(g);
  g->far_force_fp64 = 0;
  if (s) return s;
  for (size_t r = 0; r < g->grp.size(); r++) {
    ves3d_sv* sv = g->grp[r];
    ImplicitWork iw;
    if ((s = implicit_work(sv, iw))) return s;
    if ((s = rhs_finish(sv, g->V + 3 * g->gpt0[r], iw.g2))) return s;
    if ((s = grid_to_coef(sv, iw.g2, b + g->coff[r]))) return s;
  }
  return VES3D_OK;
}

// global grid vector [u; sigma] <-> group coefficient vectors
int svp_grid_to_coef(ves3d_svp* g, const double* x, double* c) {
  int s;
  for (size_t r = 0; r < g->grp.size(); r++) {
    ves3d_sv* sv = g->grp[r];
    ImplicitWork iw;
    if ((s = implicit_work(sv, iw))) return s;
    const size_t n = (size_t)sv->npts();
    VES3D_CK(cudaMemcpyAsync(iw.g1, x + 3 * g->gpt0[r], 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, g->stream));
    VES3D_CK(cudaMemcpyAsync(iw.g1 + 3 * n, x + 3 * g->N + g->gpt0[r], n * sizeof(double), cudaMemcpyDeviceToDevice,
                             g->stream));
    if ((s = grid_to_coef(sv, iw.g1, c + g->coff[r]))) return s;
  }
  return VES3D_OK;
}

int svp_coef_to_grid(ves3d_svp* g, const double* c, double* x) {
  int s;
  for (size_t r = 0; r < g->grp.size(); r++) {
    ves3d_sv* sv = g->grp[r];
    ImplicitWork iw;
    if ((s = implicit_work(sv, iw))) return s;
    const size_t n = (size_t)sv->npts();
    if ((s = coef_to_grid(sv, c + g->coff[r], iw.g1))) return s;
    VES3D_CK(cudaMemcpyAsync(x + 3 * g->gpt0[r], iw.g1, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, g->stream));
    VES3D_CK(cudaMemcpyAsync(x + 3 * g->N + g->gpt0[r], iw.g1 + 3 * n, n * sizeof(double), cudaMemcpyDeviceToDevice,
                             g->stream));
  }
  return VES3D_OK;
}

}  // namespace

extern "C" {

int ves3d_svp_set_implicit_params(ves3d_svp* g, double dt, double kappa, double shear_rate) {
  VES3D_ARG(g != nullptr, "null context");
  VES3D_ARG(dt > 0 && kappa >= 0, "dt must be > 0 and kappa >= 0");
  g->dt = dt;
  g->kappa = kappa;
  g->shear = shear_rate;
  g->rhs_valid = false;
  return VES3D_OK;
}

int ves3d_svp_set_gravity(ves3d_svp* g, double excess_density, double gx, double gy, double gz) {
  VES3D_ARG(g != nullptr, "null context");
  g->drho = excess_density;
  g->grav[0] = gx;
  g->grav[1] = gy;
  g->grav[2] = gz;
  g->rhs_valid = false;
  return VES3D_OK;
}

int ves3d_svp_set_surface_filter(ves3d_svp* g, int filter_freq) {
  VES3D_ARG(g != nullptr, "null context");
  VES3D_ARG(filter_freq >= -1, "filter frequency: 0 (off), -1 (2p/3) or the highest degree kept");
  g->filter_freq = filter_freq;
  g->rhs_valid = false;
  return VES3D_OK;
}

int ves3d_svp_set_precond(ves3d_svp* g, int scheme, int refresh_every) {
  VES3D_ARG(g != nullptr, "null context");
  VES3D_ARG(scheme >= VES3D_PRECOND_NONE && scheme <= VES3D_PRECOND_SELF_BLOCK, "unknown preconditioner");
  VES3D_ARG(refresh_every >= 1, "refresh interval must be >= 1");
  g->precond = scheme;
  g->pc_refresh = refresh_every;
  return VES3D_OK;
}

int ves3d_svp_solver_stats(ves3d_svp* g, int* outer, int* inner) {
  VES3D_ARG(g && outer && inner, "null argument");
  *outer = g->ir_outer;
  *inner = g->ir_inner;
  return VES3D_OK;
}

int ves3d_svp_implicit_solve(ves3d_svp* g, const double* x0, double* x, double* tol, int* max_iter, int* code,
                             int is_device) {
  NvtxRange nvtx("ves3d svp implicit_solve");
  VES3D_ARG(g && x && tol && max_iter && code, "null argument");
  if (g->grp.empty()) {
    set_error("no surfaces set");
    return VES3D_ERR_STATE;
  }
  VES3D_CK(cudaSetDevice(g->device));
  int s;
  if ((s = svp_prepare_implicit(g))) return s;
  const long nsh = g->coff.back(), ng4 = 4 * g->N, nws = bicgstab_workspace_doubles(nsh);
  const long need = nws + 2 * nsh + ng4;
  if (g->sws_cap < need) {
    dfree(g->sws);
    g->sws = nullptr;
    g->sws_cap = 0;
    if ((s = dalloc(&g->sws, need))) return s;
    g->sws_cap = need;
  }
  double *ws = g->sws, *dc = ws + nws, *db = dc + nsh, *dg = db + nsh;
  if (x0) {
    s = copy_in(dg, x0, ng4, is_device, g->stream);
    if (!s) s = svp_grid_to_coef(g, dg, dc);
  } else {
    s = cuda_status(cudaMemsetAsync(dc, 0, nsh * sizeof(double), g->stream), "memset", __FILE__, __LINE__);
  }
  if (!s) s = svp_rhs(g, db);
  for (size_t r = 0; r < g->grp.size() && !s; r++) s = ensure_precond(g->grp[r]);
  const MatVecFn P = g->precond == VES3D_PRECOND_NONE ? nullptr : svp_precond_cb;
  if (!s) {
    if (g->prec == VES3D_PREC_FP64) {
      s = bicgstab_run(svp_matvec_cb, g, dc, db, nsh, tol, max_iter, code, ws, g->stream, P, g);
      g->ir_outer = 0;
      g->ir_inner = *max_iter;
    } else {
      SolveOps ops;
      ops.mixed = svp_matvec_cb;
      ops.fp64 = svp_matvec_fp64_cb;
      ops.P = P;
      ops.ctx = g;
      ops.st = g->stream;
      s = mixed_refinement(ops, dc, db, nsh, tol, max_iter, code, &g->ir_outer, &g->ir_inner);
    }
  }
  if (!s) s = svp_coef_to_grid(g, dc, dg);
  if (!s) s = copy_out(x, dg, ng4, is_device, g->stream);
  cudaStreamSynchronize(g->stream);
  return s;
}

}  // extern "C"

extern "C" {

// Residual-minimising combination of candidate guesses for the next implicit solve of a
// polydisperse suspension (the uniform form: ves3d_sv_implicit_combine). The candidates'
// images come from the operator the inner solves use (the FP32 far field in a mixed
// context: a guess needs no more, and the solve that follows checks its result in FP64);
// the right-hand side is FP64 and is kept for that solve.
int ves3d_svp_implicit_combine(ves3d_svp* g, int n_cand, const double* const* cand, double* x0, double* weights,
                               double* relres, int is_device) {
  VES3D_ARG(g != nullptr, "null context");
  VES3D_ARG(n_cand >= 1 && n_cand <= 8, "n_cand must be in [1, 8]");
  VES3D_ARG(cand && x0 && weights && relres, "null argument");
  for (int i = 0; i < n_cand; i++) VES3D_ARG(cand[i] != nullptr, "null candidate");
  if (g->grp.empty()) {
    set_error("no surfaces set");
    return VES3D_ERR_STATE;
  }
  VES3D_CK(cudaSetDevice(g->device));
  int s;
  if ((s = svp_prepare_implicit(g))) return s;
  const long nsh = g->coff.back(), ng4 = 4 * g->N;
  double *b = nullptr, *C = nullptr, *Y = nullptr, *dg = nullptr, *r = nullptr, *scr = nullptr;
  if ((s = dalloc(&b, nsh))) return s;
  if ((s = dalloc(&C, nsh * n_cand)) || (s = dalloc(&Y, nsh * n_cand)) || (s = dalloc(&dg, ng4)) ||
      (s = dalloc(&r, nsh)) || (s = dalloc(&scr, 1024))) {
    dfree(b); dfree(C); dfree(Y); dfree(dg); dfree(r);
    return s;
  }
  s = svp_rhs(g, b);
  for (int i = 0; i < n_cand && !s; i++) {
    s = copy_in(dg, cand[i], ng4, is_device, g->stream);
    if (!s) s = svp_grid_to_coef(g, dg, C + i * nsh);
    if (!s) s = svp_matvec_sh(g, C + i * nsh, Y + i * nsh);
  }
  std::vector<double> G(n_cand * n_cand, 0.0), h(n_cand, 0.0), a;
  std::vector<char> ok(n_cand, 1);
  double bb = 0;
  if (!s) s = dot_f64(b, b, nsh, scr, &bb, g->stream);
  const double nb = bb > 0 ? std::sqrt(bb) : 1.0;
  for (int i = 0; i < n_cand && !s; i++) {
    s = lincomb_f64(nsh, 1.0, b, -1.0, Y + i * nsh, 0.0, nullptr, r, g->stream);
    double rr = 0;
    if (!s) s = dot_f64(r, r, nsh, scr, &rr, g->stream);
    relres[i] = std::sqrt(rr) / nb;
    if (!s) s = dot_f64(Y + i * nsh, b, nsh, scr, &h[i], g->stream);
    for (int j = 0; j <= i && !s; j++) {
      s = dot_f64(Y + i * nsh, Y + j * nsh, nsh, scr, &G[i * n_cand + j], g->stream);
      G[j * n_cand + i] = G[i * n_cand + j];
    }
    if (!std::isfinite(G[i * n_cand + i]) || !std::isfinite(h[i])) ok[i] = 0;
  }
  if (!s) {
    std::vector<int> idx;
    for (int i = 0; i < n_cand; i++)
      if (ok[i] && G[i * n_cand + i] > 0) idx.push_back(i);
    const int m = (int)idx.size();
    std::vector<double> Gm(m * m), hm(m), am;
    for (int i = 0; i < m; i++) {
      hm[i] = h[idx[i]];
      for (int j = 0; j < m; j++) Gm[i * m + j] = G[idx[i] * n_cand + idx[j]];
    }
    if (m) small_solve(m, Gm, hm, am);
    for (int i = 0; i < n_cand; i++) weights[i] = 0.0;
    for (int i = 0; i < m; i++) weights[idx[i]] = am[i];
    s = cuda_status(cudaMemsetAsync(dg, 0, nsh * sizeof(double), g->stream), "memset", __FILE__, __LINE__);
    if (!s) s = copy_in(r, b, nsh, 1, g->stream);
    for (int i = 0; i < m && !s; i++) {
      s = lincomb_f64(nsh, 1.0, dg, am[i], C + idx[i] * nsh, 0.0, nullptr, dg, g->stream);
      if (!s) s = lincomb_f64(nsh, 1.0, r, -am[i], Y + idx[i] * nsh, 0.0, nullptr, r, g->stream);
    }
    double rr = 0;
    if (!s) s = dot_f64(r, r, nsh, scr, &rr, g->stream);
    relres[n_cand] = std::sqrt(rr) / nb;
    if (!s) {
      s = copy_in(b, dg, nsh, 1, g->stream);  // coefficients of the combination
      if (!s) s = svp_coef_to_grid(g, b, dg);
      if (!s) s = copy_out(x0, dg, ng4, is_device, g->stream);
    }
  }
  cudaStreamSynchronize(g->stream);
  dfree(b);
  dfree(C);
  dfree(Y);
  dfree(dg);
  dfree(r);
  dfree(scr);
  return s;
}

}  // extern "C"
