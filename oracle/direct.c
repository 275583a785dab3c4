/* CPU oracle (test infrastructure only): plain-C restatement of the reference's
 * Stokes single-layer direct sums. Only tests/, bench.py's cpu_baseline leg and
 * __graft_entry__.smoke() may load it, as the checker or the timed CPU baseline.
 *
 *   oracle_alltoall       follows StokesAlltoAll (double)      src/CPUKernels.cc:1011-1057
 *   oracle_direct_stokes  follows DirectStokesKernel (double)  src/CPUKernels.cc:123-178
 *   oracle_far            the all-pairs sum with same-vesicle sources left out, i.e.
 *                         StokesAlltoAll - DirectStokesKernel as composed in
 *                         src/InterfacialVelocity.cc:1261-1291, with the difference taken
 *                         pair by pair instead of after summation.
 *
 *   oracle_direct_stokes_dl follows DirectStokesDoubleLayerKernel (double)
 *                                            src/CPUKernels.cc:1060-1120
 *   oracle_far_dl         the double-layer sum over the points of the other vesicles, the
 *                         kernel of the far-field double layer (stokes_dl_uKernel,
 *                         src/PVFMMInterface.cc:285-360) in the composition above.
 *
 * Kernel per pair (r = x_s - x_t, d = density * weights):
 *   u_t += 1/(8 pi) [ d / |r| + (r.d) r / |r|^3 ],  and a coincident pair (r == 0)
 *   contributes nothing (invR stays 0, src/CPUKernels.cc:1036-1037).
 */
#include <math.h>
#include <stddef.h>

#define ORACLE_I_PI (1.0 / M_PI / 8.0)
/* double layer: 3/(4 pi); per pair with r = x_t - x_s the velocity gains
 * 3/(4 pi) (r.n)(r.d) r / |r|^5 (the reference's DirectStokesDoubleLayerKernel writes the
 * same with r = x_s - x_t and -3/(4 pi)); a coincident pair contributes nothing. */
#define ORACLE_DL_SCALE (3.0 / (4.0 * M_PI))

void oracle_alltoall(const double* src, const double* den, long np, double* pot) {
#pragma omp parallel for schedule(static)
  for (long t = 0; t < np; t++) {
    double tx = src[3 * t], ty = src[3 * t + 1], tz = src[3 * t + 2];
    double px = 0, py = 0, pz = 0;
    for (long s = 0; s < np; s++) {
      double dx = src[3 * s] - tx, dy = src[3 * s + 1] - ty, dz = src[3 * s + 2] - tz;
      double invR = dx * dx + dy * dy + dz * dz;
      if (invR != 0) invR = 1.0 / sqrt(invR);
      double cx = den[3 * s], cy = den[3 * s + 1], cz = den[3 * s + 2];
      double cc = (dx * cx + dy * cy + dz * cz) * invR * invR;
      cx += cc * dx;
      cy += cc * dy;
      cz += cc * dz;
      px += cx * invR;
      py += cy * invR;
      pz += cz * invR;
    }
    pot[3 * t] = px * ORACLE_I_PI;
    pot[3 * t + 1] = py * ORACLE_I_PI;
    pot[3 * t + 2] = pz * ORACLE_I_PI;
  }
}

/* AxisMajor per surface: x[v][c][stride]. Targets [trg_idx_head, trg_idx_tail). */
void oracle_direct_stokes(int src_stride, int trg_stride, int n_surfs, int trg_idx_head, int trg_idx_tail,
                          const double* qw, const double* trg, const double* src, const double* den,
                          double* pot) {
#pragma omp parallel for schedule(static)
  for (int v = 0; v < n_surfs; v++) {
    const double* S = src + 3L * src_stride * v;
    const double* D = den + 3L * src_stride * v;
    const double* T = trg + 3L * trg_stride * v;
    double* P = pot + 3L * trg_stride * v;
    for (int t = trg_idx_head; t < trg_idx_tail; t++) {
      double tx = T[t], ty = T[trg_stride + t], tz = T[2 * trg_stride + t];
      double px = 0, py = 0, pz = 0;
      for (int s = 0; s < src_stride; s++) {
        double dx = S[s] - tx, dy = S[src_stride + s] - ty, dz = S[2 * src_stride + s] - tz;
        double invR = dx * dx + dy * dy + dz * dz;
        if (invR != 0) invR = 1.0 / sqrt(invR);
        double cx = D[s] * qw[s], cy = D[src_stride + s] * qw[s], cz = D[2 * src_stride + s] * qw[s];
        double cc = (dx * cx + dy * cy + dz * cz) * invR * invR;
        cx += cc * dx;
        cy += cc * dy;
        cz += cc * dz;
        px += cx * invR;
        py += cy * invR;
        pz += cz * invR;
      }
      P[t] = px * ORACLE_I_PI;
      P[trg_stride + t] = py * ORACLE_I_PI;
      P[2 * trg_stride + t] = pz * ORACLE_I_PI;
    }
  }
}

/* Far field for n_trg targets (global point indices trg_idx[], or all points when
 * trg_idx is NULL): sources are every point of every other vesicle.
 * X, D: AxisMajor per vesicle, vesicle v holding points [pt_off[v], pt_off[v+1]) as
 * [3][n_v] starting at element 3*pt_off[v]; D already carries area * weights.
 * out: [n_trg][3] point-major. */
void oracle_far(const double* X, const double* D, long nves, const long* pt_off, const long* trg_idx, long n_trg,
                double* out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (long it = 0; it < n_trg; it++) {
    long g = trg_idx ? trg_idx[it] : it;
    long lo = 0, hi = nves;
    while (hi - lo > 1) { /* vesicle of point g */
      long mid = (lo + hi) / 2;
      if (pt_off[mid] <= g) lo = mid; else hi = mid;
    }
    long vt = lo, nt = pt_off[vt + 1] - pt_off[vt], kt = g - pt_off[vt];
    const double* Tv = X + 3 * pt_off[vt];
    double tx = Tv[kt], ty = Tv[nt + kt], tz = Tv[2 * nt + kt];
    double px = 0, py = 0, pz = 0;
    for (long v = 0; v < nves; v++) {
      if (v == vt) continue;
      long n = pt_off[v + 1] - pt_off[v];
      const double* S = X + 3 * pt_off[v];
      const double* Dv = D + 3 * pt_off[v];
      for (long s = 0; s < n; s++) {
        double dx = S[s] - tx, dy = S[n + s] - ty, dz = S[2 * n + s] - tz;
        double invR = dx * dx + dy * dy + dz * dz;
        if (invR != 0) invR = 1.0 / sqrt(invR);
        double cx = Dv[s], cy = Dv[n + s], cz = Dv[2 * n + s];
        double cc = (dx * cx + dy * cy + dz * cz) * invR * invR;
        cx += cc * dx;
        cy += cc * dy;
        cz += cc * dz;
        px += cx * invR;
        py += cy * invR;
        pz += cz * invR;
      }
    }
    out[3 * it] = px * ORACLE_I_PI;
    out[3 * it + 1] = py * ORACLE_I_PI;
    out[3 * it + 2] = pz * ORACLE_I_PI;
  }
}

/* AxisMajor per surface, unit normals norm, weights qw (NULL: none). */
void oracle_direct_stokes_dl(int src_stride, int trg_stride, int n_surfs, int trg_idx_head, int trg_idx_tail,
                             const double* qw, const double* trg, const double* src, const double* norm,
                             const double* den, double* pot) {
#pragma omp parallel for schedule(static)
  for (int v = 0; v < n_surfs; v++) {
    const double* S = src + 3L * src_stride * v;
    const double* N = norm + 3L * src_stride * v;
    const double* D = den + 3L * src_stride * v;
    const double* T = trg + 3L * trg_stride * v;
    double* P = pot + 3L * trg_stride * v;
    for (int t = trg_idx_head; t < trg_idx_tail; t++) {
      double tx = T[t], ty = T[trg_stride + t], tz = T[2 * trg_stride + t];
      double px = 0, py = 0, pz = 0;
      for (int s = 0; s < src_stride; s++) {
        double dx = tx - S[s], dy = ty - S[src_stride + s], dz = tz - S[2 * src_stride + s];
        double invR = dx * dx + dy * dy + dz * dz;
        if (invR != 0) invR = 1.0 / sqrt(invR);
        double invR5 = invR * invR;
        invR5 = invR5 * invR5 * invR;
        double rn = dx * N[s] + dy * N[src_stride + s] + dz * N[2 * src_stride + s];
        double rf = dx * D[s] + dy * D[src_stride + s] + dz * D[2 * src_stride + s];
        double q = rn * rf * invR5;
        if (qw) q *= qw[s];
        px += dx * q;
        py += dy * q;
        pz += dz * q;
      }
      P[t] = px * ORACLE_DL_SCALE;
      P[trg_stride + t] = py * ORACLE_DL_SCALE;
      P[2 * trg_stride + t] = pz * ORACLE_DL_SCALE;
    }
  }
}

/* Far double layer at every point (n_trg = pt_off[nves]): sources are the points of the
 * other vesicles, with unit normals N and densities D (already times area and weights),
 * both AxisMajor per vesicle like X. out: [n_trg][3] point-major. */
void oracle_far_dl(const double* X, const double* N, const double* D, long nves, const long* pt_off, double* out) {
  long n_trg = pt_off[nves];
#pragma omp parallel for schedule(dynamic, 16)
  for (long g = 0; g < n_trg; g++) {
    long lo = 0, hi = nves;
    while (hi - lo > 1) {
      long mid = (lo + hi) / 2;
      if (pt_off[mid] <= g) lo = mid; else hi = mid;
    }
    long vt = lo, nt = pt_off[vt + 1] - pt_off[vt], kt = g - pt_off[vt];
    const double* Tv = X + 3 * pt_off[vt];
    double tx = Tv[kt], ty = Tv[nt + kt], tz = Tv[2 * nt + kt];
    double px = 0, py = 0, pz = 0;
    for (long v = 0; v < nves; v++) {
      if (v == vt) continue;
      long n = pt_off[v + 1] - pt_off[v];
      const double* S = X + 3 * pt_off[v];
      const double* Nv = N + 3 * pt_off[v];
      const double* Dv = D + 3 * pt_off[v];
      for (long s = 0; s < n; s++) {
        double dx = tx - S[s], dy = ty - S[n + s], dz = tz - S[2 * n + s];
        double invR = dx * dx + dy * dy + dz * dz;
        if (invR != 0) invR = 1.0 / sqrt(invR);
        double invR5 = invR * invR;
        invR5 = invR5 * invR5 * invR;
        double q = (dx * Nv[s] + dy * Nv[n + s] + dz * Nv[2 * n + s]) *
                   (dx * Dv[s] + dy * Dv[n + s] + dz * Dv[2 * n + s]) * invR5;
        px += dx * q;
        py += dy * q;
        pz += dz * q;
      }
    }
    out[3 * g] = px * ORACLE_DL_SCALE;
    out[3 * g + 1] = py * ORACLE_DL_SCALE;
    out[3 * g + 2] = pz * ORACLE_DL_SCALE;
  }
}
