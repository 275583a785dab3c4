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
 * Kernel per pair (r = x_s - x_t, d = density * weights):
 *   u_t += 1/(8 pi) [ d / |r| + (r.d) r / |r|^3 ],  and a coincident pair (r == 0)
 *   contributes nothing (invR stays 0, src/CPUKernels.cc:1036-1037).
 */
#include <math.h>
#include <stddef.h>

#define ORACLE_I_PI (1.0 / M_PI / 8.0)

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
