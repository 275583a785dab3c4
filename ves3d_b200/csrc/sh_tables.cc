// Host-side spherical-harmonic operator tables (FP64). See sh_tables.h.
#include "sh_tables.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace ves3d {

static const double kPi = 3.14159265358979323846264338327950288;

void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  if (n == 1) {
    x[0] = 0.0;
    w[0] = 2.0;
    return;
  }
  for (int i = 0; i < n; i++) {
    // Newton on P_n from the standard asymptotic initial guess; nodes descending in i.
    double z = std::cos(kPi * (i + 0.75) / (n + 0.5));
    double pp = 1.0;
    for (int it = 0; it < 100; it++) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; k++) {
        double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      pp = n * (z * p1 - p0) / (z * z - 1.0);
      double dz = p1 / pp;
      z -= dz;
      if (std::fabs(dz) < 1e-17) break;
    }
    double p0 = 1.0, p1 = z;
    for (int k = 2; k <= n; k++) {
      double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    pp = n * (z * p1 - p0) / (z * z - 1.0);
    x[n - 1 - i] = z;
    w[n - 1 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

void legpoly(const double* x, const double* u_in, int N, int d, double* out) {
  std::vector<double> u(N), diag((d + 1) * (size_t)N);
  for (int k = 0; k < N; k++) {
    if (u_in) {
      u[k] = u_in[k];
    } else {
      u[k] = x[k] * x[k] > 1.0 ? 0.0 : std::sqrt(1.0 - x[k] * x[k]);
    }
    diag[k] = 1.0 / std::sqrt(4.0 * kPi);
  }
  for (int i = 1; i <= d; i++) {
    double c = std::sqrt((2.0 * i + 1.0) / (2.0 * i));
    for (int k = 0; k < N; k++) diag[(size_t)i * N + k] = -diag[(size_t)(i - 1) * N + k] * u[k] * c;
  }
  size_t off = 0;
  for (int m = 0; m <= d; m++) {
    for (int k = 0; k < N; k++) {
      double pmm = 0.0, pmmp1 = diag[(size_t)m * N + k];
      out[off * N + k] = pmmp1;
      for (int l = m + 1; l <= d; l++) {
        double a = std::sqrt(((2.0 * l - 1) * (2.0 * l + 1)) / ((double)(l - m) * (l + m)));
        double b = l > 1 ? std::sqrt(((2.0 * l + 1) * (l + m - 1.0) * (l - m - 1.0)) /
                                     ((double)(l - m) * (l + m) * (2.0 * l - 3)))
                         : 0.0;
        double pll = x[k] * a * pmmp1 - b * pmm;
        pmm = pmmp1;
        pmmp1 = pll;
        out[(off + (l - m)) * N + k] = pll;
      }
    }
    off += d + 1 - m;
  }
}

static inline size_t aidx(int d, int m, int n) { return (size_t)(((2 * d - m + 1) * m) / 2 + n); }

void legpoly_deriv(const double* x, int N, int d, double* out) {
  size_t na = (size_t)(d + 1) * (d + 2) / 2;
  std::vector<double> P(na * N);
  legpoly(x, nullptr, N, d, P.data());
  for (int m = 0; m <= d; m++)
    for (int n = m; n <= d; n++) {
      const double* Pn = &P[aidx(d, m, n) * N];
      const double* Pn_ = (m + 1 <= n) ? &P[aidx(d, m + 1, n) * N] : &P[0];
      double c1 = (double)m;
      double c2 = (m + 1 <= n) ? std::sqrt(n + m + 1.0) * std::sqrt(n > m ? (double)(n - m) : 1.0) : 0.0;
      double* H = &out[aidx(d, m, n) * N];
      for (int k = 0; k < N; k++) {
        double s = std::sqrt(1.0 - x[k] * x[k]);
        H[k] = -(c1 * x[k] * Pn[k] + c2 * s * Pn_[k]) / s;
      }
    }
}

// MatFourier (src/SphericalHarmonics.cc:607-627), 2p0 x 2p1.
static void mat_fourier(int p0, int p1, std::vector<double>& M) {
  const double s2p = std::sqrt(2.0 * kPi);
  M.assign((size_t)4 * p0 * p1, 0.0);
  for (int j = 0; j < 2 * p1; j++) {
    M[j] = s2p;
    for (int k = 1; k < p0; k++) {
      M[(size_t)(2 * k - 1) * 2 * p1 + j] = s2p * std::cos(j * k * kPi / p1);
      M[(size_t)(2 * k) * 2 * p1 + j] = s2p * std::sin(j * k * kPi / p1);
    }
    M[(size_t)(2 * p0 - 1) * 2 * p1 + j] = s2p * std::cos(j * p0 * kPi / p1);
  }
}

// MatFourierGrad (:654-674).
static void mat_fourier_grad(int p0, int p1, std::vector<double>& M) {
  const double s2p = std::sqrt(2.0 * kPi);
  M.assign((size_t)4 * p0 * p1, 0.0);
  for (int j = 0; j < 2 * p1; j++) {
    for (int k = 1; k < p0; k++) {
      M[(size_t)(2 * k - 1) * 2 * p1 + j] = -s2p * k * std::sin(j * k * kPi / p1);
      M[(size_t)(2 * k) * 2 * p1 + j] = s2p * k * std::cos(j * k * kPi / p1);
    }
    M[(size_t)(2 * p0 - 1) * 2 * p1 + j] = -s2p * p0 * std::sin(j * p0 * kPi / p1);
  }
}

// MatFourierInv (:629-652), 2p0 x 2p1.
static void mat_fourier_inv(int p0, int p1, std::vector<double>& M) {
  const double c = 1.0 / std::sqrt(2.0 * kPi) / p0;
  M.assign((size_t)4 * p0 * p1, 0.0);
  int q = std::min(p0, p1);
  for (int j = 0; j < 2 * p0; j++) {
    double* row = &M[(size_t)j * 2 * p1];
    row[0] = c * 0.5;
    for (int k = 1; k < q; k++) {
      row[2 * k - 1] = c * std::cos(j * k * kPi / p0);
      row[2 * k] = c * std::sin(j * k * kPi / p0);
    }
    row[2 * q - 1] = c * std::cos(j * q * kPi / p0);
    if (q == p0) row[2 * q - 1] *= 0.5;
  }
}

// Per-coefficient Legendre columns for a coefficient layout of order p at N points:
// out[coef][k] = A[aidx(p, m, n)][k] for coef = (Fourier block jf, degree n).
static void per_coef(int p, const std::vector<double>& A, int N, std::vector<double>& out) {
  out.assign((size_t)ncoef(p) * N, 0.0);
  size_t c = 0;
  for (int jf = 0; jf < 2 * p; jf++) {
    int m = (jf + 1) / 2;
    for (int n = m; n <= p; n++, c++)
      std::memcpy(&out[c * N], &A[aidx(p, m, n) * N], sizeof(double) * N);
  }
}

static void build_synth(int p0, int q, const std::vector<double>& xq, SynthTables& S) {
  S.p0 = p0;
  S.q = q;
  size_t na = (size_t)(p0 + 1) * (p0 + 2) / 2;
  std::vector<double> A(na * (q + 1)), D(na * (q + 1));
  legpoly(xq.data(), nullptr, q + 1, p0, A.data());
  legpoly_deriv(xq.data(), q + 1, p0, D.data());
  per_coef(p0, A, q + 1, S.leg);
  per_coef(p0, D, q + 1, S.dleg);
  mat_fourier(p0, q, S.four);
  mat_fourier_grad(p0, q, S.dfour);
}

static void build_analysis(int pin, int pout, AnalysisTables& T) {
  T.pin = pin;
  T.pout = pout;
  std::vector<double> x, w;
  gauss_legendre(pin + 1, x, w);
  size_t na = (size_t)(pout + 1) * (pout + 2) / 2;
  std::vector<double> A(na * (pin + 1));
  legpoly(x.data(), nullptr, pin + 1, pout, A.data());
  per_coef(pout, A, pin + 1, T.leg);
  for (size_t c = 0; c < (size_t)ncoef(pout); c++)
    for (int k = 0; k <= pin; k++) T.leg[c * (pin + 1) + k] *= w[k] * 2.0 * kPi;
  mat_fourier_inv(pin, pout, T.four);
}

void build_synth_tables(int p0, int q, SynthTables& S) {
  std::vector<double> x, w;
  gauss_legendre(q + 1, x, w);
  build_synth(p0, q, x, S);
}

void build_analysis_tables(int pin, int pout, AnalysisTables& A) { build_analysis(pin, pout, A); }

void coef_blocks(int p, std::vector<int>& blk_off, std::vector<int>& jf_of_coef) {
  blk_off.assign(2 * p + 1, 0);
  jf_of_coef.assign(ncoef(p), 0);
  int c = 0;
  for (int jf = 0; jf < 2 * p; jf++) {
    blk_off[jf] = c;
    for (int n = (jf + 1) / 2; n <= p; n++) jf_of_coef[c++] = jf;
  }
  blk_off[2 * p] = c;
}

void host_grid2shc(const AnalysisTables& A, const double* X, long nfun, double* S) {
  int pin = A.pin, pout = A.pout, nlat = pin + 1, nlon = 2 * pin, nf = 2 * pout, nc = ncoef(pout);
  std::vector<double> F((size_t)nlat * nf);
  std::vector<int> jf(nc);
  {
    int c = 0;
    for (int j = 0; j < 2 * pout; j++)
      for (int n = (j + 1) / 2; n <= pout; n++) jf[c++] = j;
  }
  for (long f = 0; f < nfun; f++) {
    const double* x = X + (size_t)f * nlat * nlon;
    for (int i = 0; i < nlat; i++)
      for (int k = 0; k < nf; k++) {
        double s = 0;
        for (int j = 0; j < nlon; j++) s += x[i * nlon + j] * A.four[(size_t)j * nf + k];
        F[(size_t)i * nf + k] = s;
      }
    for (int c = 0; c < nc; c++) {
      double s = 0;
      for (int i = 0; i < nlat; i++) s += F[(size_t)i * nf + jf[c]] * A.leg[(size_t)c * nlat + i];
      S[(size_t)f * nc + c] = s;
    }
  }
}

void pole_table(int p0, std::vector<double>& qp) {
  const double s2p = std::sqrt(2.0 * kPi);
  const double xm[2] = {-1.0, 1.0};
  std::vector<double> alp((size_t)(p0 + 1) * (p0 + 2) / 2);
  qp.assign((size_t)2 * (p0 + 1), 0.0);
  for (int t = 0; t < 2; t++) {
    legpoly(&xm[t], nullptr, 1, p0, alp.data());
    for (int n = 0; n <= p0; n++) qp[(size_t)t * (p0 + 1) + n] = alp[n] * s2p;
  }
}

void build_tables(int p0, int p1, ShTables& T) {
  T.p0 = p0;
  T.p1 = p1;
  gauss_legendre(p0 + 1, T.x0, T.w0);
  gauss_legendre(p1 + 1, T.x1, T.w1);
  const int nc = ncoef(p0), ng = ngrid(p0);

  T.jf_of_coef.assign(nc, 0);
  T.m_of_coef.assign(nc, 0);
  T.n_of_coef.assign(nc, 0);
  T.partner.assign(nc, -1);
  T.is_sin.assign(nc, 0);
  T.blk_off.assign(2 * p0 + 1, 0);
  {
    int c = 0;
    for (int jf = 0; jf < 2 * p0; jf++) {
      T.blk_off[jf] = c;
      int m = (jf + 1) / 2;
      for (int n = m; n <= p0; n++, c++) {
        T.jf_of_coef[c] = jf;
        T.m_of_coef[c] = m;
        T.n_of_coef[c] = n;
      }
    }
    T.blk_off[2 * p0] = c;
    // cos block of m (0<m<p0) is jf = 2m-1, sin block is jf = 2m, same length.
    for (int m = 1; m < p0; m++) {
      int cb = T.blk_off[2 * m - 1], sb = T.blk_off[2 * m], len = p0 + 1 - m;
      for (int k = 0; k < len; k++) {
        T.partner[cb + k] = sb + k;
        T.partner[sb + k] = cb + k;
        T.is_sin[sb + k] = 1;
      }
    }
  }

  build_analysis(p0, p0, T.ana);
  // (second-derivative Legendre table filled below, once degrees are known)
  build_synth(p0, p0, T.x0, T.syn0);
  // P_uu = cot(theta) P_u - (n(n+1) - m^2 / sin^2 theta) P from the associated Legendre
  // equation; P_u = syn0.dleg is the latitude derivative (-d/dtheta).
  T.syn0_d2leg.assign((size_t)nc * (p0 + 1), 0.0);
  T.syn0_d2four.assign((size_t)4 * p0 * p0, 0.0);
  {
    const double s2p = std::sqrt(2.0 * kPi);
    for (int j = 0; j < 2 * p0; j++) {
      for (int k = 1; k < p0; k++) {
        T.syn0_d2four[(size_t)(2 * k - 1) * 2 * p0 + j] = -s2p * k * k * std::cos(j * k * kPi / p0);
        T.syn0_d2four[(size_t)(2 * k) * 2 * p0 + j] = -s2p * k * k * std::sin(j * k * kPi / p0);
      }
      T.syn0_d2four[(size_t)(2 * p0 - 1) * 2 * p0 + j] = -s2p * p0 * p0 * std::cos(j * p0 * kPi / p0);
    }
  }
  build_synth(p0, p1, T.x1, T.syn1);
  // SHC2GridTranspose(., p1, p0): Fourier = MatFourier(p0,p1)^T, Legendre = MatLegendre(p0,p1)^T.
  T.synT.pin = p1;
  T.synT.pout = p0;
  T.synT.four.assign((size_t)4 * p0 * p1, 0.0);
  for (int r = 0; r < 2 * p0; r++)
    for (int c = 0; c < 2 * p1; c++) T.synT.four[(size_t)c * 2 * p0 + r] = T.syn1.four[(size_t)r * 2 * p1 + c];
  T.synT.leg = T.syn1.leg;  // [Ncoef0][p1+1]

  for (int c = 0; c < nc; c++) {
    const int m = T.m_of_coef[c], n = T.n_of_coef[c];
    for (int i = 0; i <= p0; i++) {
      const double x = T.x0[i], sn = std::sqrt(1.0 - x * x);
      const size_t o = (size_t)c * (p0 + 1) + i;
      T.syn0_d2leg[o] = (x / sn) * T.syn0.dleg[o] - (n * (n + 1.0) - (double)(m * m) / (sn * sn)) * T.syn0.leg[o];
    }
  }

  // coeff_perm (:365-376)
  std::vector<std::vector<int>> perm(p0 + 1);
  for (int n = 0; n <= p0; n++) perm[n].assign(std::min(2 * n + 1, 2 * p0), 0);
  {
    int itr = 0;
    for (int i = 0; i < 2 * p0; i++) {
      int m = (i + 1) / 2;
      for (int n = m; n <= p0; n++) perm[n][i] = itr++;
    }
  }
  T.perm.clear();
  T.perm_off.assign(p0 + 2, 0);
  T.pos_in_block.assign(nc, 0);
  for (int n = 0; n <= p0; n++) {
    T.perm_off[n] = (int)T.perm.size();
    for (size_t b = 0; b < perm[n].size(); b++) {
      T.perm.push_back(perm[n][b]);
      T.pos_in_block[perm[n][b]] = (int)b;
    }
  }
  T.perm_off[p0 + 1] = (int)T.perm.size();

  // Rotation blocks (src/SphericalHarmonics.cc:760-860) with sin(theta) of each rotated
  // grid point taken as hypot(y, z): the reference's sqrt(1 - x^2) turns the ~1e-16
  // rounding of x at rotated points that land on a pole into ~1e-8 noise.
  const double s2p = std::sqrt(2.0 * kPi);
  std::vector<double> c0((size_t)3 * ng), c1((size_t)3 * ng), ucol(ng), theta(ng);
  for (int i = 0; i <= p0; i++)
    for (int j = 0; j < 2 * p0; j++) {
      int k = i * 2 * p0 + j;
      double s = std::sqrt(1.0 - T.x0[i] * T.x0[i]);
      c0[k] = T.x0[i];
      c0[ng + k] = s * std::sin(kPi * j / p0);
      c0[2 * ng + k] = s * std::cos(kPi * j / p0);
    }
  size_t na = (size_t)(p0 + 1) * (p0 + 2) / 2;
  std::vector<double> mleg(na * ng), m2g((size_t)nc * ng), c2c((size_t)nc * nc);
  T.mr.clear();
  T.mr_off.assign((size_t)(p0 + 1) * (p0 + 1), 0);
  for (int l = 0; l <= p0; l++) {
    double cs = -T.x0[l], sn = -std::sqrt(1.0 - T.x0[l] * T.x0[l]);
    for (int k = 0; k < ng; k++) {
      double a = c0[k], b = c0[ng + k], c = c0[2 * ng + k];
      c1[k] = cs * a - sn * c;
      c1[ng + k] = b;
      c1[2 * ng + k] = sn * a + cs * c;
      ucol[k] = std::hypot(c1[ng + k], c1[2 * ng + k]);
      theta[k] = std::atan2(c1[ng + k], c1[2 * ng + k]);
    }
    legpoly(c1.data(), ucol.data(), ng, p0, mleg.data());
    size_t o0 = 0, o1 = 0;
    for (int m = 0; m <= p0; m++) {
      int len = p0 + 1 - m;
      for (int jj = 0; jj < len; jj++)
        for (int k = 0; k < ng; k++)
          m2g[(o1 + jj) * ng + k] = s2p * mleg[(o0 + jj) * ng + k] * std::cos(m * theta[k]);
      o1 += len;
      if (m != 0 && m != p0) {
        for (int jj = 0; jj < len; jj++)
          for (int k = 0; k < ng; k++)
            m2g[(o1 + jj) * ng + k] = s2p * mleg[(o0 + jj) * ng + k] * std::sin(m * theta[k]);
        o1 += len;
      }
      o0 += len;
    }
    host_grid2shc(T.ana, m2g.data(), nc, c2c.data());
    for (int n = 0; n <= p0; n++) {
      T.mr_off[(size_t)l * (p0 + 1) + n] = (int)T.mr.size();
      const std::vector<int>& pn = perm[n];
      for (size_t a = 0; a < pn.size(); a++)
        for (size_t b = 0; b < pn.size(); b++) T.mr.push_back(c2c[(size_t)pn[a] * nc + pn[b]]);
    }
  }

  // SingularWeights(p1) (:573-604)
  {
    size_t na1 = (size_t)(p1 + 1) * (p1 + 2) / 2;
    std::vector<double> alp0(na1), alp(na1 * (p1 + 1));
    double one = 1.0;
    legpoly(&one, nullptr, 1, p1, alp0.data());
    legpoly(T.x1.data(), nullptr, p1 + 1, p1, alp.data());
    T.sing_w.assign(p1 + 1, 0.0);
    for (int i = 0; i <= p1; i++) {
      double yf = 0;
      for (int j = 0; j <= p1; j++) yf += 4.0 * kPi / (2 * j + 1) * alp0[j] * alp[(size_t)j * (p1 + 1) + i];
      T.sing_w[i] = (T.w1[i] * kPi / p1) * yf / std::cos(std::acos(T.x1[i]) / 2.0);
    }
  }
  T.smooth_w0.assign(p0 + 1, 0.0);
  for (int i = 0; i <= p0; i++) T.smooth_w0[i] = T.w0[i] * kPi / p0 / std::sqrt(1.0 - T.x0[i] * T.x0[i]);
  pole_table(p0, T.qp);
  T.cos_tab.assign(2 * p0, 0.0);
  T.sin_tab.assign(2 * p0, 0.0);
  for (int q = 0; q < 2 * p0; q++) {
    T.cos_tab[q] = std::cos(q * kPi / p0);
    T.sin_tab[q] = std::sin(q * kPi / p0);
  }
}

}  // namespace ves3d
