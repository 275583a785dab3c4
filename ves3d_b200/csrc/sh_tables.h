// Host-side spherical-harmonic operator tables for one (p0, p1) pair, built in FP64.
//
// The math is that of the reference's SphericalHarmonics<Real> matrices
// (src/SphericalHarmonics.cc:544-860): Gauss-Legendre nodes, normalised associated
// Legendre functions and their theta-derivatives, the DFT matrices of SHC2Grid /
// Grid2SHC, the pole-singular quadrature weights and the per-degree rotation blocks.
// Layouts are flattened for the GPU kernels (see each member).
#pragma once
#include <vector>

namespace ves3d {

inline int ncoef(int p) { return p * (p + 2); }
inline int ngrid(int p) { return 2 * p * (p + 1); }

// Gauss-Legendre rule on [-1, 1], nodes ascending (the reference's cgqf(n, 1, 0, 0, -1, 1),
// src/legendre_rule.cc:269; computed here by Newton iteration on P_n).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w);

// Normalised associated Legendre functions up to `degree` at N points, m-major layout
// [(m=0,n=0..d), (m=1,n=1..d), ...][N] (src/SphericalHarmonics.cc:889-928). If u is
// given it is sin(theta) at each point, otherwise sqrt(1-x^2).
void legpoly(const double* x, const double* u, int N, int degree, double* out);
// theta-derivative (src/SphericalHarmonics.cc:931-950).
void legpoly_deriv(const double* x, int N, int degree, double* out);

// Synthesis tables: coefficients at order p0 -> grid at order q (SHC2Grid(p0, q)).
struct SynthTables {
  int p0 = 0, q = 0;
  std::vector<double> leg;    // [Ncoef0][q+1]   P_n^m(x_q[lat])
  std::vector<double> dleg;   // [Ncoef0][q+1]   d/dtheta
  std::vector<double> four;   // [2p0][2q]       MatFourier(p0, q)
  std::vector<double> dfour;  // [2p0][2q]       MatFourierGrad(p0, q)
};

// Analysis tables: grid at order pin -> coefficients at order pout (Grid2SHC(pin, pout)).
struct AnalysisTables {
  int pin = 0, pout = 0;
  std::vector<double> four;   // [2pin][2pout]  MatFourierInv(pin, pout)
  std::vector<double> leg;    // [Ncoef_out][pin+1]  P_n^m(x_pin[lat]) w[lat] 2pi
};

struct ShTables {
  int p0 = 0, p1 = 0;
  std::vector<double> x0, w0, x1, w1;  // Gauss-Legendre rules with p0+1 and p1+1 nodes
  std::vector<int> jf_of_coef;         // [Ncoef0] Fourier index of each coefficient
  std::vector<int> blk_off;            // [2p0+1]  coefficient offset of each Fourier block
  std::vector<int> m_of_coef;          // [Ncoef0]
  std::vector<int> n_of_coef;          // [Ncoef0] degree
  std::vector<int> partner;            // [Ncoef0] cos<->sin partner coefficient, -1 if none
  std::vector<int> is_sin;             // [Ncoef0]
  AnalysisTables ana;                  // Grid2SHC(p0, p0)
  SynthTables syn0;                    // SHC2Grid(p0, p0)
  SynthTables syn1;                    // SHC2Grid(p0, p1)
  // Second derivatives at order p0 (Surface curvatures, src/Surface.cc:264-323):
  std::vector<double> syn0_d2leg;      // [Ncoef0][p0+1] d^2/du^2 of P_n^m at the p0 nodes (u = latitude)
  std::vector<double> syn0_d2four;     // [2p0][2p0]     d^2/dv^2 of MatFourier(p0, p0)
  // Transpose of SHC2Grid(p0, p1), used as an analysis-like map p1 grid -> p0 coefficients
  // (SHC2GridTranspose(., p1, p0), src/SphericalHarmonics.cc:238-322).
  AnalysisTables synT;
  // Rotation blocks Mr[t][n] (src/SphericalHarmonics.cc:760-860), t = 0..p0, n = 0..p0,
  // each bn x bn with bn = min(2n+1, 2p0), row-major, concatenated in (t, n) order.
  std::vector<double> mr;
  std::vector<int> mr_off;             // [(p0+1)*(p0+1)] offset of block (t, n)
  std::vector<int> perm;               // concatenated coeff_perm[n][b] (:365-376)
  std::vector<int> perm_off;           // [p0+2]
  std::vector<int> pos_in_block;       // [Ncoef0] b such that perm[n][b] == coef
  std::vector<double> sing_w;          // [p1+1] SingularWeights(p1) (:573-604)
  std::vector<double> smooth_w0;       // [p0+1] LegendreWeights(p0) (:558-570)
  std::vector<double> qp;              // [2][p0+1] pole evaluation at x = -1, +1 (:325-360)
  std::vector<double> cos_tab, sin_tab;// [2p0] cos/sin(q pi / p0)
};

void build_tables(int p0, int p1, ShTables& T);
// SHC2Pole's weights (src/SphericalHarmonics.cc:325-338): [2][p0+1], the m = 0 block's
// normalised Legendre functions times sqrt(2 pi) at x = -1 (row 0) and x = +1 (row 1).
void pole_table(int p0, std::vector<double>& qp);

// Stand-alone transform tables for SHC2Grid(p0, q) and Grid2SHC(pin, pout).
void build_synth_tables(int p0, int q, SynthTables& S);
void build_analysis_tables(int pin, int pout, AnalysisTables& A);
// Fourier-block offsets of the order-p coefficient layout ([2p+1]) and the Fourier
// index of each coefficient ([Ncoef]).
void coef_blocks(int p, std::vector<int>& blk_off, std::vector<int>& jf_of_coef);

// Host reference transforms used while building tables.
void host_grid2shc(const AnalysisTables& A, const double* X, long nfun, double* S);

}  // namespace ves3d
