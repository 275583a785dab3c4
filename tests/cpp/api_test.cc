// C++ caller of the B200 path through include/ves3d_b200.hpp, written the way Ves3D's
// C++ code uses StokesVelocity<Real> (SetSrcCoord / SetDensitySL / operator()).
//   api_test --version            prints the library version (no GPU needed)
//   api_test --filter p f e       prints SHTrans's two filters (no GPU needed)
//   api_test <in.bin> <out.bin>   in: int32 p, int32 n_ves, X[n], f[n] (doubles, AxisMajor);
//                                 out: vel[n] then the implicit solution x[4 n / 3]
//   api_test --vtk <in.bin> p1 f  WriteVTK of in.bin's surfaces (field: its f) at order p1
//                                 into f_000000.vtp and f.pvtp
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ves3d_b200.hpp"

// in.bin: int32 p, int32 n_ves, X[n], f[n] (doubles, AxisMajor); false on a short file
static bool read_input(const char* path, int& p, int& nv, std::vector<double>& X, std::vector<double>& f) {
  std::FILE* fi = std::fopen(path, "rb");
  if (!fi) return false;
  int hdr[2];
  bool ok = std::fread(hdr, sizeof(int), 2, fi) == 2;
  if (ok) {
    p = hdr[0];
    nv = hdr[1];
    const size_t n = (size_t)nv * 3 * 2 * p * (p + 1);
    X.resize(n);
    f.resize(n);
    ok = std::fread(&X[0], sizeof(double), n, fi) == n && std::fread(&f[0], sizeof(double), n, fi) == n;
  }
  std::fclose(fi);
  return ok;
}

int main(int argc, char** argv) {
  if (argc == 2 && std::strcmp(argv[1], "--version") == 0) {
    // instantiate the device-pointer members of the SHTrans mirror (a compile check)
    typedef ves3d_b200::SHTrans<double> Sht;
    void (Sht::*d2[4])(const double*, long, double*) const = {&Sht::backward_d2u, &Sht::backward_d2v,
                                                                &Sht::backward_duv, &Sht::SHC2Pole};
    (void)d2;
    typedef ves3d_b200::StokesVelocity<double> Sv;
    double (Sv::*monitor)(double) = &Sv::MonitorError;
    void (Sv::*set_trg)(const double*, long, bool) = &Sv::SetTrgCoord;
    void (Sv::*eval_trg)(double*, bool) = &Sv::EvalTrg;
    (void)monitor;
    (void)set_trg;
    (void)eval_trg;
    std::printf("%d\n", ves3d_version());
    return 0;
  }
  if (argc == 5 && std::strcmp(argv[1], "--filter") == 0) {
    // SHTrans filters on the host: p, filter_freq, exponent -> hard and polynomial rows
    ves3d_b200::SHTrans<double> sht(std::atoi(argv[2]), 0, std::atoi(argv[3]), std::atof(argv[4]));
    std::vector<double> hard, poly;
    sht.filterCoeffs(hard, poly);
    for (size_t i = 0; i < hard.size(); i++) std::printf("%.17g%c", hard[i], i + 1 < hard.size() ? ' ' : '\n');
    for (size_t i = 0; i < poly.size(); i++) std::printf("%.17g%c", poly[i], i + 1 < poly.size() ? ' ' : '\n');
    std::printf("%d %.17g\n", sht.getShFilterFreq(), sht.getShFilterExponent());
    return 0;
  }
  if (argc == 5 && std::strcmp(argv[1], "--vtk") == 0) {
    int p = 0, nv = 0;
    std::vector<double> X, f;
    if (!read_input(argv[2], p, nv, X, f)) return 3;
    try {
      ves3d_b200::WriteVTK(X, p, std::atoi(argv[3]), argv[4], 0.0, &f);
    } catch (const ves3d_b200::Error& e) {
      std::fprintf(stderr, "%s\n", e.what());
      return 1;
    }
    return 0;
  }
  if (argc != 3) {
    std::fprintf(stderr, "usage: api_test --version | api_test in.bin out.bin\n");
    return 2;
  }
  int p = 0, nv = 0;
  std::vector<double> X, f;
  if (!read_input(argv[1], p, nv, X, f)) return 3;
  const size_t n = X.size();
  std::vector<double> vel(n), x(4 * n / 3);
  try {
    ves3d_b200::StokesVelocity<double> stokes(p, 2 * p);
    stokes.SetSrcCoord(X);
    stokes.SetDensitySL(&f);
    stokes(vel);
    stokes.SetDensityDL((const std::vector<double>*)0);  // InterfacialVelocity's call without contrast
    // the reference's implicit step on the same surfaces, self-block preconditioned
    stokes.SetViscosityContrast((const double*)0, 0);  // no contrast
    stokes.SetImplicitParams(0.01, 0.05, 1.0);
    stokes.SetPrecond(VES3D_PRECOND_SELF_BLOCK);
    double tol = 1e-9;
    int iters = 500;
    const int code = stokes.ImplicitSolve(0, &x[0], tol, iters);
    std::fprintf(stderr, "implicit: code %d, %d iterations, relres %.3e\n", code, iters, tol);
    if (code != 100) return 4;
  } catch (const ves3d_b200::Error& e) {
    std::fprintf(stderr, "error %d: %s\n", e.status(), e.what());
    return 5;
  }
  std::FILE* fo = std::fopen(argv[2], "wb");
  if (!fo) return 3;
  std::fwrite(&vel[0], sizeof(double), n, fo);
  std::fwrite(&x[0], sizeof(double), x.size(), fo);
  std::fclose(fo);
  return 0;
}
