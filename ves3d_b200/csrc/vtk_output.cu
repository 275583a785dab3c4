// VTK PolyData output of vesicle surfaces in the reference's layout (WriteVTK,
// src/StokesVelocity.cc:773-993), so that ParaView files of a run look the same whichever
// code wrote them. The mesh and the file are built on the host; ves3d_vtk_write first takes
// the surfaces to the output order on the GPU with this library's transforms.
//
// Per vesicle: the (p1+1) x 2p1 grid points, latitude-major, then the poles at x = -1 and
// x = +1 (SHC2Pole); 2p1 pairs of triangles (x = -1 pole with latitude row 0, x = +1 pole
// with row p1), then p1 x 2p1 quads (i, j), (i+1, j), (i+1, j+1), (i, j+1), longitudes
// wrapping. The file is XML PolyData with one raw appended block per array, each led by its
// byte count as an int32.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "common.cuh"
#include "sh_tables.h"

namespace ves3d {
namespace {

struct Mesh {
  std::vector<double> coord, value;
  std::vector<int32_t> connect, offset;
};

// Points (recentred by the nearest multiple of period when period > 0), point values, and
// polygons, exactly in the reference's order (src/StokesVelocity.cc:800-876).
void build_mesh(const double* X1, const double* Xp, const double* V1, const double* Vp, long n_ves, int p1,
                double period, Mesh& M) {
  const long ng = 2L * p1 * (p1 + 1), npt = ng + 2;
  M.coord.resize((size_t)(n_ves * npt * 3));
  for (long k = 0; k < n_ves; k++) {
    double C[3] = {0.0, 0.0, 0.0};
    if (period > 0) {
      for (int l = 0; l < 3; l++) {
        const double* x = X1 + (k * 3 + l) * ng;
        for (long g = 0; g < ng; g++) C[l] += x[g];
        C[l] += Xp[(k * 3 + l) * 2 + 0];
        C[l] += Xp[(k * 3 + l) * 2 + 1];
        C[l] /= (double)npt;
        C[l] = std::round(C[l] / period) * period;  // halves away from zero, as C's round()
      }
    }
    double* out = &M.coord[(size_t)(k * npt * 3)];
    for (long g = 0; g < ng; g++)
      for (int l = 0; l < 3; l++) out[g * 3 + l] = X1[(k * 3 + l) * ng + g] - C[l];
    for (int t = 0; t < 2; t++)
      for (int l = 0; l < 3; l++) out[(ng + t) * 3 + l] = Xp[(k * 3 + l) * 2 + t] - C[l];
  }
  if (V1 && Vp && n_ves > 0) {
    M.value.resize(M.coord.size());
    for (long k = 0; k < n_ves; k++) {
      double* out = &M.value[(size_t)(k * npt * 3)];
      for (long g = 0; g < ng; g++)
        for (int l = 0; l < 3; l++) out[g * 3 + l] = V1[(k * 3 + l) * ng + g];
      for (int t = 0; t < 2; t++)
        for (int l = 0; l < 3; l++) out[(ng + t) * 3 + l] = Vp[(k * 3 + l) * 2 + t];
    }
  }
  // one vesicle's polygons relative to its first point, then shifted per vesicle
  std::vector<int32_t> con, off;
  const int lon = 2 * p1;
  auto close_poly = [&]() { off.push_back((int32_t)con.size()); };
  for (int j = 0; j < lon; j++) {
    const int j1 = (j + 1) % lon;
    con.push_back((int32_t)ng);
    con.push_back(j);
    con.push_back(j1);
    close_poly();
    con.push_back((int32_t)ng + 1);
    con.push_back(lon * p1 + j);
    con.push_back(lon * p1 + j1);
    close_poly();
  }
  for (int i = 0; i < p1; i++)
    for (int j = 0; j < lon; j++) {
      const int j1 = (j + 1) % lon;
      con.push_back(lon * i + j);
      con.push_back(lon * (i + 1) + j);
      con.push_back(lon * (i + 1) + j1);
      con.push_back(lon * i + j1);
      close_poly();
    }
  M.connect.resize(con.size() * (size_t)n_ves);
  M.offset.resize(off.size() * (size_t)n_ves);
  for (long k = 0; k < n_ves; k++) {
    for (size_t i = 0; i < con.size(); i++) M.connect[k * con.size() + i] = (int32_t)(k * npt) + con[i];
    for (size_t i = 0; i < off.size(); i++) M.offset[k * off.size() + i] = (int32_t)(k * con.size()) + off[i];
  }
}

template <class T>
void write_block(std::ofstream& f, const std::vector<T>& v) {
  const int32_t bytes = (int32_t)(v.size() * sizeof(T));
  f.write((const char*)&bytes, sizeof(int32_t));
  if (!v.empty()) f.write((const char*)v.data(), (std::streamsize)(v.size() * sizeof(T)));
}

bool little_endian() {
  const uint16_t one = 1;
  unsigned char b;
  std::memcpy(&b, &one, 1);
  return b == 1;
}

std::string piece_name(const std::string& base, int rank) {
  char buf[16];
  std::snprintf(buf, sizeof(buf), "_%06d.vtp", rank);
  return base + buf;
}

int write_piece(const std::string& path, const Mesh& M) {
  const long pt_cnt = (long)(M.coord.size() / 3), poly_cnt = (long)M.offset.size();
  std::ofstream f(path.c_str(), std::ios::out | std::ios::binary | std::ios::trunc);
  if (!f) {
    set_error("cannot open %s for writing", path.c_str());
    return VES3D_ERR_IO;
  }
  size_t data = 0;
  std::ostringstream h;
  h << "<?xml version=\"1.0\"?>\n";
  h << "<VTKFile type=\"PolyData\" version=\"0.1\" byte_order=\"" << (little_endian() ? "LittleEndian" : "BigEndian")
    << "\">\n";
  h << "  <PolyData>\n";
  h << "    <Piece NumberOfPoints=\"" << pt_cnt
    << "\" NumberOfVerts=\"0\" NumberOfLines=\"0\" NumberOfStrips=\"0\" NumberOfPolys=\"" << poly_cnt << "\">\n";
  h << "      <Points>\n";
  h << "        <DataArray type=\"Float64\" NumberOfComponents=\"3\" Name=\"Position\" format=\"appended\" offset=\""
    << data << "\" />\n";
  data += sizeof(uint32_t) + M.coord.size() * sizeof(double);
  h << "      </Points>\n";
  if (!M.value.empty()) {
    h << "      <PointData>\n";
    h << "        <DataArray type=\"Float64\" NumberOfComponents=\"" << M.value.size() / pt_cnt
      << "\" Name=\"value\" format=\"appended\" offset=\"" << data << "\" />\n";
    data += sizeof(uint32_t) + M.value.size() * sizeof(double);
    h << "      </PointData>\n";
  }
  h << "      <Polys>\n";
  h << "        <DataArray type=\"Int32\" Name=\"connectivity\" format=\"appended\" offset=\"" << data << "\" />\n";
  data += sizeof(uint32_t) + M.connect.size() * sizeof(int32_t);
  h << "        <DataArray type=\"Int32\" Name=\"offsets\" format=\"appended\" offset=\"" << data << "\" />\n";
  h << "      </Polys>\n";
  h << "    </Piece>\n";
  h << "  </PolyData>\n";
  h << "  <AppendedData encoding=\"raw\">\n";
  h << "    _";
  const std::string head = h.str();
  f.write(head.data(), (std::streamsize)head.size());
  write_block(f, M.coord);
  if (!M.value.empty()) write_block(f, M.value);
  write_block(f, M.connect);
  write_block(f, M.offset);
  const char tail[] = "\n  </AppendedData>\n</VTKFile>\n";
  f.write(tail, (std::streamsize)(sizeof(tail) - 1));
  f.close();
  if (!f) {
    set_error("writing %s failed", path.c_str());
    return VES3D_ERR_IO;
  }
  return VES3D_OK;
}

// the index file rank 0 writes: one piece per rank, named without the directory part
int write_index(const std::string& base, int n_ranks, bool has_value) {
  const std::string path = base + ".pvtp";
  std::ofstream f(path.c_str(), std::ios::out | std::ios::trunc);
  if (!f) {
    set_error("cannot open %s for writing", path.c_str());
    return VES3D_ERR_IO;
  }
  const size_t slash = base.find_last_of("/\\");
  const std::string name = slash == std::string::npos ? base : base.substr(slash + 1);
  f << "<?xml version=\"1.0\"?>\n";
  f << "<VTKFile type=\"PPolyData\">\n";
  f << "  <PPolyData GhostLevel=\"0\">\n";
  f << "      <PPoints>\n";
  f << "        <PDataArray type=\"Float64\" NumberOfComponents=\"3\" Name=\"Position\"/>\n";
  f << "      </PPoints>\n";
  if (has_value) {
    f << "      <PPointData>\n";
    f << "        <PDataArray type=\"Float64\" NumberOfComponents=\"3\" Name=\"value\"/>\n";
    f << "      </PPointData>\n";
  }
  for (int i = 0; i < n_ranks; i++) f << "      <Piece Source=\"" << piece_name(name, i) << "\"/>\n";
  f << "  </PPolyData>\n";
  f << "</VTKFile>\n";
  f.close();
  if (!f) {
    set_error("writing %s failed", path.c_str());
    return VES3D_ERR_IO;
  }
  return VES3D_OK;
}

// device buffer released on scope exit
struct DevBuf {
  double* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  int alloc(size_t n) {
    if (n) VES3D_CK(cudaMalloc((void**)&p, n * sizeof(double)));
    return VES3D_OK;
  }
};

// nf grid functions at order p0 (host or device) -> host grid values at order p1 and host
// pole values [nf][2], through Grid2SHC(p0, p0), SHC2Grid(p0, p1) and SHC2Pole on the GPU
int to_order(const double* in, long nf, int p0, int p1, int is_device, double* grid, double* pole) {
  cudaStream_t st = nullptr;
  DevBuf din, coef, dgrid, dpole;
  const double* src = in;
  int s;
  if (!is_device) {
    if ((s = din.alloc((size_t)nf * ngrid(p0)))) return s;
    VES3D_CK(cudaMemcpy(din.p, in, (size_t)nf * ngrid(p0) * sizeof(double), cudaMemcpyHostToDevice));
    src = din.p;
  }
  if ((s = coef.alloc((size_t)nf * ncoef(p0))) || (s = dgrid.alloc((size_t)nf * ngrid(p1))) ||
      (s = dpole.alloc((size_t)nf * 2)))
    return s;
  if ((s = ves3d_sht_forward(src, nf, p0, p0, coef.p, st))) return s;
  if ((s = ves3d_sht_backward(coef.p, nf, p0, p1, dgrid.p, nullptr, nullptr, st))) return s;
  if ((s = ves3d_sht_pole(coef.p, nf, p0, dpole.p, st))) return s;
  VES3D_CK(cudaMemcpy(grid, dgrid.p, (size_t)nf * ngrid(p1) * sizeof(double), cudaMemcpyDeviceToHost));
  VES3D_CK(cudaMemcpy(pole, dpole.p, (size_t)nf * 2 * sizeof(double), cudaMemcpyDeviceToHost));
  return VES3D_OK;
}

}  // namespace
}  // namespace ves3d

using namespace ves3d;

extern "C" {

int ves3d_vtk_write_grid(const double* X1, const double* Xp, const double* V1, const double* Vp, long n_ves, int p1,
                         const char* fname, double period, int rank, int n_ranks) {
  VES3D_ARG(fname != nullptr && fname[0] != 0, "file name is empty");
  VES3D_ARG(n_ves >= 0, "n_ves < 0");
  VES3D_ARG(n_ves == 0 || (X1 && Xp), "null positions");
  VES3D_ARG((V1 == nullptr) == (Vp == nullptr), "V1 and Vp go together");
  VES3D_ARG(p1 >= 1 && p1 <= 256, "order must be in [1, 256]");
  VES3D_ARG(n_ranks >= 1 && rank >= 0 && rank < n_ranks && n_ranks <= 999999, "rank out of range");
  VES3D_ARG(std::isfinite(period), "period is not finite");
  const double npt = (2.0 * p1 * (p1 + 1) + 2.0) * (double)n_ves;
  // raw blocks carry an int32 byte count and polygons int32 point indices
  VES3D_ARG(npt * 3 * sizeof(double) < 2147483647.0, "too many points for one VTK piece");
  Mesh M;
  build_mesh(X1, Xp, V1, Vp, n_ves, p1, period, M);
  const std::string base(fname);
  int s = write_piece(piece_name(base, rank), M);
  if (s || rank != 0) return s;
  return write_index(base, n_ranks, !M.value.empty());
}

int ves3d_vtk_write(const double* X, const double* V, long n_ves, int p0, int p1, const char* fname, double period,
                    int rank, int n_ranks, int is_device) {
  VES3D_ARG(fname != nullptr && fname[0] != 0, "file name is empty");
  VES3D_ARG(n_ves >= 0, "n_ves < 0");
  VES3D_ARG(n_ves == 0 || X, "null positions");
  VES3D_ARG(p0 >= 1 && p0 <= 128 && p1 >= 1 && p1 <= 128, "orders must be in [1, 128]");
  VES3D_ARG(n_ranks >= 1 && rank >= 0 && rank < n_ranks && n_ranks <= 999999, "rank out of range");
  VES3D_ARG((2.0 * p1 * (p1 + 1) + 2.0) * n_ves * 3 * sizeof(double) < 2147483647.0,
            "too many points for one VTK piece");
  NvtxRange nv("ves3d vtk");
  const long nf = 3 * n_ves;
  std::vector<double> X1((size_t)nf * ngrid(p1)), Xp((size_t)nf * 2), V1, Vp;
  int s;
  if (n_ves > 0 && (s = to_order(X, nf, p0, p1, is_device, X1.data(), Xp.data()))) return s;
  if (V) {
    V1.resize(X1.size());
    Vp.resize(Xp.size());
    if (n_ves > 0 && (s = to_order(V, nf, p0, p1, is_device, V1.data(), Vp.data()))) return s;
  }
  return ves3d_vtk_write_grid(X1.data(), Xp.data(), V ? V1.data() : nullptr, V ? Vp.data() : nullptr, n_ves, p1,
                              fname, period, rank, n_ranks);
}

}  // extern "C"
