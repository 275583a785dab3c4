// Test infrastructure only: the reference's own Streamable ASCII writer and reader
// (Array / Scalars / Vectors pack and unpack, src/Array.cc:107-165, src/Scalars.cc:220-285,
// src/Vectors.cc:86-130), compiled from the reference's sources in place, for the golden
// fixtures and the round-trip tests of the interchange reader/writer. Never part of the
// product path.
//   ref_stream pack <p> <n_vec> <out>   a Vectors (AxisMajor, name "position") and a Scalars
//                                       (name "tension") of fixed values, written as the
//                                       reference's checkpoints write (scientific, 16 digits)
//   ref_stream vectors <in> <out>       unpack a VECTORS block, pack it again
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>

#include "Device.h"
#include "Scalars.h"
#include "Vectors.h"

// BLAS / LAPACK symbols that Device<CPU> refers to; this driver never reaches them
extern "C" {
void sgemm_(const char*, const char*, const int*, const int*, const int*, const float*, const float*, const int*,
            const float*, const int*, const float*, float*, const int*) {
  std::abort();
}
void dgemm_(const char*, const char*, const int*, const int*, const int*, const double*, const double*, const int*,
            const double*, const int*, const double*, double*, const int*) {
  std::abort();
}
void ssteqr_(char*, const int*, float*, float*, float*, const int*, float*, const int*) { std::abort(); }
void dsteqr_(char*, const int*, double*, double*, double*, const int*, double*, const int*) { std::abort(); }
}

typedef Device<CPU> DevCPU;
extern const DevCPU the_cpu_device(0);
typedef Scalars<double, DevCPU, the_cpu_device> Sca;
typedef Vectors<double, DevCPU, the_cpu_device> Vec;

int main(int argc, char** argv) {
  if (argc == 5 && std::string(argv[1]) == "pack") {
    const int p = std::atoi(argv[2]), nv = std::atoi(argv[3]);
    Vec x(nv, p);
    x.set_name("position");
    for (size_t i = 0; i < x.size(); i++) x.begin()[i] = std::sin(0.37 * i) + 1e-3 * i;
    Sca s(nv, p);
    s.set_name("tension");
    for (size_t i = 0; i < s.size(); i++) s.begin()[i] = std::cos(0.11 * i) / (1.0 + i);
    std::ofstream out(argv[4]);
    out << std::scientific << std::setprecision(16);
    x.pack(out, Streamable::ASCII);
    s.pack(out, Streamable::ASCII);
    return out.good() ? 0 : 3;
  }
  if (argc == 4 && std::string(argv[1]) == "vectors") {
    std::ifstream in(argv[2]);
    Vec x;
    if (x.unpack(in, Streamable::ASCII) != ErrorEvent::Success) return 4;
    std::ofstream out(argv[3]);
    out << std::scientific << std::setprecision(16);
    x.pack(out, Streamable::ASCII);
    return out.good() ? 0 : 3;
  }
  std::fprintf(stderr, "usage: ref_stream pack <p> <n_vec> <out> | vectors <in> <out>\n");
  return 2;
}
