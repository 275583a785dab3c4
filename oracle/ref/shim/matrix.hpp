// Test infrastructure only (oracle build). A minimal, project-written stand-in for
// the pvfmm Vector/Matrix containers that the reference's SphericalHarmonics code is
// written against (pvfmm itself is not vendored with the reference and is unpinned;
// the reference only reads ${PVFMM_DIR}/MakeVariables, makefile.in.files/makefile.default:67-79).
//
// Semantics restated from the reference's call sites (src/SphericalHarmonics.cc,
// src/StokesVelocity.cc): row-major dense matrices, non-owning views via
// ReInit(n, ptr, false), operator[] returning a mutable reference even on const
// objects, and GEMM(C, A, B) meaning C = A * B with C preallocated.
#ifndef VES3D_ORACLE_PVFMM_MATRIX_SHIM_HPP
#define VES3D_ORACLE_PVFMM_MATRIX_SHIM_HPP

#include <cassert>
#include <cstring>
#include <cstdlib>
#include <algorithm>
#include <vector>
#include <omp.h>

#ifndef COORD_DIM
#define COORD_DIM 3
#endif

extern "C" {
void scipy_dgemm_(const char*, const char*, const int*, const int*, const int*,
                  const double*, const double*, const int*, const double*, const int*,
                  const double*, double*, const int*);
void scipy_sgemm_(const char*, const char*, const int*, const int*, const int*,
                  const float*, const float*, const int*, const float*, const int*,
                  const float*, float*, const int*);
}

namespace pvfmm {

namespace shim {
#ifdef VES3D_SHIM_NAIVE_GEMM
// Variant used to measure how much the reference's results depend on GEMM rounding
// order: plain i-k-j loops instead of OpenBLAS.
template <class T>
inline void gemm_rm(long m, long n, long k, const T* A, const T* B, T* C) {
  for (long i = 0; i < m; i++) {
    for (long j = 0; j < n; j++) C[i * n + j] = 0;
    for (long l = 0; l < k; l++) {
      T a = A[i * k + l];
      for (long j = 0; j < n; j++) C[i * n + j] += a * B[l * n + j];
    }
  }
}
#else
// Row-major C(m x n) = A(m x k) * B(k x n) through column-major BLAS: C^T = B^T A^T.
inline void gemm_rm(long m, long n, long k, const double* A, const double* B, double* C) {
  if (m <= 0 || n <= 0) return;
  if (k <= 0) { std::memset(C, 0, sizeof(double) * m * n); return; }
  int M = (int)n, N = (int)m, K = (int)k, lda = (int)n, ldb = (int)k, ldc = (int)n;
  double one = 1.0, zero = 0.0;
  scipy_dgemm_("N", "N", &M, &N, &K, &one, B, &lda, A, &ldb, &zero, C, &ldc);
}
inline void gemm_rm(long m, long n, long k, const float* A, const float* B, float* C) {
  if (m <= 0 || n <= 0) return;
  if (k <= 0) { std::memset(C, 0, sizeof(float) * m * n); return; }
  int M = (int)n, N = (int)m, K = (int)k, lda = (int)n, ldb = (int)k, ldc = (int)n;
  float one = 1.0f, zero = 0.0f;
  scipy_sgemm_("N", "N", &M, &N, &K, &one, B, &lda, A, &ldb, &zero, C, &ldc);
}
#endif
}  // namespace shim

template <class T>
class Vector {
 public:
  Vector() : dim_(0), data_(NULL), own_(true) {}
  explicit Vector(long n, T* ptr = NULL, bool own = true) : dim_(0), data_(NULL), own_(true) {
    ReInit(n, ptr, own);
  }
  Vector(const Vector& o) : dim_(0), data_(NULL), own_(true) { ReInit(o.dim_, o.data_, true); }
  Vector(const std::vector<T>& v) : dim_(0), data_(NULL), own_(true) {
    ReInit((long)v.size(), v.empty() ? NULL : (T*)&v[0], true);
  }
  ~Vector() { release(); }

  void ReInit(long n, T* ptr = NULL, bool own = true) {
    if (own) {
      T* fresh = n > 0 ? (T*)std::malloc(sizeof(T) * n) : NULL;
      if (ptr && n > 0) std::memcpy(fresh, ptr, sizeof(T) * n);
      else if (n > 0) std::memset(fresh, 0, sizeof(T) * n);
      release();
      data_ = fresh;
      dim_ = n;
      own_ = true;
    } else {
      release();
      data_ = ptr;
      dim_ = n;
      own_ = false;
    }
  }
  Vector& operator=(const Vector& o) {
    if (this == &o) return *this;
    if (dim_ != o.dim_) ReInit(o.dim_);
    if (dim_) std::memcpy(data_, o.data_, sizeof(T) * dim_);
    return *this;
  }
  Vector& operator=(const std::vector<T>& v) {
    if (dim_ != (long)v.size()) ReInit((long)v.size());
    if (dim_) std::memcpy(data_, &v[0], sizeof(T) * dim_);
    return *this;
  }
  void Swap(Vector& o) {
    std::swap(dim_, o.dim_);
    std::swap(data_, o.data_);
    std::swap(own_, o.own_);
  }
  long Dim() const { return dim_; }
  T& operator[](long i) const { return data_[i]; }
  T* begin() const { return data_; }

 private:
  void release() {
    if (own_ && data_) std::free(data_);
    data_ = NULL;
    dim_ = 0;
  }
  long dim_;
  T* data_;
  bool own_;
};

template <class T>
class Matrix {
 public:
  Matrix() : r_(0), c_(0), data_(NULL), own_(true) {}
  Matrix(long r, long c, T* ptr = NULL, bool own = true) : r_(0), c_(0), data_(NULL), own_(true) {
    ReInit(r, c, ptr, own);
  }
  Matrix(const Matrix& o) : r_(0), c_(0), data_(NULL), own_(true) { ReInit(o.r_, o.c_, o.data_, true); }
  ~Matrix() { release(); }

  void ReInit(long r, long c, T* ptr = NULL, bool own = true) {
    long n = r * c;
    if (own) {
      T* fresh = n > 0 ? (T*)std::malloc(sizeof(T) * n) : NULL;
      if (ptr && n > 0) std::memcpy(fresh, ptr, sizeof(T) * n);
      else if (n > 0) std::memset(fresh, 0, sizeof(T) * n);
      release();
      data_ = fresh;
      own_ = true;
    } else {
      release();
      data_ = ptr;
      own_ = false;
    }
    r_ = r;
    c_ = c;
  }
  Matrix& operator=(const Matrix& o) {
    if (this == &o) return *this;
    if (r_ * c_ != o.r_ * o.c_) ReInit(o.r_, o.c_);
    r_ = o.r_;
    c_ = o.c_;
    if (r_ * c_) std::memcpy(data_, o.data_, sizeof(T) * r_ * c_);
    return *this;
  }
  long Dim(int i) const { return i == 0 ? r_ : c_; }
  T* operator[](long i) const { return data_ + i * c_; }
  void SetZero() {
    if (r_ * c_) std::memset(data_, 0, sizeof(T) * r_ * c_);
  }
  Matrix Transpose() const {
    Matrix t(c_, r_);
    for (long i = 0; i < r_; i++)
      for (long j = 0; j < c_; j++) t.data_[j * r_ + i] = data_[i * c_ + j];
    return t;
  }
  Matrix operator*(const Matrix& B) const {
    assert(c_ == B.r_);
    Matrix C(r_, B.c_);
    shim::gemm_rm(r_, B.c_, c_, data_, B.data_, C.data_);
    return C;
  }
  static void GEMM(Matrix& C, const Matrix& A, const Matrix& B) {
    assert(A.c_ == B.r_);
    assert(C.r_ == A.r_ && C.c_ == B.c_);
    shim::gemm_rm(A.r_, B.c_, A.c_, A.data_, B.data_, C.data_);
  }

 private:
  void release() {
    if (own_ && data_) std::free(data_);
    data_ = NULL;
  }
  long r_, c_;
  T* data_;
  bool own_;
};

// The reference wraps its stages in pvfmm::Profile timers; they are no-ops here.
class Profile {
 public:
  static bool Enable(bool) { return false; }
  template <class C>
  static void Tic(const char*, C*, bool = false, int = 0) {}
  static void Tic(const char*) {}
  static void Toc() {}
  static void Add_FLOP(long long) {}
  static void Add_MEM(long long) {}
};

}  // namespace pvfmm

#endif
