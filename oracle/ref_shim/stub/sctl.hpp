// Minimal stand-in for the parts of the SCTL library that the reference's
// header-only math (pswf.hpp, kernels.hpp, shiftmat.hpp, utils.hpp,
// nudft.hpp, vecops.hpp) names. SCTL itself is an unvendored submodule of the
// reference (extern/SCTL is empty); only a growable array, the Long type and a
// tree node-attribute type are needed to compile those headers. This stub is
// test infrastructure for the oracle's reference build only.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>
#include <algorithm>

extern "C" void dgemm_(char* TransA, char* TransB, int* M, int* N, int* K, double* alpha,
                       double* A, int* lda, double* B, int* ldb, double* beta, double* C, int* ldc);

namespace sctl {
using Long = long;
using Integer = long;

template <class T>
class Vector {
 public:
  Vector() = default;
  explicit Vector(Long n) : v_(static_cast<std::size_t>(n)) {}
  Vector(Long n, T* ptr, bool own = true) : v_(ptr, ptr + n) { (void)own; }
  void ReInit(Long n) { v_.assign(static_cast<std::size_t>(n), T()); }
  Long Dim() const { return static_cast<Long>(v_.size()); }
  T& operator[](Long i) { return v_[static_cast<std::size_t>(i)]; }
  const T& operator[](Long i) const { return v_[static_cast<std::size_t>(i)]; }
  void PushBack(const T& x) { v_.push_back(x); }
  void SetZero() { std::fill(v_.begin(), v_.end(), T()); }
  T* begin() { return v_.data(); }
  T* end() { return v_.data() + v_.size(); }
  const T* begin() const { return v_.data(); }
  const T* end() const { return v_.data() + v_.size(); }
  template <class S> Vector& operator-=(const S& s) { for (auto& x : v_) x -= s; return *this; }
  template <class S> Vector& operator*=(const S& s) { for (auto& x : v_) x *= s; return *this; }
 private:
  std::vector<T> v_;
};

template <int DIM>
struct Tree {
  struct NodeAttr { unsigned char Leaf = 0, Ghost = 0; };
};
}  // namespace sctl
