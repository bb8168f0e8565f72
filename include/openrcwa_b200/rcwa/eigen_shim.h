// Minimal stand-ins for the Eigen dense types the RCWA callers use, for
// builds without Eigen (sol/rcwa_bridge.cpp and rcwa/RCWADriver.cpp only
// construct, index, size, sum and read data() of these).  When <Eigen/Core>
// is available, defns.h uses the real Eigen instead.  Storage is
// column-major, as in Eigen.
#pragma once
#include <complex>
#include <cstddef>
#include <vector>

namespace Eigen {
typedef std::ptrdiff_t Index;

template <class T>
class ShimVector {
 public:
  ShimVector() {}
  explicit ShimVector(Index n) : v_((size_t)n) {}
  Index size() const { return (Index)v_.size(); }
  void resize(Index n) { v_.assign((size_t)n, T()); }
  void setZero() { for (auto& x : v_) x = T(); }
  T& operator[](Index i) { return v_[(size_t)i]; }
  const T& operator[](Index i) const { return v_[(size_t)i]; }
  T& operator()(Index i) { return v_[(size_t)i]; }
  const T& operator()(Index i) const { return v_[(size_t)i]; }
  T sum() const {
    T s = T();
    for (const auto& x : v_) s += x;
    return s;
  }
  T* data() { return v_.data(); }
  const T* data() const { return v_.data(); }

 private:
  std::vector<T> v_;
};

template <class T>
class ShimMatrix {
 public:
  ShimMatrix() {}
  ShimMatrix(Index r, Index c) : r_(r), c_(c), v_((size_t)(r * c)) {}
  Index rows() const { return r_; }
  Index cols() const { return c_; }
  Index size() const { return r_ * c_; }
  void resize(Index r, Index c) { r_ = r; c_ = c; v_.assign((size_t)(r * c), T()); }
  void setZero() { for (auto& x : v_) x = T(); }
  T& operator()(Index r, Index c) { return v_[(size_t)(c * r_ + r)]; }
  const T& operator()(Index r, Index c) const { return v_[(size_t)(c * r_ + r)]; }
  T* data() { return v_.data(); }
  const T* data() const { return v_.data(); }

 private:
  Index r_ = 0, c_ = 0;
  std::vector<T> v_;
};

typedef ShimVector<double> VectorXs;
typedef ShimVector<std::complex<double>> VectorXcs;
typedef ShimVector<int> VectorXi;
typedef ShimMatrix<double> MatrixXs;
typedef ShimMatrix<std::complex<double>> MatrixXcs;
}  // namespace Eigen
