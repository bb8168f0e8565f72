// FourierSolver1D (rcwa/FourierSolver1D.h:7-59 of the reference) over the
// device coefficient kernel: solve() is FourierSolver1D.cpp:11-41.
#pragma once
#include <iostream>
#include <vector>

#include "defns.h"
#include "engine_handle.h"

class FourierSolver1D {
 public:
  FourierSolver1D(const Eigen::VectorXs& x, scalar d) : x_(x), d_(d) {}

  void solve(const Eigen::VectorXcs& f, int M, Eigen::VectorXcs& Ff) {
    Ff.resize(M);
    if ((Eigen::Index)f.size() != (Eigen::Index)x_.size() - 1) {
      std::cerr << "The function configuration does not match the coordinates!\n";
      return;
    }
    rcwa_engine* e = rcwa_b200::engine();
    if (!e) return;
    std::vector<double> x((size_t)x_.size());
    for (Eigen::Index i = 0; i < (Eigen::Index)x_.size(); ++i) x[(size_t)i] = x_[i];
    std::vector<rcwa_cplx> fi((size_t)f.size()), fo((size_t)M);
    for (Eigen::Index i = 0; i < (Eigen::Index)f.size(); ++i) fi[(size_t)i] = rcwa_cplx{f[i].real(), f[i].imag()};
    const int rc = rcwa_fourier1d(e, x.data(), (int)x.size(), d_, fi.data(), M, fo.data());
    if (rc) {
      std::cerr << "[rcwa_b200] fourier1d: " << rcwa_status_string(rc) << "\n";
      return;
    }
    for (int i = 0; i < M; ++i) Ff[i] = scalex(fo[(size_t)i].re, fo[(size_t)i].im);
  }

 private:
  Eigen::VectorXs x_;
  scalar d_;
};
