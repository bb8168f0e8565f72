// FourierSolver2D (rcwa/FourierSolver2D.h:15-44 of the reference) over the
// device convolution-matrix kernels: solve() is FourierSolver2D.cpp:12-351
// without the parameter derivatives (dFfs), which are off the efficiency path.
#pragma once
#include <iostream>
#include <vector>

#include "defns.h"
#include "engine_handle.h"

enum FourierSolverOption { ContinuousXY = 0, DiscontinuousX = 1, DiscontinuousY = 2 };

class FourierSolver2D {
 public:
  FourierSolver2D(const Eigen::VectorXs& coordX, const Eigen::VectorXs& coordY) : cx_(coordX), cy_(coordY) {}

  void solve(const Eigen::MatrixXcs& f, int nx, int ny, FourierSolverOption opt, Eigen::MatrixXcs& Ff) {
    Ff.resize(nx * ny, nx * ny);
    rcwa_engine* e = rcwa_b200::engine();
    if (!e) return;
    std::vector<double> cx((size_t)cx_.size()), cy((size_t)cy_.size());
    for (Eigen::Index i = 0; i < (Eigen::Index)cx_.size(); ++i) cx[(size_t)i] = cx_[i];
    for (Eigen::Index i = 0; i < (Eigen::Index)cy_.size(); ++i) cy[(size_t)i] = cy_[i];
    std::vector<rcwa_cplx> fr((size_t)(f.rows() * f.cols()));
    for (Eigen::Index r = 0; r < f.rows(); ++r)
      for (Eigen::Index c = 0; c < f.cols(); ++c)
        fr[(size_t)(r * f.cols() + c)] = rcwa_cplx{f(r, c).real(), f(r, c).imag()};
    const size_t N = (size_t)nx * ny;
    std::vector<rcwa_cplx> out(N * N);
    const int rc = rcwa_fourier2d(e, cx.data(), (int)cx.size(), cy.data(), (int)cy.size(), fr.data(), nx, ny,
                                  (int)opt, out.data());
    if (rc) {
      std::cerr << "[rcwa_b200] fourier2d: " << rcwa_status_string(rc) << "\n";
      return;
    }
    for (size_t r = 0; r < N; ++r)
      for (size_t c = 0; c < N; ++c) Ff((Eigen::Index)r, (Eigen::Index)c) = scalex(out[r * N + c].re, out[r * N + c].im);
  }

 private:
  Eigen::VectorXs cx_, cy_;
};
