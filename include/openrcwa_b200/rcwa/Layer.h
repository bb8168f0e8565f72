// Layer (rcwa/Layer.h:8-138 of the reference): a piecewise-constant
// permittivity, and optionally a relative permeability, on a cell grid.  Its
// modes are solved on the device as part of RCWASolver::solve; this class only
// holds the geometry and exposes the accessors the callers use.  A layer is
// magnetic when some cell's mu differs from 1 by more than 1e-12
// (rcwa/Layer.cpp:64-71).
#pragma once
#include <iostream>

#include "defns.h"

class Layer {
 public:
  Layer(const Eigen::VectorXs& coordX, const Eigen::VectorXs& coordY, const Eigen::MatrixXcs& eps)
      : coordX_(coordX), coordY_(coordY), eps_(eps) {
    if (eps.rows() != (Eigen::Index)coordY.size() - 1 || eps.cols() != (Eigen::Index)coordX.size() - 1)
      std::cerr << "The configuration of permittivity does not match coordinates!\n";
    unit_mu();
  }
  Layer(const Eigen::VectorXs& coordX, const Eigen::VectorXs& coordY, const Eigen::MatrixXcs& eps,
        const Eigen::MatrixXcs& mu)
      : Layer(coordX, coordY, eps) {
    if (mu.rows() != eps.rows() || mu.cols() != eps.cols()) {
      std::cerr << "The configuration of permeability does not match permittivity!\n";
      return;
    }
    mu_ = mu;
    for (Eigen::Index i = 0; i < mu.rows(); ++i)
      for (Eigen::Index j = 0; j < mu.cols(); ++j)
        if (std::abs(mu(i, j) - scalex(1.0, 0.0)) > 1e-12) magnetic_ = true;
  }

  const Eigen::MatrixXcs& eps() const { return eps_; }
  const Eigen::MatrixXcs& mu() const { return mu_; }
  bool isMagnetic() const { return magnetic_; }
  int nCx() const { return (int)coordX_.size(); }
  int nCy() const { return (int)coordY_.size(); }
  const Eigen::VectorXs& coordX() const { return coordX_; }
  const Eigen::VectorXs& coordY() const { return coordY_; }
  scalar coordX(int i) const { return coordX_[i]; }
  scalar coordY(int i) const { return coordY_[i]; }
  scalar Lx() const { return coordX_[nCx() - 1] - coordX_[0]; }
  scalar Ly() const { return coordY_[nCy() - 1] - coordY_[0]; }
  scalar b0() const { return coordY_[0]; }
  scalar b1() const { return coordY_[1]; }
  scalar u0() const { return coordY_[nCy() - 2]; }
  scalar u1() const { return coordY_[nCy() - 1]; }
  scalar l0() const { return coordX_[0]; }
  scalar l1() const { return coordX_[1]; }
  scalar r0() const { return coordX_[nCx() - 2]; }
  scalar r1() const { return coordX_[nCx() - 1]; }

  // Layer::eps(x, y): the cell containing (x, y), x periodic (rcwa/Layer.cpp:383-429)
  scalex eps(scalar x, scalar y) const { return at(eps_, x, y); }
  // Layer::mu(x, y): the same cell lookup on the permeability (rcwa/Layer.cpp:431-450)
  scalex mu(scalar x, scalar y) const { return at(mu_, x, y); }

 private:
  void unit_mu() {
    mu_.resize(eps_.rows(), eps_.cols());
    for (Eigen::Index i = 0; i < eps_.rows(); ++i)
      for (Eigen::Index j = 0; j < eps_.cols(); ++j) mu_(i, j) = scalex(1.0, 0.0);
  }
  scalex at(const Eigen::MatrixXcs& m, scalar x, scalar y) const {
    while (x < l0()) x += Lx();
    while (x > r1()) x -= Lx();
    if (y < b0() || y > u1()) {
      std::cerr << "The coordinate y is out of range!\n";
      return scalex(0.0);
    }
    int ix = 0, iy = 0;
    for (int i = 0; i < nCx() - 1; ++i)
      if (x <= coordX_[i + 1]) { ix = i; break; }
    for (int j = 0; j < nCy() - 1; ++j)
      if (y <= coordY_[j + 1]) { iy = j; break; }
    return m(iy, ix);
  }

  Eigen::VectorXs coordX_, coordY_;
  Eigen::MatrixXcs eps_, mu_;
  bool magnetic_ = false;
};
