// C++ API adapter check: the 1D grating through RCWASolver / Layer (the calls
// sol/rcwa_bridge.cpp makes), printing R and T for TE and TM at 650 THz.
#include <cstdio>

#include "rcwa/FourierSolver1D.h"
#include "rcwa/FourierSolver2D.h"
#include "rcwa/RCWASolver.h"

int main() {
  Eigen::VectorXs cx(3), cy(2);
  cx[0] = 0; cx[1] = 1.5e-7; cx[2] = 3e-7;
  cy[0] = 0; cy[1] = 3e-7;
  Eigen::MatrixXcs e0(1, 2), e1(1, 2), e2(1, 2);
  e0(0, 0) = e0(0, 1) = 1.0;
  e1(0, 0) = 4.0; e1(0, 1) = 1.0;
  e2(0, 0) = e2(0, 1) = 2.25;
  RCWASolver s(5, 0);
  s.disablePML();
  s.addLayer(Layer(cx, cy, e0));
  s.addLayer(Layer(cx, cy, e1));
  s.addLayer(Layer(cx, cy, e2));
  s.setBlochWavevector(0, 0);
  const double lam = 2.99792458e8 / 6.5e14, k0 = 2 * Pi / lam;
  s.solve(lam, {0, 1, 2}, {0, 2e-7, 0});
  for (int pol = 0; pol < 2; ++pol) {  // TE = E//y, TM = E//x at normal incidence
    Eigen::VectorXcs c;
    s.generateHorizontalPlaneWave(pol == 0 ? 0.0 : 1.0, pol == 0 ? 1.0 : 0.0, 0, c);
    Eigen::VectorXs R, T;
    s.scatterPlaneWave(c, 0, 2, k0, R, T);
    std::printf("%.12f %.12f\n", R.sum(), T.sum());
  }
  // the solved scattering matrices (RCWASolver::Rud(), Tdd()), row by row
  const Eigen::MatrixXcs& Rud = s.Rud();
  const Eigen::MatrixXcs& Tdd = s.Tdd();
  std::printf("%d %d\n", (int)Rud.rows(), (int)Tdd.cols());
  for (int i = 0; i < (int)Rud.rows(); ++i)
    for (int j = 0; j < (int)Rud.cols(); ++j)
      std::printf("%.17g %.17g %.17g %.17g\n", Rud(i, j).real(), Rud(i, j).imag(), Tdd(i, j).real(),
                  Tdd(i, j).imag());
  return 0;
}
