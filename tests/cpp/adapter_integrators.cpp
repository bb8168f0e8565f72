// C++ API adapter check for the z-integrators: a sampler with the shape of
// the reference's LayerSampler (core/LayerSampler.h: lambda(), nDim(), a
// virtual sample(z, P, Q)) drives RCWAIntegrator, DifferentialIntegrator and
// RedhefferIntegrator as the reference's integrator test does, and the sizes
// of their outputs are printed (empty when no device is present).
#include <cstdio>
#include <memory>

#include "rcwa/defns.h"

class LayerSampler {
 public:
  LayerSampler(scalar lambda, int nx, int ny) : lambda_(lambda), nx_(nx), ny_(ny) {}
  virtual ~LayerSampler() {}
  scalar lambda() const { return lambda_; }
  int nDim() const { return 2 * nx_ * ny_; }
  virtual void sample(scalar z, Eigen::MatrixXcs& P, Eigen::MatrixXcs& Q) = 0;

 protected:
  scalar lambda_;
  int nx_, ny_;
};

#include "core/DifferentialIntegrator.h"
#include "core/RCWAIntegrator.h"
#include "core/RedhefferIntegrator.h"

// a homogeneous medium whose permittivity grows with depth, orders on a
// square lattice (P and Q of Layer::waveEqnCoeff with Kx, Ky diagonal)
class GradedSampler : public LayerSampler {
 public:
  GradedSampler() : LayerSampler(1.55, 3, 3) {}
  void sample(scalar z, Eigen::MatrixXcs& P, Eigen::MatrixXcs& Q) override {
    const int N = nx_ * ny_, n = 2 * N;
    const scalar k0 = 2 * Pi / lambda_, eps = 2.0 + 0.5 * z;
    P.resize(n, n);
    Q.resize(n, n);
    P.setZero();
    Q.setZero();
    for (int i = 0; i < nx_; ++i)
      for (int j = 0; j < ny_; ++j) {
        const int m = ny_ * i + j;
        const scalar kx = 2 * Pi / 2.0 * (i - nx_ / 2), ky = 2 * Pi / 2.0 * (j - ny_ / 2);
        P(m, m) = kx * ky / eps;
        P(m, N + m) = k0 * k0 - kx * kx / eps;
        P(N + m, m) = ky * ky / eps - k0 * k0;
        P(N + m, N + m) = -ky * kx / eps;
        Q(m, m) = -kx * ky;
        Q(m, N + m) = kx * kx - k0 * k0 * eps;
        Q(N + m, m) = k0 * k0 * eps - ky * ky;
        Q(N + m, N + m) = ky * kx;
      }
  }
};

int main() {
  auto s = std::make_shared<GradedSampler>();
  RCWAIntegrator a(0.0, 1.0, s);
  a.compute(16);
  DifferentialIntegrator b(0.0, 1.0, s);
  b.compute(16);
  RedhefferIntegrator c(0.0, 1.0, s);
  c.compute(0, 100000, 1e-3);
  std::printf("%ld %ld %ld %d\n", (long)a.Tuu().rows(), (long)b.Tuu().rows(), (long)c.Tuu().rows(), c.N());
  return 0;
}
