// DifferentialIntegrator (core/DifferentialIntegrator.h:8-40 of the
// reference) on the B200 engine: compute(N) samples the caller's
// LayerSampler at z0 + k dz/2 (k = 0 .. 2N: every slab's ends and midpoint)
// and hands the matrices to rcwa_differential_integrate (all slabs' transfer
// blocks and S-matrices in batches on the device, then the cascade).  The
// reference samples z1 and z0 again for the end modes; here the modes of the
// first and last samples serve (the same depths up to the rounding of
// z0 + N dz).  A failing call reports on std::cerr and leaves the accessors
// empty.
#pragma once
#include <iostream>
#include <memory>

#include "integrator_common.h"

class DifferentialIntegrator {
 public:
  DifferentialIntegrator(scalar z0, scalar z1, std::shared_ptr<LayerSampler> sampler)
      : z0_(z0), z1_(z1), sampler_(std::move(sampler)) {}

  // core/DifferentialIntegrator.cpp:21-133
  template <class S = LayerSampler>
  void compute(int N) {
    S& s = *sampler_;
    const int n = s.nDim();
    if (N < 1 || n < 1) {
      std::cerr << "[rcwa_b200] DifferentialIntegrator::compute: invalid slab count or sampler size\n";
      return;
    }
    rcwa_engine* e = rcwa_b200::engine();
    if (!e) return;
    const size_t nn = (size_t)n * n;
    const int ns = 2 * N + 1;
    std::vector<rcwa_cplx> P(nn * ns), Q(nn * ns);
    const scalar dz = (z1_ - z0_) / static_cast<scalar>(N);
    bool ok = true;
    for (int k = 0; ok && k < ns; ++k)
      ok = rcwa_b200::integ::sample_rows(s, z0_ + k * dz / 2, n, P.data() + nn * k, Q.data() + nn * k);
    if (!ok) {
      std::cerr << "[rcwa_b200] DifferentialIntegrator::compute: the sampler's matrices are not nDim x nDim\n";
      return;
    }
    b_.alloc(n);
    const int rc = rcwa_differential_integrate(e, n, N, s.lambda(), z0_, z1_, P.data(), Q.data(), b_.p(0),
                                               b_.p(1), b_.p(2), b_.p(3), b_.p(4), b_.p(5), b_.p(6), b_.p(7),
                                               b_.p(8), b_.p(9));
    if (rc != RCWA_OK) {
      std::cerr << "[rcwa_b200] DifferentialIntegrator::compute: " << rcwa_status_string(rc) << "\n";
      return;
    }
    b_.publish(n);
  }

  const Eigen::MatrixXcs& Tdd() const { return b_.Tdd; }
  const Eigen::MatrixXcs& Tuu() const { return b_.Tuu; }
  const Eigen::MatrixXcs& Rud() const { return b_.Rud; }
  const Eigen::MatrixXcs& Rdu() const { return b_.Rdu; }
  const Eigen::MatrixXcs& W0() const { return b_.W0; }
  const Eigen::MatrixXcs& V0() const { return b_.V0; }
  const Eigen::VectorXcs& gam0() const { return b_.gam0; }
  const Eigen::MatrixXcs& W1() const { return b_.W1; }
  const Eigen::MatrixXcs& V1() const { return b_.V1; }
  const Eigen::VectorXcs& gam1() const { return b_.gam1; }

 private:
  scalar z0_, z1_;
  std::shared_ptr<LayerSampler> sampler_;
  rcwa_b200::integ::Blocks b_;
};
