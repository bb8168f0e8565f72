// RCWAIntegrator (core/RCWAIntegrator.h:8-40 of the reference) on the B200
// engine: compute(N) samples the caller's LayerSampler at z0, at the N slab
// midpoints and at z1, and hands the matrices to rcwa_rcwa_integrate, which
// solves every sample's modes and every slab's S-matrix in batches on the
// device and cascades the slabs there.  The accessors return the results
// (same bases and conventions as the reference).  A failing call reports on
// std::cerr and leaves the accessors empty.
#pragma once
#include <iostream>
#include <memory>

#include "integrator_common.h"

class RCWAIntegrator {
 public:
  RCWAIntegrator(scalar z0, scalar z1, std::shared_ptr<LayerSampler> sampler)
      : z0_(z0), z1_(z1), sampler_(std::move(sampler)) {}

  // core/RCWAIntegrator.cpp:21-86
  template <class S = LayerSampler>
  void compute(int N) {
    S& s = *sampler_;
    const int n = s.nDim();
    if (N < 0 || n < 1) {
      std::cerr << "[rcwa_b200] RCWAIntegrator::compute: invalid slab count or sampler size\n";
      return;
    }
    rcwa_engine* e = rcwa_b200::engine();
    if (!e) return;
    const size_t nn = (size_t)n * n;
    std::vector<rcwa_cplx> P(nn * (N + 2)), Q(nn * (N + 2));
    const scalar dz = N > 0 ? (z1_ - z0_) / static_cast<scalar>(N) : 0.0;
    bool ok = rcwa_b200::integ::sample_rows(s, z0_, n, P.data(), Q.data());
    for (int i = 0; ok && i < N; ++i)
      ok = rcwa_b200::integ::sample_rows(s, z0_ + (i + 0.5) * dz, n, P.data() + nn * (1 + i), Q.data() + nn * (1 + i));
    ok = ok && rcwa_b200::integ::sample_rows(s, z1_, n, P.data() + nn * (N + 1), Q.data() + nn * (N + 1));
    if (!ok) {
      std::cerr << "[rcwa_b200] RCWAIntegrator::compute: the sampler's matrices are not nDim x nDim\n";
      return;
    }
    b_.alloc(n);
    const int rc = rcwa_rcwa_integrate(e, n, N, s.lambda(), z0_, z1_, P.data(), Q.data(), b_.p(0), b_.p(1), b_.p(2),
                                       b_.p(3), b_.p(4), b_.p(5), b_.p(6), b_.p(7), b_.p(8), b_.p(9));
    if (rc != RCWA_OK) {
      std::cerr << "[rcwa_b200] RCWAIntegrator::compute: " << rcwa_status_string(rc) << "\n";
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
