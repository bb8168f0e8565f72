// RedhefferIntegrator (core/RedhefferIntegrator.h:9-90 of the reference) on
// the B200 engine: compute(p, maxN, pe) hands the caller's LayerSampler to
// rcwa_redheffer_integrate as a callback (the depths it samples depend on the
// subdivision), which evaluates every subdivision level in one batch on the
// device.  As in the reference, p and maxN do not steer the computation;
// the engine's own cap on accepted intervals is 2^20.  N() is the number of
// accepted intervals; nEigVal() the eigen-solves performed (the reference's
// active branch leaves it at 2).  A failing call reports on std::cerr and
// leaves the accessors empty.
#pragma once
#include <iostream>
#include <memory>

#include "integrator_common.h"

class RedhefferIntegrator {
 public:
  RedhefferIntegrator(scalar z0, scalar z1, std::shared_ptr<LayerSampler> sampler)
      : z0_(z0), z1_(z1), sampler_(std::move(sampler)) {}

  // core/RedhefferIntegrator.cpp:190-245
  template <class S = LayerSampler>
  void compute(int p, int maxN = 10, scalar pe = 1e-2) {
    (void)p;
    (void)maxN;
    S& s = *sampler_;
    const int n = s.nDim();
    if (n < 1) return;
    rcwa_engine* e = rcwa_b200::engine();
    if (!e) return;
    struct Ctx {
      S* s;
      int n;
    } ctx{&s, n};
    auto cb = [](void* user, double z, rcwa_cplx* P, rcwa_cplx* Q) -> int {
      Ctx* c = static_cast<Ctx*>(user);
      return rcwa_b200::integ::sample_rows(*c->s, z, c->n, P, Q) ? 0 : 1;
    };
    b_.alloc(n);
    const int rc = rcwa_redheffer_integrate(e, n, s.lambda(), z0_, z1_, pe, 1 << 20, cb, &ctx, b_.p(0), b_.p(1),
                                            b_.p(2), b_.p(3), b_.p(4), b_.p(5), b_.p(6), b_.p(7), b_.p(8),
                                            b_.p(9), &N_, &nEigVal_);
    if (rc != RCWA_OK) {
      std::cerr << "[rcwa_b200] RedhefferIntegrator::compute: " << rcwa_status_string(rc) << "\n";
      return;
    }
    b_.publish(n);
  }

  int N() const { return N_; }
  int nEigVal() const { return nEigVal_; }
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
  int N_ = 0, nEigVal_ = 0;
};
