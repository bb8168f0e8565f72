// Shared pieces of the z-integrator adapters (core/RCWAIntegrator.h,
// core/DifferentialIntegrator.h, core/RedhefferIntegrator.h of the
// reference): the caller's LayerSampler (core/LayerSampler.h of the
// reference, or any class with lambda(), nDim() and
// sample(z, MatrixXcs& P, MatrixXcs& Q)) is only declared here; the calls on
// it are member templates instantiated where the caller, who has the
// sampler's definition, calls compute().
#pragma once
#include <complex>
#include <vector>

#include "../rcwa/defns.h"
#include "../rcwa/engine_handle.h"

class LayerSampler;

namespace rcwa_b200 {
namespace integ {

// P, Q of the sampler at depth z, row-major into P, Q (n*n each); false when
// the sampler's matrices are not n x n
template <class S>
bool sample_rows(S& s, scalar z, int n, rcwa_cplx* P, rcwa_cplx* Q) {
  Eigen::MatrixXcs Pm, Qm;
  s.sample(z, Pm, Qm);
  if (Pm.rows() != n || Pm.cols() != n || Qm.rows() != n || Qm.cols() != n) return false;
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) {
      const scalex p = Pm(r, c), q = Qm(r, c);
      P[(size_t)r * n + c] = rcwa_cplx{p.real(), p.imag()};
      Q[(size_t)r * n + c] = rcwa_cplx{q.real(), q.imag()};
    }
  return true;
}

// the accessors' storage: filled from the C ABI's row-major outputs
struct Blocks {
  Eigen::MatrixXcs Tdd, Tuu, Rud, Rdu, W0, V0, W1, V1;
  Eigen::VectorXcs gam0, gam1;
  std::vector<rcwa_cplx> buf[10];  // Rud, Rdu, Tdd, Tuu, W0, V0, gam0, W1, V1, gam1

  void alloc(int n) {
    for (int k = 0; k < 10; ++k) buf[k].assign((k == 6 || k == 9) ? (size_t)n : (size_t)n * n, rcwa_cplx{0, 0});
  }
  rcwa_cplx* p(int k) { return buf[k].data(); }
  static void to_matrix(const std::vector<rcwa_cplx>& v, int n, Eigen::MatrixXcs& m) {
    m.resize(n, n);
    for (int r = 0; r < n; ++r)
      for (int c = 0; c < n; ++c) m(r, c) = scalex(v[(size_t)r * n + c].re, v[(size_t)r * n + c].im);
  }
  static void to_vector(const std::vector<rcwa_cplx>& v, int n, Eigen::VectorXcs& x) {
    x.resize(n);
    for (int i = 0; i < n; ++i) x(i) = scalex(v[(size_t)i].re, v[(size_t)i].im);
  }
  void publish(int n) {
    to_matrix(buf[0], n, Rud); to_matrix(buf[1], n, Rdu); to_matrix(buf[2], n, Tdd); to_matrix(buf[3], n, Tuu);
    to_matrix(buf[4], n, W0); to_matrix(buf[5], n, V0); to_vector(buf[6], n, gam0);
    to_matrix(buf[7], n, W1); to_matrix(buf[8], n, V1); to_vector(buf[9], n, gam1);
  }
};

}  // namespace integ
}  // namespace rcwa_b200
