// RCWASolver (rcwa/RCWASolver.h:14-233 of the reference) on the B200 engine.
//
// The public calls the reference's callers make keep their signatures:
// RCWASolver(nX, nY), addLayer, disablePML, setBlochWavevector, solve,
// generateHorizontalPlaneWave and scatterPlaneWave (sol/rcwa_bridge.cpp:273-318,
// rcwa/RCWADriver.cpp:284-339).  solve() runs the whole layer / interface /
// cascade computation on the device through the C ABI and keeps the
// scattering matrices there; every scatterPlaneWave after it only re-evaluates
// the efficiencies for the new incident vector.  generateHorizontalPlaneWave
// returns the plane wave's tangential field [px delta; py delta] and
// scatterPlaneWave takes it as such: the engine itself applies the
// incidence layer's modal basis (the identity for a uniform half-space,
// W_ref^-1 for a patterned one), so the efficiencies are the reference's
// while c holds the field rather than the modal amplitudes of a patterned
// incidence layer.
//
// Tdd() and Rud() copy the solved scattering matrices from the device on
// first access after solve().
//
// Outside this engine (they report on std::cerr and leave outputs empty):
// PML (enablePML), layer translations in solve and saveFieldImage, and
// incident vectors other than generateHorizontalPlaneWave's.
#pragma once
#include <algorithm>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <utility>
#include <vector>

#include "Layer.h"
#include "defns.h"
#include "engine_handle.h"

class RCWASolver {
 public:
  RCWASolver(int nX, int nY) : nx_(2 * nX + 1), ny_(2 * nY + 1), nX_(nX), nY_(nY) {}
  ~RCWASolver() { release(); }
  RCWASolver(const RCWASolver&) = delete;
  RCWASolver& operator=(const RCWASolver&) = delete;

  // rcwa/RCWASolver.cpp:108-137: layers must share the boundary cells
  void addLayer(const Layer& layer) {
    if (!layers_.empty()) {
      const Layer& a = layers_.front();
      if (a.Lx() != layer.Lx() || a.Ly() != layer.Ly() || a.b0() != layer.b0() || a.b1() != layer.b1() ||
          a.u0() != layer.u0() || a.u1() != layer.u1() || a.l0() != layer.l0() || a.l1() != layer.l1() ||
          a.r0() != layer.r0() || a.r1() != layer.r1()) {
        std::cerr << "The new layer does not match layers before!\n";
        return;
      }
    }
    layers_.push_back(layer);
  }
  int nLayerTypes() const { return (int)layers_.size(); }
  void enablePML() { pml_ = true; }
  void disablePML() { pml_ = false; }
  void setBlochWavevector(scalar kx0, scalar ky0) { kx0_ = kx0; ky0_ = ky0; }
  int nx() const { return nx_; }
  int ny() const { return ny_; }

  void solve(scalar lambda, const std::vector<int>& layerStack, const std::vector<scalar>& thickness,
             const std::vector<scalar>* translation = nullptr) {
    release();
    if (pml_ || translation || layerStack.size() < 2 || thickness.size() != layerStack.size()) {
      std::cerr << "[rcwa_b200] solve: PML, translations and stacks of fewer than 2 layers are not supported\n";
      return;
    }
    rcwa_engine* e = rcwa_b200::engine();
    if (!e) return;
    for (int li : layerStack)
      if (li < 0 || li >= (int)layers_.size()) {
        std::cerr << "[rcwa_b200] solve: invalid layer in the stack\n";
        return;
      }
    bool magnetic = false;
    for (int li : layerStack) magnetic = magnetic || layers_[(size_t)li].isMagnetic();
    // common cell grid over every layer of the stack; subdividing a
    // piecewise-constant cell does not change its Fourier coefficients
    cx_ = merged(true, layerStack);
    cy_ = merged(false, layerStack);
    const size_t ncx = cx_.size(), ncy = cy_.size(), cells = (ncx - 1) * (ncy - 1);
    eps_.assign(cells * layerStack.size(), rcwa_cplx{1.0, 0.0});
    mu_.assign(magnetic ? cells * layerStack.size() : 0, rcwa_cplx{1.0, 0.0});
    for (size_t l = 0; l < layerStack.size(); ++l) {
      const Layer& L = layers_[(size_t)layerStack[l]];
      for (size_t j = 0; j + 1 < ncy; ++j)
        for (size_t i = 0; i + 1 < ncx; ++i) {
          const scalar xc = 0.5 * (cx_[i] + cx_[i + 1]), yc = 0.5 * (cy_[j] + cy_[j + 1]);
          const scalex v = L.eps(xc, yc);
          eps_[l * cells + j * (ncx - 1) + i] = rcwa_cplx{v.real(), v.imag()};
          if (magnetic) {
            const scalex m = L.mu(xc, yc);
            mu_[l * cells + j * (ncx - 1) + i] = rcwa_cplx{m.real(), m.imag()};
          }
        }
    }
    thick_.assign(thickness.begin(), thickness.end());
    rcwa_stack st{nX_, nY_, (int)ncx, (int)ncy, cx_.data(), cy_.data(), (int)layerStack.size(), eps_.data(),
                  thick_.data(), magnetic ? mu_.data() : nullptr};
    rcwa_point pt{0, lambda, kx0_, ky0_};
    rcwa_cplx pxy[2] = {{1.0, 0.0}, {0.0, 0.0}};
    int rc = rcwa_plan_create(e, &st, 1, &pt, 1, 1, pxy, RCWA_PREC_FP64, &plan_);
    if (rc == RCWA_OK) rc = rcwa_plan_execute(plan_, nullptr);
    double R, T;
    int status = 0;
    if (rc == RCWA_OK) rc = rcwa_plan_results(plan_, &R, &T, nullptr, nullptr, &status);
    if (rc != RCWA_OK && rc != RCWA_ERR_GRAZING) {
      std::cerr << "[rcwa_b200] solve: " << rcwa_status_string(rc) << " " << rcwa_engine_last_error(e) << "\n";
      release();
      return;
    }
    stack_ = layerStack;
  }

  // generateHorizontalPlaneWave (rcwa/RCWASolver.cpp:1778-1789)
  void generateHorizontalPlaneWave(scalex px, scalex py, int layerType, Eigen::VectorXcs& c) {
    const int N = nx_ * ny_;
    c.resize(2 * N);
    c.setZero();
    if (!plan_ || stack_.empty() || layerType != stack_.front()) {
      std::cerr << "[rcwa_b200] generateHorizontalPlaneWave: solve() the stack and use its incidence layer\n";
      return;
    }
    const int k0 = ny_ * ((nx_ - 1) / 2) + (ny_ - 1) / 2;
    c[k0] = px;
    c[N + k0] = py;
  }

  // scatterPlaneWave (rcwa/RCWASolver.cpp:1792-1908)
  void scatterPlaneWave(const Eigen::VectorXcs& cInc, int refLayerType, int trnLayerType, scalar /*k0*/,
                        Eigen::VectorXs& REF, Eigen::VectorXs& TRN) {
    const int N = nx_ * ny_;
    const int k0i = ny_ * ((nx_ - 1) / 2) + (ny_ - 1) / 2;
    if (!plan_ || stack_.empty() || refLayerType != stack_.front() || trnLayerType != stack_.back() ||
        (int)cInc.size() != 2 * N) {
      std::cerr << "The scatter matrix has not been solved!\n";
      return;
    }
    for (int i = 0; i < 2 * N; ++i)
      if (i != k0i && i != N + k0i && std::abs(cInc[i]) != 0.0) {
        std::cerr << "[rcwa_b200] scatterPlaneWave: only plane waves of generateHorizontalPlaneWave\n";
        return;
      }
    const rcwa_cplx pxy[2] = {{cInc[k0i].real(), cInc[k0i].imag()}, {cInc[N + k0i].real(), cInc[N + k0i].imag()}};
    int rc = rcwa_plan_rescatter(plan_, pxy);
    double R, T;
    std::vector<double> ref((size_t)N), trn((size_t)N);
    int status = 0;
    if (rc == RCWA_OK) rc = rcwa_plan_results(plan_, &R, &T, ref.data(), trn.data(), &status);
    if (rc != RCWA_OK) {
      if (rc == RCWA_ERR_GRAZING) std::cerr << "Warning: incident kz is near zero (grazing incidence?)\n";
      else std::cerr << "[rcwa_b200] scatterPlaneWave: " << rcwa_status_string(rc) << "\n";
      return;
    }
    REF.resize(N);
    TRN.resize(N);
    for (int i = 0; i < N; ++i) {
      REF[i] = ref[(size_t)i];
      TRN[i] = trn[(size_t)i];
    }
  }

  // rcwa/RCWASolver.h:141-142: the cascade's final Tdd_ and Rud_ (empty
  // before a successful solve), downloaded once per solve
  const Eigen::MatrixXcs& Tdd() const { fetch(); return tdd_; }
  const Eigen::MatrixXcs& Rud() const { fetch(); return rud_; }

  // saveFieldImage (rcwa/RCWASolver.cpp:707-1012): one field component on a
  // slice of the solved stack, 500 samples along the first slice axis, the
  // CSV of writeFieldCSV (8 significant digits, ", " between columns; the
  // modulus, real or imaginary part).  The input is the plane wave of
  // generateHorizontalPlaneWave (the zero-order entries of inputCoeffs);
  // layer translations are not provided.
  void saveFieldImage(const std::string& filename, SliceType sliceType, scalar sliceCoord,
                      FieldComponent fieldComponent, SaveOption opt,
                      const std::vector<std::pair<int, scalex>>& inputCoeffs, const std::vector<int>& layerStack,
                      const std::vector<scalar>& /*thickness*/, const std::vector<scalar>* translation = nullptr) {
    const int N = nx_ * ny_;
    const int k0i = ny_ * ((nx_ - 1) / 2) + (ny_ - 1) / 2;
    if (!plan_ || translation || layerStack != stack_) {
      std::cerr << "[rcwa_b200] saveFieldImage: solve() this stack first (no translations)\n";
      return;
    }
    rcwa_cplx px{0.0, 0.0}, py{0.0, 0.0};
    for (const auto& ic : inputCoeffs) {
      if (ic.first == k0i) px = rcwa_cplx{ic.second.real(), ic.second.imag()};
      else if (ic.first == N + k0i) py = rcwa_cplx{ic.second.real(), ic.second.imag()};
      else if (std::abs(ic.second) != 0.0) {
        std::cerr << "[rcwa_b200] saveFieldImage: only the zero-order plane wave of generateHorizontalPlaneWave\n";
        return;
      }
    }
    const int nres1 = 500;
    int rows = 0;
    if (rcwa_plan_field_rows(plan_, 0, (int)sliceType, nres1, &rows) != RCWA_OK) return;
    std::vector<rcwa_cplx> f((size_t)rows * nres1);
    const int rc = rcwa_plan_field(plan_, 0, px, py, (int)sliceType, sliceCoord, (int)fieldComponent, nres1, f.data());
    if (rc != RCWA_OK) {
      std::cerr << "[rcwa_b200] saveFieldImage: " << rcwa_status_string(rc) << "\n";
      return;
    }
    std::ofstream fout(filename);
    if (!fout) {
      std::cerr << "Cannot open field output file: " << filename << "\n";
      return;
    }
    fout << std::setprecision(8);
    for (int i = 0; i < rows; ++i) {
      for (int j = 0; j < nres1; ++j) {
        const rcwa_cplx v = f[(size_t)i * nres1 + j];
        fout << (opt == realpart ? v.re : opt == imagpart ? v.im : std::hypot(v.re, v.im));
        if (j + 1 < nres1) fout << ", ";
      }
      fout << "\n";
    }
  }
  // saveDeviceImage (rcwa/RCWASolver.cpp:1322-1487): the real part of the
  // permittivity of the interior layers on a slice, 2000 samples along the
  // first slice axis, in writeFieldCSV's format; host code on the layers'
  // cell grids (a depth z belongs to the layer with z0 <= z < z1).
  void saveDeviceImage(const std::string& filename, SliceType sliceType, scalar sliceCoord,
                       const std::vector<int>& layerStack, const std::vector<scalar>& thickness,
                       const std::vector<scalar>* translation = nullptr) {
    if (layers_.empty() || layerStack.size() < 3 || thickness.size() != layerStack.size()) {
      std::cerr << "Device image requires at least one finite-thickness interior layer!\n";
      return;
    }
    const Layer& L0 = layers_.front();
    scalar s1 = L0.l0(), L1 = L0.Lx(), s2 = 0.0, L2 = 0.0;
    if (sliceType == sliceYZ) { s1 = L0.b0(); L1 = L0.Ly(); }
    if (sliceType == sliceXY) { s2 = L0.b0(); L2 = L0.Ly(); }
    else
      for (size_t i = 1; i + 1 < layerStack.size(); ++i) L2 += thickness[i];
    const int n1 = 2000;
    int n2 = (int)(n1 * L2 / L1);
    if (n2 < 1) n2 = 1;
    const scalar st1 = L1 / n1, st2 = L2 / n2;
    auto layer_at = [&](scalar z) -> int {
      scalar z0 = 0.0;
      for (size_t j = 1; j + 1 < layerStack.size(); ++j) {
        const scalar z1 = z0 + thickness[j];
        if (z0 <= z && z < z1) return (int)j;
        z0 = z1;
      }
      return -1;
    };
    std::vector<double> dev((size_t)n1 * n2);
    int lfix = sliceType == sliceXY ? layer_at(sliceCoord) : -1;
    if (sliceType == sliceXY && lfix < 0) {
      std::cerr << "Device image requires at least one finite-thickness interior layer!\n";
      return;
    }
    for (int i = 0; i < n2; ++i) {
      const scalar c2 = s2 + st2 * (i + 0.5);
      const int l = sliceType == sliceXY ? lfix : layer_at(c2);
      if (l < 0) {
        std::cerr << "Device image requires at least one finite-thickness interior layer!\n";
        return;
      }
      const Layer& Ly = layers_[(size_t)layerStack[(size_t)l]];
      const scalar tx = translation ? (*translation)[(size_t)l] : 0.0;
      for (int j = 0; j < n1; ++j) {
        const scalar c1 = s1 + st1 * (j + 0.5);
        scalex v;
        if (sliceType == sliceXZ) v = Ly.eps(c1 - tx, sliceCoord);
        else if (sliceType == sliceYZ) v = Ly.eps(sliceCoord - tx, c1);
        else v = Ly.eps(c1 - tx, c2);
        dev[(size_t)i * n1 + j] = v.real();
      }
    }
    std::ofstream fout(filename);
    if (!fout) {
      std::cerr << "Cannot open field output file: " << filename << "\n";
      return;
    }
    fout << std::setprecision(8);
    for (int i = 0; i < n2; ++i) {
      for (int j = 0; j < n1; ++j) {
        fout << dev[(size_t)i * n1 + j];
        if (j + 1 < n1) fout << ", ";
      }
      fout << "\n";
    }
  }

 private:
  std::vector<double> merged(bool xaxis, const std::vector<int>& stack) const {
    std::vector<double> e;
    for (int li : stack) {
      const Layer& L = layers_[(size_t)li];
      const int nc = xaxis ? L.nCx() : L.nCy();
      for (int i = 0; i < nc; ++i) e.push_back(xaxis ? L.coordX(i) : L.coordY(i));
    }
    std::sort(e.begin(), e.end());
    const double span = e.back() - e.front();
    std::vector<double> u;
    for (double v : e)
      if (u.empty() || v - u.back() > 1e-12 * span) u.push_back(v);
    return u;
  }
  void release() {
    if (plan_) rcwa_plan_destroy(plan_);
    plan_ = nullptr;
    fetched_ = false;
    tdd_.resize(0, 0);
    rud_.resize(0, 0);
  }
  void fetch() const {
    if (fetched_ || !plan_ || stack_.empty()) return;
    fetched_ = true;
    const int n = 2 * nx_ * ny_;
    std::vector<rcwa_cplx> r((size_t)n * n), t((size_t)n * n);
    const int rc = rcwa_plan_smatrix(plan_, 0, r.data(), t.data());
    if (rc != RCWA_OK) {
      std::cerr << "[rcwa_b200] Tdd/Rud: " << rcwa_status_string(rc) << "\n";
      return;
    }
    rud_.resize(n, n);
    tdd_.resize(n, n);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        const rcwa_cplx a = r[(size_t)i * n + j], b = t[(size_t)i * n + j];
        rud_(i, j) = scalex(a.re, a.im);
        tdd_(i, j) = scalex(b.re, b.im);
      }
  }

  int nx_, ny_, nX_, nY_;
  bool pml_ = true;
  scalar kx0_ = 0.0, ky0_ = 0.0;
  std::vector<Layer> layers_;
  std::vector<int> stack_;
  std::vector<double> cx_, cy_, thick_;
  std::vector<rcwa_cplx> eps_, mu_;
  rcwa_plan* plan_ = nullptr;
  mutable bool fetched_ = false;
  mutable Eigen::MatrixXcs tdd_, rud_;
};
