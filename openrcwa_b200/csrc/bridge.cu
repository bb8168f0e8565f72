// Host side of the .ofd RCWA mode: sol/rcwa_bridge.cpp restated on top of the
// batched engine.  The reference builds one RCWASolver per frequency and
// solves them one after another (sol/rcwa_bridge.cpp:244-366); here every
// frequency becomes one point of a single batched solve, both polarisations
// being extracted from the same scattering matrix.
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

#include "engine_internal.cuh"

namespace {

constexpr double kC0 = 2.99792458e8;        // sol/rcwa_bridge.cpp:44
constexpr double kPi = 3.1415926535897932;  // rcwa/defns.h:25

// commonEdges (sol/rcwa_bridge.cpp:52-67): cell edges shared by all layers.
std::vector<double> common_edges(const rcwa_ofd_setup& s, double period, bool use_y) {
  std::vector<double> e{0.0};
  for (int n = 0; n < s.n_layers; ++n) {
    const double f = use_y ? s.layers[n].fill_y : s.layers[n].fill;
    if (f < 1.0) e.push_back(f * period);
  }
  e.push_back(period);
  std::sort(e.begin(), e.end());
  std::vector<double> u;
  for (double v : e)
    if (u.empty() || (v - u.back()) > 1e-12 * period) u.push_back(v);
  return u;
}

bool has_dispersion(const rcwa_ofd_setup& s, int n, int side) {
  for (int p = 0; p < s.n_poles; ++p) {
    const rcwa_pole_spec& q = s.poles[p];
    if (q.layer == n && q.side == side && q.ae != 0.0) return true;
  }
  return false;
}

// layerEps (sol/rcwa_bridge.cpp:105-123): static value or Lorentz poles
// eps = einf + sum ae^2 / (ce^2 - w^2 - i be w), einf from the last row.
std::complex<double> layer_eps(const rcwa_ofd_setup& s, int n, int side, double omega) {
  const rcwa_layer_spec& l = s.layers[n];
  if (!has_dispersion(s, n, side))
    return side == 1 ? std::complex<double>(l.eps1, l.eps1i) : std::complex<double>(l.eps2, l.eps2i);
  double einf = 0.0;
  for (int p = 0; p < s.n_poles; ++p)
    if (s.poles[p].layer == n && s.poles[p].side == side) einf = s.poles[p].einf;
  std::complex<double> e(einf, 0.0);
  for (int p = 0; p < s.n_poles; ++p) {
    const rcwa_pole_spec& q = s.poles[p];
    if (q.layer != n || q.side != side || q.ae == 0.0) continue;
    e += std::complex<double>(q.ae * q.ae, 0.0) / std::complex<double>(q.ce * q.ce - omega * omega, -q.be * omega);
  }
  return e;
}

}  // namespace

extern "C" int rcwa_ofd_solve(rcwa_engine* e, const rcwa_ofd_setup* s, double* R, double* T, double* ordR,
                              double* ordT, int* status) {
  if (!e || !s || !R || !T) return RCWA_ERR_INVALID;
  if (s->n_layers < 2 || !(s->period_x > 0) || s->n_freq < 1 || !s->layers || !s->freq) {
    e->last_error = "invalid rcwa setup";
    return RCWA_ERR_INVALID;
  }
  for (int f = 0; f < s->n_freq; ++f)
    if (!(s->freq[f] > 0)) {
      e->last_error = "invalid frequency1 data";
      return RCWA_ERR_INVALID;
    }
  const int L = s->n_layers;
  const double py_period = s->nHy > 0 ? s->period_y : s->period_x;
  if (!(py_period > 0)) return RCWA_ERR_INVALID;
  const double th = s->theta_deg * kPi / 180.0, ph = s->phi_deg * kPi / 180.0;
  // TE/TM transverse unit vectors (sol/rcwa_bridge.cpp:187-196)
  double tmX, tmY, teX, teY;
  if (std::fabs(std::sin(th)) < 1e-9) {
    tmX = 1.0; tmY = 0.0; teX = 0.0; teY = 1.0;
  } else {
    tmX = std::cos(th) * std::cos(ph);
    tmY = std::cos(th) * std::sin(ph);
    teX = -std::sin(ph);
    teY = std::cos(ph);
  }
  const std::vector<double> xe = common_edges(*s, s->period_x, false);
  const std::vector<double> ye = common_edges(*s, py_period, true);
  const int ncx = (int)xe.size(), ncy = (int)ye.size();
  const size_t cells = (size_t)(ncx - 1) * (ncy - 1);
  std::vector<double> thick(L);
  for (int n = 0; n < L; ++n) thick[n] = (n == 0 || n == L - 1) ? 0.0 : s->layers[n].thickness;
  // dispersive layers need one stack per frequency; static ones share one
  bool dispersive = false;
  for (int n = 0; n < L; ++n) dispersive = dispersive || has_dispersion(*s, n, 1) || has_dispersion(*s, n, 2);
  const int nst = dispersive ? s->n_freq : 1;
  std::vector<rcwa_cplx> eps((size_t)nst * L * cells);
  std::vector<rcwa_stack> stacks(nst);
  std::vector<rcwa_point> pts(s->n_freq);
  std::vector<rcwa_cplx> pxy((size_t)s->n_freq * 4);
  for (int st = 0; st < nst; ++st) {
    const double omega = 2.0 * kPi * s->freq[st];
    for (int n = 0; n < L; ++n) {
      // makeLayer (sol/rcwa_bridge.cpp:72-89): eps1 inside [0,fill*px]x[0,fill_y*py]
      const std::complex<double> e1 = layer_eps(*s, n, 1, omega), e2 = layer_eps(*s, n, 2, omega);
      for (int j = 0; j + 1 < ncy; ++j) {
        const double yc = 0.5 * (ye[j] + ye[j + 1]);
        for (int i = 0; i + 1 < ncx; ++i) {
          const double xc = 0.5 * (xe[i] + xe[i + 1]);
          const bool in1 = (xc < s->layers[n].fill * xe.back()) && (yc < s->layers[n].fill_y * ye.back());
          const std::complex<double> v = in1 ? e1 : e2;
          eps[((size_t)st * L + n) * cells + (size_t)j * (ncx - 1) + i] = rcwa_cplx{v.real(), v.imag()};
        }
      }
    }
    rcwa_stack& sk = stacks[st];
    sk.nHx = s->nHx;
    sk.nHy = s->nHy;
    sk.ncx = ncx;
    sk.ncy = ncy;
    sk.cx = xe.data();
    sk.cy = ye.data();
    sk.n_layers = L;
    sk.eps = eps.data() + (size_t)st * L * cells;
    sk.thickness = thick.data();
  }
  std::vector<double> kx0(s->n_freq), ky0(s->n_freq), k0v(s->n_freq);
  std::vector<std::complex<double>> einc(s->n_freq), etrn(s->n_freq);
  for (int f = 0; f < s->n_freq; ++f) {
    const double lambda = kC0 / s->freq[f];
    const double k0 = 2.0 * kPi / lambda;
    const double omega = 2.0 * kPi * s->freq[f];
    einc[f] = layer_eps(*s, 0, 1, omega);
    etrn[f] = layer_eps(*s, L - 1, 1, omega);
    const double n_inc = std::max(std::sqrt(einc[f]).real(), 1e-6);  // :258-259
    kx0[f] = k0 * n_inc * std::sin(th) * std::cos(ph);               // :280-281
    ky0[f] = k0 * n_inc * std::sin(th) * std::sin(ph);
    k0v[f] = k0;
    pts[f] = rcwa_point{dispersive ? f : 0, lambda, kx0[f], ky0[f]};
    pxy[(size_t)f * 4 + 0] = rcwa_cplx{teX, 0.0};
    pxy[(size_t)f * 4 + 1] = rcwa_cplx{teY, 0.0};
    pxy[(size_t)f * 4 + 2] = rcwa_cplx{tmX, 0.0};
    pxy[(size_t)f * 4 + 3] = rcwa_cplx{tmY, 0.0};
  }
  const int nOrdX = 2 * s->nHx + 1, nOrdY = 2 * s->nHy + 1;
  const size_t nOrd = (size_t)nOrdX * nOrdY;
  std::vector<double> ref(ordR ? (size_t)s->n_freq * 2 * nOrd : 0), trn(ordT ? (size_t)s->n_freq * 2 * nOrd : 0);
  std::vector<double> RT((size_t)s->n_freq * 2), TT((size_t)s->n_freq * 2);
  std::vector<int> st_pts(s->n_freq, 0);
  const int rc = rcwa_engine_solve_batch(e, stacks.data(), nst, pts.data(), s->n_freq, 2, pxy.data(), RCWA_PREC_FP64,
                                         RT.data(), TT.data(), ordR ? ref.data() : nullptr,
                                         ordT ? trn.data() : nullptr, st_pts.data());
  if (rc != RCWA_OK && rc != st_pts[0]) {
    bool per_point = false;
    for (int v : st_pts) per_point = per_point || v != 0;
    if (!per_point) return rc;
  }
  for (int f = 0; f < s->n_freq; ++f) {
    R[2 * f] = RT[2 * f];
    R[2 * f + 1] = RT[2 * f + 1];
    T[2 * f] = TT[2 * f];
    T[2 * f + 1] = TT[2 * f + 1];
    if (status) status[f] = st_pts[f];
  }
  // masks of propagating orders (sol/rcwa_bridge.cpp:289-300), layout [pol][freq][order]
  if (ordR || ordT) {
    for (int f = 0; f < s->n_freq; ++f) {
      const double k0 = k0v[f];
      const double kr2 = k0 * k0 * einc[f].real(), kt2 = k0 * k0 * etrn[f].real();
      for (size_t k = 0; k < nOrd; ++k) {
        const int m = (int)(k / (size_t)nOrdY) - s->nHx;
        const int nn = (int)(k % (size_t)nOrdY) - s->nHy;
        const double kx = kx0[f] + 2.0 * kPi * m / s->period_x;
        const double ky = ky0[f] + 2.0 * kPi * nn / py_period;
        const double kt = kx * kx + ky * ky;
        for (int pol = 0; pol < 2; ++pol) {
          const size_t dst = ((size_t)pol * s->n_freq + f) * nOrd + k;
          const size_t src = ((size_t)f * 2 + pol) * nOrd + k;
          if (ordR) ordR[dst] = (kt < kr2) ? ref[src] : 0.0;
          if (ordT) ordT[dst] = (kt < kt2) ? trn[src] : 0.0;
        }
      }
    }
  }
  return rc;
}
