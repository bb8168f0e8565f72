// Host orchestration of the batched RCWA solve and the C ABI.
//
// A plan groups the points by their harmonic grid (nx, ny); each group is cut
// into chunks sized to the device memory budget.  For one chunk the device
// work is:
//   conv    per distinct (stack, patterned layer): fe11, fe22, fe33 -> E = fe33^-1
//   modes   per (point, patterned layer): X1 = E Da fe11, X2 = E Db fe22,
//           M = PQ/k0^2, eig(M) -> (mu, W), gamma, V = QW/keff; analytic
//           half-space modes per point
//   cascade per interface, bottom to top (rcwa/RCWASolver.cpp:378-492):
//           IE = Wa^-1 Wb, IH = Va^-1 Vb (below the uniform superstrate:
//           IE = Wb and a 2x2 solve per order), phase, F, G,
//           tau = (F+G)^-1, Rud = I - 2 G tau, Tdd = 2 waveTdd tau; in mixed
//           plans the products of points without a metallic layer run in
//           3xTF32 on the tensor cores, the others on the FP64 path
//   scatter per (point, excitation): per-order efficiencies and their sums.
// Every batched call receives device pointer arrays that the plan built once,
// so executing a plan is a fixed sequence of kernel launches on one stream.
// The LU schedules, the Schur crossover and the product path of each chunk
// come from the engine's schedule tuner or its built-in rules (tuner.cu).
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstring>
#include <functional>
#include <map>
#include <tuple>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include "eig.cuh"
#include "engine_internal.cuh"
#include "field.cuh"
#include "fourier.cuh"
#include "linalg.cuh"
#include "gemm_tc.cuh"
#include "rcwa_kernels.cuh"
#include "lu_blocked.cuh"
#include "tuner.cuh"


namespace {

constexpr double kPi = 3.1415926535897932;

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  bool borrowed = false;          // the engine's cached workspace, not freed here
  rcwa_engine* pool = nullptr;    // block from the engine's pool: returned there
  size_t cap = 0;                 // pooled block size
  bool take(rcwa_engine* e, size_t n) {
    p = engine_take_block(e, n, &cap);
    if (!p) return false;
    pool = e;
    bytes = n;
    return true;
  }
  ~DevBuf() {
    if (!p || borrowed) return;
    if (pool) engine_release_block(pool, p, cap);
    else cudaFree(p);
  }
};

// pooled blocks: up to 64 MB each, 512 MB in total per engine
constexpr size_t kPoolBlockMax = (size_t)64 << 20;
constexpr size_t kPoolTotalMax = (size_t)512 << 20;

// Bump allocator over byte offsets; turned into addresses once the base exists.
struct Layout {
  size_t off = 0;
  size_t take(size_t bytes) {
    size_t o = (off + 255) & ~(size_t)255;
    off = o + bytes;
    return o;
  }
};

// Host-side staging of plan metadata (item structs and pointer arrays) that is
// uploaded in one copy.  Entries are recorded as offsets.
struct Meta {
  std::vector<unsigned char> bytes;
  size_t add(const void* src, size_t n) {
    size_t o = (bytes.size() + 15) & ~(size_t)15;
    bytes.resize(o + n);
    if (n) std::memcpy(bytes.data() + o, src, n);
    return o;
  }
  template <class T>
  size_t add_vec(const std::vector<T>& v) { return add(v.data(), v.size() * sizeof(T)); }
};

struct StackInfo {
  int nx, ny, N, L;
  double Lx, Ly;
  std::vector<double> cx, cy;
  std::vector<cplx> eps;   // L * cells
  // relative permeability (L * cells) when some layer is magnetic, else
  // empty; mag[l]: layer l has a cell with |mu - 1| > 1e-12 (Layer::Layer,
  // rcwa/Layer.cpp:64-71)
  std::vector<cplx> mu;
  std::vector<char> mag;
  std::vector<double> thick;
  // a half-space whose cells differ (incidence side, transmission side): its
  // modes come from the eigensolver like a patterned layer's, as in the
  // reference, which solves every layer type (rcwa/RCWASolver.cpp:194-210)
  char pat0 = 0, patL = 0;
  int ncx, ncy;
  // stacks given by Laurent tables: one (2nx-1) x (2ny-1) table per
  // patterned layer (layers 1..L-2); the cell grid is then one cell per layer
  bool tables = false;
  std::vector<cplx> f2d;
};

}  // namespace

struct rcwa_plan {
  rcwa_engine* e = nullptr;
  int n_pts = 0, n_exc = 0;
  std::vector<int> point_N;            // orders per point
  std::vector<size_t> order_offset;    // per point, into ref/trn outputs
  size_t total_orders = 0;
  DevBuf inputs, meta, work, outputs;
  double* dR = nullptr;
  double* dT = nullptr;
  double* dRef = nullptr;
  double* dTrn = nullptr;
  int* dStatus = nullptr;
  int* dTcErr = nullptr;   // set when a tensor-core completion wait ran out
  int* dTcScale = nullptr; // operand scale exponents of the tensor-core products (2 x 2048)
  // per chunk: n, points, interface LU schedule, tau LU schedule, Schur
  // crossover, product path (0: 3xTF32 on 128 x 128 tiles, 1: FP64 tensor
  // path, 2: 3xTF32 on 128 x 256 tiles)
  std::vector<std::array<int, 6>> sched;
  int precision = RCWA_PREC_FP64;
  std::vector<std::function<cudaError_t(cudaStream_t, StageProf&)>> steps;
  long long launches = 0;
  std::unique_ptr<StageProf> prof{new StageProf()};
  // scatter items of a single-chunk plan, kept for rcwa_plan_rescatter
  int chunks = 0;
  std::vector<ScatterItem> scatter_items;
  size_t scatter_meta = 0;
  int scatter_N = 0, scatter_nx = 0, scatter_ny = 0;
  // launch sequence as a CUDA graph, captured on the second execution
  cudaGraphExec_t graph_exec = nullptr;
  bool graph_prof = false;   // the graph holds the stage-timing event records
  long long graph_launches = 0;
  long long executions = 0;
  // per point: the device data the fields inside the stack need (valid for
  // single-chunk plans, whose workspace holds every point after execution)
  std::vector<FieldPoint> field_pts;
  ~rcwa_plan() {
    // kernels of this plan may still run on a caller's stream; its pooled
    // blocks and the borrowed workspace go back to the engine only after them
    cudaDeviceSynchronize();
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (work.borrowed && e) e->work_cache_busy = false;
  }
};

namespace {

int fail(rcwa_engine* e, int code, const std::string& msg) {
  if (e) e->last_error = msg;
  return code;
}

bool finite_c(const rcwa_cplx& z) { return std::isfinite(z.re) && std::isfinite(z.im); }

int validate_stack(const rcwa_stack& s, std::string& why) {
  if (s.nHx < 0 || s.nHy < 0) { why = "negative harmonic count"; return RCWA_ERR_INVALID; }
  if (s.ncx < 2 || s.ncy < 2 || !s.cx || !s.cy) { why = "need >= 2 cell edges per axis"; return RCWA_ERR_INVALID; }
  if (s.n_layers < 2 || !s.eps || !s.thickness) { why = "need >= 2 layers"; return RCWA_ERR_INVALID; }
  for (int i = 0; i + 1 < s.ncx; ++i)
    if (!(s.cx[i + 1] >= s.cx[i]) || !std::isfinite(s.cx[i + 1])) { why = "x edges must ascend"; return RCWA_ERR_INVALID; }
  for (int i = 0; i + 1 < s.ncy; ++i)
    if (!(s.cy[i + 1] >= s.cy[i]) || !std::isfinite(s.cy[i + 1])) { why = "y edges must ascend"; return RCWA_ERR_INVALID; }
  if (!(s.cx[s.ncx - 1] > s.cx[0]) || !(s.cy[s.ncy - 1] > s.cy[0])) { why = "zero period"; return RCWA_ERR_INVALID; }
  const size_t cells = (size_t)(s.ncx - 1) * (s.ncy - 1);
  for (int l = 0; l < s.n_layers; ++l) {
    for (size_t c = 0; c < cells; ++c) {
      const rcwa_cplx z = s.eps[(size_t)l * cells + c];
      if (!finite_c(z)) { why = "non-finite permittivity"; return RCWA_ERR_NONFINITE; }
      if (z.re == 0.0 && z.im == 0.0) { why = "zero permittivity"; return RCWA_ERR_INVALID; }
    }
    if (s.mu)
      for (size_t c = 0; c < cells; ++c) {
        const rcwa_cplx z = s.mu[(size_t)l * cells + c];
        if (!finite_c(z)) { why = "non-finite permeability"; return RCWA_ERR_NONFINITE; }
        if (z.re == 0.0 && z.im == 0.0) { why = "zero permeability"; return RCWA_ERR_INVALID; }
      }
    if (l > 0 && l < s.n_layers - 1 && (!std::isfinite(s.thickness[l]) || s.thickness[l] < 0)) {
      why = "invalid thickness";
      return RCWA_ERR_INVALID;
    }
  }
  return RCWA_OK;
}

StackInfo make_stack_info(const rcwa_stack& s) {
  StackInfo si;
  si.nx = 2 * s.nHx + 1;
  si.ny = 2 * s.nHy + 1;
  si.N = si.nx * si.ny;
  si.L = s.n_layers;
  si.ncx = s.ncx;
  si.ncy = s.ncy;
  si.cx.assign(s.cx, s.cx + s.ncx);
  si.cy.assign(s.cy, s.cy + s.ncy);
  si.Lx = si.cx.back() - si.cx.front();
  si.Ly = si.cy.back() - si.cy.front();
  const size_t cells = (size_t)(s.ncx - 1) * (s.ncy - 1);
  si.eps.resize(cells * s.n_layers);
  for (size_t i = 0; i < si.eps.size(); ++i) si.eps[i] = mkc(s.eps[i].re, s.eps[i].im);
  si.thick.assign(s.thickness, s.thickness + s.n_layers);
  si.mag.assign(s.n_layers, 0);
  bool any = false;
  if (s.mu)
    for (int l = 0; l < s.n_layers; ++l)
      for (size_t c = 0; c < cells; ++c) {
        const rcwa_cplx z = s.mu[(size_t)l * cells + c];
        if (std::hypot(z.re - 1.0, z.im) > 1e-12) { si.mag[l] = 1; any = true; break; }
      }
  if (any) {
    si.mu.resize(cells * s.n_layers);
    for (size_t i = 0; i < si.mu.size(); ++i) si.mu[i] = mkc(s.mu[i].re, s.mu[i].im);
  }
  for (int side = 0; side < 2; ++side) {
    const size_t l = side == 0 ? 0 : (size_t)s.n_layers - 1;
    bool pat = false;
    for (size_t c = 1; c < cells && !pat; ++c) {
      const rcwa_cplx z = s.eps[l * cells + c], z0 = s.eps[l * cells];
      pat = z.re != z0.re || z.im != z0.im;
      if (s.mu) {
        const rcwa_cplx m = s.mu[l * cells + c], m0 = s.mu[l * cells];
        pat = pat || m.re != m0.re || m.im != m0.im;
      }
    }
    (side == 0 ? si.pat0 : si.patL) = pat ? 1 : 0;
  }
  return si;
}

// layers whose modes come from the eigensolver: the patterned layers, and a
// half-space whose cells differ
std::vector<int> eig_layers(const StackInfo& si) {
  std::vector<int> ls;
  if (si.pat0) ls.push_back(0);
  for (int l = 1; l + 1 < si.L; ++l) ls.push_back(l);
  if (si.patL && si.L > 1) ls.push_back(si.L - 1);
  return ls;
}

// Layer::eps(x, y) / Layer::mu(x, y): the cell containing (x, y), x periodic,
// y outside the grid gives 0 (rcwa/Layer.cpp:383-450); used for the
// efficiencies of a patterned half-space (scatterPlaneWave takes its values
// at (0, 0), rcwa/RCWASolver.cpp:1823-1827)
cplx cell_value(const StackInfo& si, const std::vector<cplx>& f, int l, double x, double y) {
  const double Lx = si.cx.back() - si.cx.front();
  while (x < si.cx.front()) x += Lx;
  while (x > si.cx.back()) x -= Lx;
  if (y < si.cy.front() || y > si.cy.back()) return mkc(0.0, 0.0);
  int ix = 0, iy = 0;
  for (int i = 0; i + 1 < si.ncx; ++i)
    if (x <= si.cx[i + 1]) { ix = i; break; }
  for (int j = 0; j + 1 < si.ncy; ++j)
    if (y <= si.cy[j + 1]) { iy = j; break; }
  return f[(size_t)l * (si.ncx - 1) * (si.ncy - 1) + (size_t)iy * (si.ncx - 1) + ix];
}

bool is_mag(const StackInfo& si, int l) { return !si.mag.empty() && si.mag[l]; }

// conv jobs of a layer's permeability are keyed (stack, layer + kMuJob)
constexpr int kMuJob = 1 << 20;

// relative permeability of a uniform layer (the half-spaces): 1 unless given
cplx layer_mu0(const StackInfo& si, int l) {
  if (si.mu.empty()) return mkc(1.0, 0.0);
  return si.mu[(size_t)l * (si.ncx - 1) * (si.ncy - 1)];
}

// alpha/beta of RCWASolver::evaluateAlphaBeta (rcwa/RCWASolver.cpp:242-266):
// mode k = ny*i + j, alpha = 2 pi (i - Nx)/Lx + kx0, beta = 2 pi (j - Ny)/Ly + ky0.
void alpha_beta(const StackInfo& si, double kx0, double ky0, cplx* ab) {
  const int Nx = (si.nx - 1) / 2, Ny = (si.ny - 1) / 2;
  const double Kx = 2 * kPi / si.Lx, Ky = 2 * kPi / si.Ly;
  for (int i = 0; i < si.nx; ++i)
    for (int j = 0; j < si.ny; ++j) {
      const double m = i - Nx, n = j - Ny;
      ab[si.ny * i + j] = mkc(Kx * m + kx0, 0.0);
      ab[si.N + si.ny * i + j] = mkc(Ky * n + ky0, 0.0);
    }
}


}  // namespace

void* engine_take_block(rcwa_engine* e, size_t bytes, size_t* got) {
  bytes = (bytes + 4095) & ~(size_t)4095;
  {
    std::lock_guard<std::mutex> lk(e->pool_mu);
    int best = -1;
    for (int i = 0; i < (int)e->block_pool.size(); ++i) {
      const size_t sz = e->block_pool[i].second;
      if (sz >= bytes && sz <= 4 * bytes + ((size_t)1 << 20) && (best < 0 || sz < e->block_pool[best].second))
        best = i;
    }
    if (best >= 0) {
      void* p = e->block_pool[best].first;
      *got = e->block_pool[best].second;
      e->block_pool_bytes -= *got;
      e->block_pool.erase(e->block_pool.begin() + best);
      return p;
    }
  }
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  *got = bytes;
  return p;
}

void engine_release_block(rcwa_engine* e, void* p, size_t bytes) {
  {
    std::lock_guard<std::mutex> lk(e->pool_mu);
    if (bytes <= kPoolBlockMax && e->block_pool_bytes + bytes <= kPoolTotalMax) {
      e->block_pool.push_back({p, bytes});
      e->block_pool_bytes += bytes;
      return;
    }
  }
  cudaFree(p);
}

// ------------------------------------------------------------------ C ABI
extern "C" {

const char* rcwa_status_string(int status) {
  switch (status) {
    case RCWA_OK: return "ok";
    case RCWA_ERR_INVALID: return "invalid argument";
    case RCWA_ERR_CUDA: return "CUDA error";
    case RCWA_ERR_NOCONV: return "eigenvalue iteration did not converge";
    case RCWA_ERR_SINGULAR: return "singular matrix";
    case RCWA_ERR_NONFINITE: return "non-finite result";
    case RCWA_ERR_GRAZING: return "grazing / zero kz";
    case RCWA_ERR_NOMEM: return "out of device memory";
    case RCWA_ERR_NODEVICE: return "no CUDA device";
    case RCWA_ERR_UNSUPPORTED: return "unsupported input";
    default: return "unknown status";
  }
}

int rcwa_engine_create(int device, rcwa_engine** out) {
  if (!out) return RCWA_ERR_INVALID;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= device || device < 0) return RCWA_ERR_NODEVICE;
  if (cudaSetDevice(device) != cudaSuccess) return RCWA_ERR_NODEVICE;
  auto* e = new rcwa_engine();
  e->device = device;
  if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete e;
    return RCWA_ERR_CUDA;
  }
  *out = e;
  return RCWA_OK;
}

void rcwa_engine_destroy(rcwa_engine* e) {
  if (!e) return;
  cudaSetDevice(e->device);
  cudaDeviceSynchronize();
  for (auto& b : e->block_pool) cudaFree(b.first);
  e->block_pool.clear();
  if (e->work_cache) cudaFree(e->work_cache);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

const char* rcwa_engine_last_error(const rcwa_engine* e) { return e ? e->last_error.c_str() : ""; }

}  // extern "C"

namespace {

// Workspace offsets of one chunk (relative to the workspace base).
struct ChunkWork {
  // conv
  std::vector<int> conv_stack, conv_layer;       // per conv job
  std::map<std::pair<int, int>, int> conv_index;  // (stack, layer) -> job
  size_t conv_jobs_off = 0, fe11 = 0, fe22 = 0, fe33 = 0, Einv = 0, tab = 0, tab_elems = 0;
  size_t tptr = 0, tipiv = 0, tinfo = 0, cipiv = 0, cinfo = 0, convptr = 0;
  int max_ncx = 2, max_ncy = 2;
  // layer jobs
  std::vector<int> job_point, job_layer;          // per layer job (chunk-local point)
  size_t X1 = 0, X2 = 0, M = 0, W = 0, V = 0, mu = 0, gam = 0, eigw = 0, einfo = 0;
  // per point
  std::vector<int> points;                        // global point index
  size_t hW0 = 0, hV0 = 0, hWL = 0, hVL = 0, hg0 = 0, hgL = 0;
  size_t Rud = 0, Tdd = 0, F = 0, G = 0, tau = 0, IE = 0, IH = 0, WLU = 0, VLU = 0, pipiv = 0, pinfo = 0;
  size_t planes = 0, planes_bytes = 0;  // mixed plans: pre-split TF32 planes of one batched product
  size_t total = 0;
  // mixed plans: per chunk point, whether its products stay FP64 (its stack
  // has a layer with Re(eps) < 0, whose cascade the 3xTF32 products cannot
  // resolve)
  std::vector<char> fp64_pt;
  // schedules (tuner or built-in rules): LU of the interface and tau
  // factorisations, Schur crossover, product path of mixed plans
  int lu_if = -1, lu_tau = -1, ms_min = kSchurCrossover, prod = 0;
};

}  // namespace

static size_t chunk_layout(ChunkWork& c, const std::vector<StackInfo>& stacks, int N, bool mixed) {
  const size_t n = 2 * (size_t)N;
  const size_t NN = (size_t)N * N, nn = n * n;
  const size_t cs = sizeof(cplx);
  Layout L;
  const size_t nconv = c.conv_stack.size();
  const int nx = stacks[c.conv_stack.empty() ? 0 : c.conv_stack[0]].nx;
  const int ny = stacks[c.conv_stack.empty() ? 0 : c.conv_stack[0]].ny;
  c.tab_elems = conv_table_elems(nx, ny, c.max_ncx, c.max_ncy);
  const size_t strips = (size_t)std::max(c.max_ncx - 1, c.max_ncy - 1);
  c.conv_jobs_off = L.take(sizeof(ConvJob) * std::max<size_t>(nconv, 1));
  c.fe11 = L.take(cs * NN * nconv);
  c.fe22 = L.take(cs * NN * nconv);
  c.fe33 = L.take(cs * NN * nconv);
  c.Einv = L.take(cs * NN * nconv);
  c.tab = L.take(cs * c.tab_elems * nconv);
  c.tptr = L.take(sizeof(void*) * 4 * strips * std::max<size_t>(nconv, 1));
  c.tipiv = L.take(sizeof(int) * strips * std::max(nx, ny) * std::max<size_t>(nconv, 1));
  c.tinfo = L.take(sizeof(int) * strips * std::max<size_t>(nconv, 1));
  c.cipiv = L.take(sizeof(int) * N * std::max<size_t>(nconv, 1));
  c.cinfo = L.take(sizeof(int) * std::max<size_t>(nconv, 1));
  const size_t nj = c.job_point.size();
  c.X1 = L.take(cs * NN * nj);
  c.X2 = L.take(cs * NN * nj);
  c.M = L.take(cs * nn * nj);
  c.W = L.take(cs * nn * nj);
  c.V = L.take(cs * nn * nj);
  c.mu = L.take(cs * n * nj);
  c.gam = L.take(cs * n * nj);
  c.eigw = L.take(zgeev_workspace_bytes((int)n) * nj);
  c.einfo = L.take(sizeof(int) * std::max<size_t>(nj, 1));
  const size_t np = c.points.size();
  c.hW0 = L.take(cs * nn * np);
  c.hV0 = L.take(cs * nn * np);
  c.hWL = L.take(cs * nn * np);
  c.hVL = L.take(cs * nn * np);
  c.hg0 = L.take(cs * n * np);
  c.hgL = L.take(cs * n * np);
  c.Rud = L.take(cs * nn * np);
  c.Tdd = L.take(cs * nn * np);
  c.F = L.take(cs * nn * np);
  c.G = L.take(cs * nn * np);
  c.tau = L.take(cs * nn * np);
  c.IE = L.take(cs * nn * np);
  c.IH = L.take(cs * nn * np);
  c.WLU = L.take(cs * nn * np);
  c.VLU = L.take(cs * nn * np);
  c.pipiv = L.take(sizeof(int) * n * 3 * np);
  c.pinfo = L.take(sizeof(int) * 3 * np);
  c.planes_bytes = mixed ? zgemm_tf32x3_planes_bytes((int)n, (int)n, (int)n, (int)np) : 0;
  c.planes = L.take(std::max<size_t>(c.planes_bytes, 16));
  c.total = L.off;
  return L.off;
}

// Lm: magnetic layers of the stack, each with a second set of four
// convolution matrices (the permeability's)
static size_t chunk_bytes_per_point(int N, int Lp, int Lm, bool mixed) {
  const double n = 2.0 * N;
  const double nn = n * n * sizeof(cplx), NN = (double)N * N * sizeof(cplx);
  const double per_job = 2 * NN + 3 * nn + zgeev_workspace_bytes((int)n) + 4 * NN;
  const double planes = mixed ? (double)zgemm_tf32x3_planes_bytes((int)n, (int)n, (int)n, 1) : 0.0;
  return (size_t)(13 * nn + planes + per_job * std::max(Lp - 2, 0) + 4 * NN * Lm);
}

namespace {
int plan_create_impl(rcwa_engine* e, const std::vector<StackInfo>& si, const rcwa_point* pts, int n_pts, int n_exc,
                     const rcwa_cplx* pxy, int precision, rcwa_plan** out);

// A Laurent-table stack as a StackInfo: a one-cell grid per layer (the
// half-spaces' permittivity, the patterned layers' mean permittivity, which
// only decides whether a mixed plan keeps FP64 products for the stack) and
// the tables themselves.
int table_stack_info(const rcwa_table_stack& t, StackInfo& si, std::string& why) {
  if (t.nHx < 0 || t.nHy < 0) { why = "negative harmonic count"; return RCWA_ERR_INVALID; }
  if (!(t.Lx > 0) || !(t.Ly > 0) || !std::isfinite(t.Lx) || !std::isfinite(t.Ly)) {
    why = "invalid period";
    return RCWA_ERR_INVALID;
  }
  if (t.n_layers < 2 || !t.eps_half || !t.thickness || (t.n_layers > 2 && !t.f2d)) {
    why = "need >= 2 layers and their tables";
    return RCWA_ERR_INVALID;
  }
  si = StackInfo();
  si.nx = 2 * t.nHx + 1;
  si.ny = 2 * t.nHy + 1;
  si.N = si.nx * si.ny;
  si.L = t.n_layers;
  si.ncx = si.ncy = 2;
  si.cx = {0.0, t.Lx};
  si.cy = {0.0, t.Ly};
  si.Lx = t.Lx;
  si.Ly = t.Ly;
  si.tables = true;
  const size_t tab = (size_t)(2 * si.nx - 1) * (2 * si.ny - 1);
  si.f2d.resize(tab * (size_t)(t.n_layers - 2));
  for (size_t i = 0; i < si.f2d.size(); ++i) {
    if (!finite_c(t.f2d[i])) { why = "non-finite Laurent coefficient"; return RCWA_ERR_NONFINITE; }
    si.f2d[i] = mkc(t.f2d[i].re, t.f2d[i].im);
  }
  si.eps.resize(t.n_layers);
  for (int side = 0; side < 2; ++side) {
    const rcwa_cplx z = t.eps_half[side];
    if (!finite_c(z)) { why = "non-finite permittivity"; return RCWA_ERR_NONFINITE; }
    if (z.re == 0.0 && z.im == 0.0) { why = "zero permittivity"; return RCWA_ERR_INVALID; }
    si.eps[side == 0 ? 0 : t.n_layers - 1] = mkc(z.re, z.im);
  }
  const size_t mid = (size_t)(si.nx - 1) * (2 * si.ny - 1) + (si.ny - 1);  // F2D[0][0]
  for (int l = 1; l + 1 < t.n_layers; ++l) si.eps[l] = si.f2d[(size_t)(l - 1) * tab + mid];
  si.thick.assign(t.thickness, t.thickness + t.n_layers);
  for (int l = 1; l + 1 < t.n_layers; ++l)
    if (!std::isfinite(si.thick[l]) || si.thick[l] < 0) { why = "invalid thickness"; return RCWA_ERR_INVALID; }
  return RCWA_OK;
}
}  // namespace

extern "C" int rcwa_plan_create(rcwa_engine* e, const rcwa_stack* stacks, int n_stacks, const rcwa_point* pts,
                                int n_pts, int n_exc, const rcwa_cplx* pxy, int precision, rcwa_plan** out) {
  if (!e || !out) return RCWA_ERR_INVALID;
  *out = nullptr;
  if (n_stacks <= 0 || !stacks || n_pts <= 0 || !pts || n_exc <= 0 || !pxy)
    return fail(e, RCWA_ERR_INVALID, "empty batch or null pointer");
  std::vector<StackInfo> si;
  for (int s = 0; s < n_stacks; ++s) {
    std::string why;
    int rc = validate_stack(stacks[s], why);
    if (rc) return fail(e, rc, "stack " + std::to_string(s) + ": " + why);
    si.push_back(make_stack_info(stacks[s]));
  }
  return plan_create_impl(e, si, pts, n_pts, n_exc, pxy, precision, out);
}

extern "C" int rcwa_plan_create_tables(rcwa_engine* e, const rcwa_table_stack* stacks, int n_stacks,
                                       const rcwa_point* pts, int n_pts, int n_exc, const rcwa_cplx* pxy,
                                       int precision, rcwa_plan** out) {
  if (!e || !out) return RCWA_ERR_INVALID;
  *out = nullptr;
  if (n_stacks <= 0 || !stacks || n_pts <= 0 || !pts || n_exc <= 0 || !pxy)
    return fail(e, RCWA_ERR_INVALID, "empty batch or null pointer");
  std::vector<StackInfo> si(n_stacks);
  for (int s = 0; s < n_stacks; ++s) {
    std::string why;
    int rc = table_stack_info(stacks[s], si[s], why);
    if (rc) return fail(e, rc, "stack " + std::to_string(s) + ": " + why);
  }
  return plan_create_impl(e, si, pts, n_pts, n_exc, pxy, precision, out);
}

namespace {
int plan_create_impl(rcwa_engine* e, const std::vector<StackInfo>& si, const rcwa_point* pts, int n_pts, int n_exc,
                     const rcwa_cplx* pxy, int precision, rcwa_plan** out) {
  const int n_stacks = (int)si.size();
  if (precision != RCWA_PREC_FP64 && precision != RCWA_PREC_MIXED)
    return fail(e, RCWA_ERR_INVALID, "unknown precision mode");
  if (cudaSetDevice(e->device) != cudaSuccess) return fail(e, RCWA_ERR_CUDA, "cudaSetDevice failed");
  for (int p = 0; p < n_pts; ++p) {
    const rcwa_point& q = pts[p];
    if (q.stack < 0 || q.stack >= n_stacks) return fail(e, RCWA_ERR_INVALID, "point stack index out of range");
    if (!(q.lambda > 0) || !std::isfinite(q.lambda) || !std::isfinite(q.kx0) || !std::isfinite(q.ky0))
      return fail(e, RCWA_ERR_INVALID, "invalid wavelength or Bloch vector");
  }
  std::unique_ptr<rcwa_plan> P(new rcwa_plan());
  P->e = e;
  P->n_pts = n_pts;
  P->precision = precision;
  P->n_exc = n_exc;
  P->point_N.resize(n_pts);
  P->order_offset.resize(n_pts);
  size_t acc = 0;
  for (int p = 0; p < n_pts; ++p) {
    P->point_N[p] = si[pts[p].stack].N;
    P->order_offset[p] = acc;
    acc += (size_t)n_exc * P->point_N[p];
  }
  P->total_orders = acc;

  // ---- inputs: stack arrays and per-point alpha/beta
  Layout il;
  std::vector<size_t> cx_off(n_stacks), cy_off(n_stacks), eps_off(n_stacks), f2d_off(n_stacks), mu_off(n_stacks);
  for (int s = 0; s < n_stacks; ++s) {
    cx_off[s] = il.take(sizeof(double) * si[s].cx.size());
    cy_off[s] = il.take(sizeof(double) * si[s].cy.size());
    eps_off[s] = il.take(sizeof(cplx) * si[s].eps.size());
    f2d_off[s] = il.take(sizeof(cplx) * si[s].f2d.size());
    mu_off[s] = il.take(sizeof(cplx) * si[s].mu.size());
  }
  std::vector<size_t> ab_off(n_pts);
  for (int p = 0; p < n_pts; ++p) ab_off[p] = il.take(sizeof(cplx) * 2 * P->point_N[p]);
  if (!P->inputs.take(e, il.off)) return fail(e, RCWA_ERR_NOMEM, "input allocation failed");
  {
    std::vector<unsigned char> h(il.off);
    for (int s = 0; s < n_stacks; ++s) {
      std::memcpy(h.data() + cx_off[s], si[s].cx.data(), sizeof(double) * si[s].cx.size());
      std::memcpy(h.data() + cy_off[s], si[s].cy.data(), sizeof(double) * si[s].cy.size());
      std::memcpy(h.data() + eps_off[s], si[s].eps.data(), sizeof(cplx) * si[s].eps.size());
      if (!si[s].f2d.empty()) std::memcpy(h.data() + f2d_off[s], si[s].f2d.data(), sizeof(cplx) * si[s].f2d.size());
      if (!si[s].mu.empty()) std::memcpy(h.data() + mu_off[s], si[s].mu.data(), sizeof(cplx) * si[s].mu.size());
    }
    for (int p = 0; p < n_pts; ++p) alpha_beta(si[pts[p].stack], pts[p].kx0, pts[p].ky0, (cplx*)(h.data() + ab_off[p]));
    if (cudaMemcpy(P->inputs.p, h.data(), il.off, cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(e, RCWA_ERR_CUDA, "input upload failed");
  }
  char* inb = (char*)P->inputs.p;

  // ---- outputs
  {
    Layout ol;
    size_t oR = ol.take(sizeof(double) * n_pts * n_exc), oT = ol.take(sizeof(double) * n_pts * n_exc);
    size_t oRef = ol.take(sizeof(double) * std::max<size_t>(acc, 1)), oTrn = ol.take(sizeof(double) * std::max<size_t>(acc, 1));
    size_t oS = ol.take(sizeof(int) * n_pts);
    size_t oE = ol.take(sizeof(int));
    size_t oSc = ol.take(sizeof(int) * 2 * 2048);
    if (!P->outputs.take(e, ol.off)) return fail(e, RCWA_ERR_NOMEM, "output allocation failed");
    char* b = (char*)P->outputs.p;
    P->dR = (double*)(b + oR);
    P->dT = (double*)(b + oT);
    P->dRef = (double*)(b + oRef);
    P->dTrn = (double*)(b + oTrn);
    P->dStatus = (int*)(b + oS);
    P->dTcErr = (int*)(b + oE);
    P->dTcScale = (int*)(b + oSc);
  }

  // ---- chunking: group by (nx, ny), then fill chunks up to the memory budget
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  if (!e->work_cache_busy) free_b += e->work_cache_bytes;
  const size_t budget = std::min<size_t>((size_t)(0.6 * free_b), (size_t)96 << 30);
  // In mixed plans, stacks with a metallic layer (Re(eps) < 0 in some cell)
  // keep FP64 products: the evanescent modes of such layers make the cascade
  // ill-conditioned beyond what 3xTF32 (about 21 bits) can carry.  They share
  // chunks with the other points; each cascade product is then two batched
  // calls, one per precision.
  std::vector<char> metallic(n_stacks, 0);
  for (int s = 0; s < n_stacks; ++s) {
    for (const cplx& z : si[s].eps)
      if (z.x < 0.0) { metallic[s] = 1; break; }
    for (const cplx& z : si[s].mu)
      if (z.x < 0.0) { metallic[s] = 1; break; }
  }
  std::map<std::tuple<int, int, int>, std::vector<int>> groups;
  for (int p = 0; p < n_pts; ++p) {
    const int s = pts[p].stack;
    groups[{si[s].nx, si[s].ny, 0}].push_back(p);
  }
  std::vector<ChunkWork> chunks;
  std::vector<int> chunk_N;
  for (auto& g : groups) {
    const int N = std::get<0>(g.first) * std::get<1>(g.first);
    size_t used = 0;
    ChunkWork cur;
    auto flush = [&]() {
      if (!cur.points.empty()) {
        for (int p : cur.points) cur.fp64_pt.push_back(precision == RCWA_PREC_MIXED ? metallic[pts[p].stack] : 1);
        chunks.push_back(cur);
        chunk_N.push_back(N);
      }
      cur = ChunkWork();
      used = 0;
    };
    for (int p : g.second) {
      const StackInfo& sp = si[pts[p].stack];
      const int Lm = (int)std::count(sp.mag.begin(), sp.mag.end(), (char)1);
      const size_t need = chunk_bytes_per_point(N, sp.L + sp.pat0 + sp.patL, Lm, precision == RCWA_PREC_MIXED);
      if (!cur.points.empty() && (used + need > budget || cur.points.size() >= 1024)) flush();
      cur.points.push_back(p);
      used += need;
    }
    flush();
  }
  // conv jobs and layer jobs per chunk
  for (auto& c : chunks) {
    for (size_t lp = 0; lp < c.points.size(); ++lp) {
      const int p = c.points[lp];
      const int s = pts[p].stack;
      c.max_ncx = std::max(c.max_ncx, si[s].ncx);
      c.max_ncy = std::max(c.max_ncy, si[s].ncy);
      for (int l : eig_layers(si[s])) {
        for (int k = 0; k < (is_mag(si[s], l) ? 2 : 1); ++k) {
          auto key = std::make_pair(s, l + k * kMuJob);
          if (!c.conv_index.count(key)) {
            c.conv_index[key] = (int)c.conv_stack.size();
            c.conv_stack.push_back(s);
            c.conv_layer.push_back(l + k * kMuJob);
          }
        }
        c.job_point.push_back((int)lp);
        c.job_layer.push_back(l);
      }
    }
  }
  // schedules of each chunk's large operations (may time candidates on the
  // device when the engine's tuner measures on a miss)
  for (size_t ci = 0; ci < chunks.size(); ++ci) {
    ChunkWork& c = chunks[ci];
    const int n = 2 * chunk_N[ci], np = (int)c.points.size(), nj = (int)c.job_point.size();
    c.lu_if = tune_resolve(e, kTuneLU, n, 2 * np);
    c.lu_tau = tune_resolve(e, kTuneLU, n, np);
    if (nj > 0) c.ms_min = tune_resolve(e, kTuneSchur, n, nj);
    int n_tc = 0;
    for (char f : c.fp64_pt) n_tc += f ? 0 : 1;
    c.prod = n_tc > 0 ? tune_resolve(e, kTuneProduct, n, n_tc) : 1;
    P->sched.push_back({n, np, c.lu_if, c.lu_tau, c.ms_min, c.prod});
  }
  size_t wbytes = 0;
  for (size_t ci = 0; ci < chunks.size(); ++ci)
    wbytes = std::max(wbytes, chunk_layout(chunks[ci], si, chunk_N[ci], precision == RCWA_PREC_MIXED));
  const size_t wneed = std::max<size_t>(wbytes, 256);
  if (!e->work_cache_busy) {
    if (e->work_cache_bytes < wneed) {
      if (e->work_cache) cudaFree(e->work_cache);
      e->work_cache = nullptr;
      e->work_cache_bytes = 0;
      if (cudaMalloc(&e->work_cache, wneed) != cudaSuccess) {
        e->work_cache = nullptr;
        return fail(e, RCWA_ERR_NOMEM, "workspace allocation failed (" + std::to_string(wbytes >> 20) + " MiB)");
      }
      e->work_cache_bytes = wneed;
    }
    P->work.p = e->work_cache;
    P->work.borrowed = true;
    e->work_cache_busy = true;
  } else if (cudaMalloc(&P->work.p, wneed) != cudaSuccess) {
    P->work.p = nullptr;
    return fail(e, RCWA_ERR_NOMEM, "workspace allocation failed (" + std::to_string(wbytes >> 20) + " MiB)");
  }
  P->work.bytes = wbytes;
  char* wb = (char*)P->work.p;

  // ---- metadata (items and pointer arrays) per chunk, and the launch steps
  Meta meta;
  rcwa_plan* plan = P.get();
  const bool same_conv_as_prev_possible = true;
  std::vector<std::pair<int, int>> prev_conv_keys;
  int prev_N = -1;

  for (size_t ci = 0; ci < chunks.size(); ++ci) {
    ChunkWork& c = chunks[ci];
    const int N = chunk_N[ci];
    const int n = 2 * N;
    const size_t NN = (size_t)N * N, nn = (size_t)n * n;
    const StackInfo& s0 = si[pts[c.points[0]].stack];
    const int nx = s0.nx, ny = s0.ny;
    auto W_ = [&](size_t off) { return (cplx*)(wb + off); };
    const int nconv = (int)c.conv_stack.size();
    const int nj = (int)c.job_point.size();
    const int np = (int)c.points.size();

    // ---------------- conv
    std::vector<std::pair<int, int>> keys;
    for (int j = 0; j < nconv; ++j) keys.push_back({c.conv_stack[j], c.conv_layer[j]});
    const bool reuse_conv = same_conv_as_prev_possible && prev_N == N && keys == prev_conv_keys && ci > 0 &&
                            chunks[ci - 1].conv_jobs_off == c.conv_jobs_off && chunks[ci - 1].tab_elems == c.tab_elems;
    prev_conv_keys = keys;
    prev_N = N;
    if (nconv > 0 && !reuse_conv) {
      std::vector<ConvJob> jobs(nconv);
      for (int j = 0; j < nconv; ++j) {
        const int s = c.conv_stack[j], lk = c.conv_layer[j];
        const bool of_mu = lk >= kMuJob;
        const int l = of_mu ? lk - kMuJob : lk;
        const size_t cells = (size_t)(si[s].ncx - 1) * (si[s].ncy - 1);
        jobs[j].cx = (const double*)(inb + cx_off[s]);
        jobs[j].cy = (const double*)(inb + cy_off[s]);
        jobs[j].eps = (const cplx*)(inb + (of_mu ? mu_off[s] : eps_off[s])) + (size_t)l * cells;
        jobs[j].ncx = si[s].ncx;
        jobs[j].ncy = si[s].ncy;
        jobs[j].fe11 = W_(c.fe11) + NN * j;
        jobs[j].fe22 = W_(c.fe22) + NN * j;
        jobs[j].fe33 = W_(c.fe33) + NN * j;
        jobs[j].tab = W_(c.tab) + c.tab_elems * j;
        jobs[j].f2d = si[s].tables && !of_mu
                          ? (const cplx*)(inb + f2d_off[s]) + (size_t)(l - 1) * (2 * nx - 1) * (2 * ny - 1)
                          : nullptr;
      }
      // ConvJob array lives in the workspace (uploaded by a memcpy step)
      const size_t jobs_meta = meta.add_vec(jobs);
      ConvLaunch CL;
      CL.jobs = nullptr;  // set at execution: the job array lives in the metadata block
      CL.njobs = nconv;
      CL.nx = nx;
      CL.ny = ny;
      CL.max_ncx = c.max_ncx;
      CL.max_ncy = c.max_ncy;
      const size_t strips = (size_t)std::max(c.max_ncx - 1, c.max_ncy - 1);
      cplx** tp = (cplx**)(wb + c.tptr);
      CL.tx_ptrs = tp;
      CL.txinv_ptrs = tp + strips * nconv;
      CL.ty_ptrs = tp + 2 * strips * nconv;
      CL.tyinv_ptrs = tp + 3 * strips * nconv;
      CL.ipiv = (int*)(wb + c.tipiv);
      CL.info = (int*)(wb + c.tinfo);
      P->steps.push_back([plan, CL, jobs_meta](cudaStream_t st, StageProf& pf) {
        ConvLaunch cl = CL;
        cl.jobs = (ConvJob*)((char*)plan->meta.p + jobs_meta);
        cudaError_t err = conv_matrices(cl, st, &pf);
        pf.mark(st, kStConvGather);
        return err;
      });
      // E = fe33^-1: LU in place, then the inverse in the getri order
      std::vector<cplx*> f33(nconv), einv(nconv);
      for (int j = 0; j < nconv; ++j) { f33[j] = W_(c.fe33) + NN * j; einv[j] = W_(c.Einv) + NN * j; }
      const size_t o33 = meta.add_vec(f33), oE = meta.add_vec(einv);
      int* cipiv = (int*)(wb + c.cipiv);
      int* cinfo = (int*)(wb + c.cinfo);
      P->steps.push_back([plan, o33, oE, N, nconv, cipiv, cinfo](cudaStream_t st, StageProf& pf) {
        cplx* const* a = (cplx* const*)((char*)plan->meta.p + o33);
        cplx* const* b = (cplx* const*)((char*)plan->meta.p + oE);
        cudaError_t err;
        if ((err = zgetrf_batched(a, N, N, cipiv, cinfo, nconv, st)) != cudaSuccess) return err;
        err = zgetri_batched(a, N, N, cipiv, b, N, nconv, st);
        pf.mark(st, kStConvInverse);
        return err;
      });
    }

    // ---------------- modes of the patterned layers
    if (nj > 0) {
      // non-magnetic layers: the X products and the structured M; magnetic
      // layers: dense P and Q, M = (P / k0^2) Q and V = Q W as products
      std::vector<int> jn, jm;
      for (int j = 0; j < nj; ++j)
        (is_mag(si[pts[c.points[c.job_point[j]]].stack], c.job_layer[j]) ? jm : jn).push_back(j);
      const int nn_j = (int)jn.size(), nm_j = (int)jm.size();
      std::vector<const cplx*> gA(2 * nn_j), gB(2 * nn_j), gS(2 * nn_j);
      std::vector<cplx*> gD(2 * nn_j);
      std::vector<LayerItem> items(nj);
      std::vector<cplx*> Mp(nj), Wp(nj);
      std::vector<int> jpoint(nj);
      for (int j = 0; j < nj; ++j) {
        const int lp = c.job_point[j], p = c.points[lp], s = pts[p].stack, l = c.job_layer[j];
        const int cj = c.conv_index.at({s, l});
        const cplx* ab = (const cplx*)(inb + ab_off[p]);
        LayerItem& it = items[j];
        it.fe11 = W_(c.fe11) + NN * cj;
        it.fe22 = W_(c.fe22) + NN * cj;
        it.X1 = W_(c.X1) + NN * j;
        it.X2 = W_(c.X2) + NN * j;
        it.ab = ab;
        it.M = W_(c.M) + nn * j;
        it.W = W_(c.W) + nn * j;
        it.V = W_(c.V) + nn * j;
        it.mu = W_(c.mu) + (size_t)n * j;
        it.gamma = W_(c.gam) + (size_t)n * j;
        it.k0 = 2 * kPi / pts[p].lambda;
        it.point = p;
        Mp[j] = it.M;
        Wp[j] = it.W;
        jpoint[j] = p;
      }
      std::vector<LayerItem> itn, itm;
      for (int q = 0; q < nn_j; ++q) {
        const int j = jn[q];
        const int cj = c.conv_index.at({pts[c.points[c.job_point[j]]].stack, c.job_layer[j]});
        const cplx* ab = items[j].ab;
        gA[q] = W_(c.Einv) + NN * cj;
        gB[q] = W_(c.fe11) + NN * cj;
        gS[q] = ab;
        gD[q] = W_(c.X1) + NN * j;
        gA[nn_j + q] = W_(c.Einv) + NN * cj;
        gB[nn_j + q] = W_(c.fe22) + NN * cj;
        gS[nn_j + q] = ab + N;
        gD[nn_j + q] = W_(c.X2) + NN * j;
        itn.push_back(items[j]);
      }
      // magnetic jobs: P / k0^2 into the V buffer and Q into the W buffer,
      // M = P Q; after the eigensolve Q again into the M buffer and V = Q W
      std::vector<MagItem> mpq(nm_j), mq(nm_j);
      std::vector<const cplx*> pA(nm_j), pB(nm_j), qA(nm_j), qB(nm_j);
      std::vector<cplx*> pD(nm_j), qD(nm_j);
      for (int q = 0; q < nm_j; ++q) {
        const int j = jm[q];
        const int s = pts[c.points[c.job_point[j]]].stack, l = c.job_layer[j];
        const int ce = c.conv_index.at({s, l}), cm = c.conv_index.at({s, l + kMuJob});
        MagItem mi;
        mi.E = W_(c.Einv) + NN * ce;
        mi.H = W_(c.Einv) + NN * cm;
        mi.fe11 = W_(c.fe11) + NN * ce;
        mi.fe22 = W_(c.fe22) + NN * ce;
        mi.fm11 = W_(c.fe11) + NN * cm;
        mi.fm22 = W_(c.fe22) + NN * cm;
        mi.ab = items[j].ab;
        mi.k0 = items[j].k0;
        mi.P = items[j].V;
        mi.Q = items[j].W;
        mpq[q] = mi;
        mi.P = nullptr;
        mi.Q = items[j].M;
        mq[q] = mi;
        pA[q] = items[j].V; pB[q] = items[j].W; pD[q] = items[j].M;
        qA[q] = items[j].M; qB[q] = items[j].W; qD[q] = items[j].V;
        itm.push_back(items[j]);
      }
      const size_t oA = meta.add_vec(gA), oB = meta.add_vec(gB), oS = meta.add_vec(gS), oD = meta.add_vec(gD);
      const size_t oItems = meta.add_vec(itn), oM = meta.add_vec(Mp), oW = meta.add_vec(Wp);
      const size_t oJP = meta.add_vec(jpoint);
      const size_t oItemsM = meta.add_vec(itm), oMpq = meta.add_vec(mpq), oMq = meta.add_vec(mq);
      const size_t opA = meta.add_vec(pA), opB = meta.add_vec(pB), opD = meta.add_vec(pD);
      const size_t oqA = meta.add_vec(qA), oqB = meta.add_vec(qB), oqD = meta.add_vec(qD);
      // V GEMMs: top = fe22 * Wb, bottom = fe11 * Wt; the jobs of points
      // whose products run in 3xTF32 first (their top and bottom products),
      // then those of the FP64 points
      const bool tc_modes = precision == RCWA_PREC_MIXED && c.prod != 1;
      std::vector<int> vorder;
      for (int pass = 0; pass < 2; ++pass)
        for (int q = 0; q < nn_j; ++q) {
          const bool tc = tc_modes && !c.fp64_pt[c.job_point[jn[q]]];
          if (tc == (pass == 0)) vorder.push_back(q);
        }
      int ntv = 0;  // 3xTF32 V products
      for (int q = 0; q < nn_j; ++q) ntv += (tc_modes && !c.fp64_pt[c.job_point[jn[q]]]) ? 2 : 0;
      std::vector<const cplx*> vA, vB;
      std::vector<cplx*> vD;
      auto vput = [&](int q0, int q1) {
        for (int i = q0; i < q1; ++i) {
          const LayerItem& t = itn[vorder[i]];
          vA.push_back(t.fe22); vB.push_back(t.W + (size_t)N * n); vD.push_back(t.V);
        }
        for (int i = q0; i < q1; ++i) {
          const LayerItem& t = itn[vorder[i]];
          vA.push_back(t.fe11); vB.push_back(t.W); vD.push_back(t.V + (size_t)N * n);
        }
      };
      vput(0, ntv / 2);
      vput(ntv / 2, nn_j);
      const size_t ovA = meta.add_vec(vA), ovB = meta.add_vec(vB), ovD = meta.add_vec(vD);
      int* tcerr_m = P->dTcErr;
      int* tcscale_m = P->dTcScale;
      float* planes_m = (float*)(wb + c.planes);
      const size_t planes_bytes_m = c.planes_bytes;
      // 3xTF32 products per call: the scale workspace's 2048 items, and as
      // many as the plane scratch holds split (else the per-tile split kernel)
      const size_t per_v = zgemm_tf32x3_planes_bytes(N, n, N, 1);
      const int sub_v = (int)std::max<size_t>(1, std::min<size_t>(2048, per_v ? planes_bytes_m / per_v : 2048));
      cplx* mu = W_(c.mu);
      void* eigw = wb + c.eigw;
      int* einfo = (int*)(wb + c.einfo);
      int* status = P->dStatus;
      const int ms_min = c.ms_min;
      P->steps.push_back([=](cudaStream_t st, StageProf& pf) {
        char* m = (char*)plan->meta.p;
        auto dense = [&](size_t a, size_t b, size_t d) {
          GemmArgs q{};
          q.A = (const cplx* const*)(m + a);
          q.B = (const cplx* const*)(m + b);
          q.D = (cplx* const*)(m + d);
          q.M = n; q.N = n; q.K = n;
          q.lda = n; q.ldb = n; q.ldc = n; q.ldd = n;
          q.alpha = mkc(1, 0); q.beta = mkc(0, 0); q.gammaI = mkc(0, 0);
          q.batch = nm_j;
          return zgemm_batched(q, st);
        };
        cudaError_t err;
        const LayerItem* it = (const LayerItem*)(m + oItems);
        if (nn_j > 0) {
          GemmArgs g{};
          g.A = (const cplx* const*)(m + oA);
          g.B = (const cplx* const*)(m + oB);
          g.C = nullptr;
          g.D = (cplx* const*)(m + oD);
          g.s = (const cplx* const*)(m + oS);
          g.M = N; g.N = N; g.K = N;
          g.lda = N; g.ldb = N; g.ldc = N; g.ldd = N;
          g.alpha = mkc(1, 0); g.beta = mkc(0, 0); g.gammaI = mkc(0, 0);
          g.batch = 2 * nn_j;
          if ((err = zgemm_batched(g, st)) != cudaSuccess) return err;
          pf.mark(st, kStPQGemm);
          if ((err = assemble_m(it, nn_j, N, st)) != cudaSuccess) return err;
          pf.mark(st, kStAssemble);
        }
        if (nm_j > 0) {
          if ((err = assemble_pq((const MagItem*)(m + oMpq), nm_j, N, true, st)) != cudaSuccess) return err;
          pf.mark(st, kStAssemble);
          if ((err = dense(opA, opB, opD)) != cudaSuccess) return err;
          pf.mark(st, kStPQGemm);
        }
        if ((err = zgeev_batched((cplx* const*)(m + oM), n, n, mu, (cplx* const*)(m + oW), n, eigw, einfo, nj, st,
                                 &pf, ms_min)) != cudaSuccess)
          return err;
        if ((err = fold_info(einfo, (const int*)(m + oJP), nj, 0, status, st)) != cudaSuccess) return err;
        if (nn_j > 0) {
          GemmArgs v{};
          v.A = (const cplx* const*)(m + ovA);
          v.B = (const cplx* const*)(m + ovB);
          v.D = (cplx* const*)(m + ovD);
          v.M = N; v.N = n; v.K = N;
          v.lda = N; v.ldb = n; v.ldc = n; v.ldd = n;
          v.alpha = mkc(1, 0); v.beta = mkc(0, 0); v.gammaI = mkc(0, 0);
          // 3xTF32 for the points with tensor-core products (a mixed plan's
          // modal V, like its cascade products), FP64 for the rest
          for (int b0 = 0; b0 < ntv; b0 += sub_v) {
            GemmArgs t = v;
            t.A = v.A + b0; t.B = v.B + b0; t.D = v.D + b0;
            t.batch = std::min(sub_v, ntv - b0);
            if ((err = zgemm_tf32x3_batched(t, tcscale_m, tcerr_m, st, 128, planes_m, planes_bytes_m)) != cudaSuccess)
              return err;
          }
          if (ntv < 2 * nn_j) {
            GemmArgs f = v;
            f.A = v.A + ntv; f.B = v.B + ntv; f.D = v.D + ntv;
            f.batch = 2 * nn_j - ntv;
            if ((err = zgemm_batched(f, st)) != cudaSuccess) return err;
          }
          if ((err = finish_modes(it, nn_j, N, status, st)) != cudaSuccess) return err;
        }
        if (nm_j > 0) {
          if ((err = assemble_pq((const MagItem*)(m + oMq), nm_j, N, false, st)) != cudaSuccess) return err;
          if ((err = dense(oqA, oqB, oqD)) != cudaSuccess) return err;
          if ((err = finish_modes_scaled((const LayerItem*)(m + oItemsM), nm_j, N, status, st)) != cudaSuccess)
            return err;
        }
        pf.mark(st, kStModes);
        return cudaSuccess;
      });
    }

    // ---------------- half-spaces
    {
      std::vector<HalfItem> hs(2 * np);
      for (int lp = 0; lp < np; ++lp) {
        const int p = c.points[lp], s = pts[p].stack;
        const size_t cells = (size_t)(si[s].ncx - 1) * (si[s].ncy - 1);
        for (int side = 0; side < 2; ++side) {
          HalfItem& h = hs[2 * lp + side];
          h.ab = (const cplx*)(inb + ab_off[p]);
          const int lh = side == 0 ? 0 : si[s].L - 1;
          h.eps = si[s].eps[(size_t)lh * cells];
          h.mu = layer_mu0(si[s], lh);
          h.magnetic = (h.mu.x != 1.0 || h.mu.y != 0.0) ? 1 : 0;
          h.k0 = 2 * kPi / pts[p].lambda;
          h.W = W_(side == 0 ? c.hW0 : c.hWL) + nn * lp;
          h.V = W_(side == 0 ? c.hV0 : c.hVL) + nn * lp;
          h.gamma = W_(side == 0 ? c.hg0 : c.hgL) + (size_t)n * lp;
          h.point = p;
        }
      }
      const size_t oh = meta.add_vec(hs);
      int* status = P->dStatus;
      const int cnt = 2 * np;
      P->steps.push_back([=](cudaStream_t st, StageProf& pf) {
        cudaError_t err = halfspace_modes((const HalfItem*)((char*)plan->meta.p + oh), cnt, N, status, st);
        pf.mark(st, kStHalfspace);
        return err;
      });
    }

    // ---------------- cascade
    {
      std::vector<cplx*> rud(np), tdd(np), gbuf(np);
      for (int lp = 0; lp < np; ++lp) {
        rud[lp] = W_(c.Rud) + nn * lp;
        tdd[lp] = W_(c.Tdd) + nn * lp;
        gbuf[lp] = W_(c.G) + nn * lp;
      }
      const size_t oR0 = meta.add_vec(rud), oT0 = meta.add_vec(tdd);
      P->steps.push_back([=](cudaStream_t st, StageProf& pf) {
        cudaError_t err = cascade_init((cplx* const*)((char*)plan->meta.p + oR0),
                                       (cplx* const*)((char*)plan->meta.p + oT0), n, np, st);
        pf.mark(st, kStPhase);
        return err;
      });
      // layer buffers of point lp, layer l
      auto layerW = [&](int lp, int l) -> cplx* {
        const int p = c.points[lp];
        const StackInfo& sl = si[pts[p].stack];
        if (l == 0 && !sl.pat0) return W_(c.hW0) + nn * lp;
        if (l == sl.L - 1 && !sl.patL) return W_(c.hWL) + nn * lp;
        for (size_t j = 0; j < c.job_point.size(); ++j)
          if (c.job_point[j] == lp && c.job_layer[j] == l) return W_(c.W) + nn * j;
        return nullptr;
      };
      auto layerV = [&](int lp, int l) -> cplx* {
        const int p = c.points[lp];
        const StackInfo& sl = si[pts[p].stack];
        if (l == 0 && !sl.pat0) return W_(c.hV0) + nn * lp;
        if (l == sl.L - 1 && !sl.patL) return W_(c.hVL) + nn * lp;
        for (size_t j = 0; j < c.job_point.size(); ++j)
          if (c.job_point[j] == lp && c.job_layer[j] == l) return W_(c.V) + nn * j;
        return nullptr;
      };
      auto layerG = [&](int lp, int l) -> cplx* {
        for (size_t j = 0; j < c.job_point.size(); ++j)
          if (c.job_point[j] == lp && c.job_layer[j] == l) return W_(c.gam) + (size_t)n * j;
        return nullptr;
      };
      int maxL = 0;
      for (int lp = 0; lp < np; ++lp) maxL = std::max(maxL, si[pts[c.points[lp]].stack].L);
      for (int step = 0; step + 1 < maxL; ++step) {
        std::vector<int> part;
        for (int lp = 0; lp < np; ++lp)
          if (si[pts[c.points[lp]].stack].L - 1 > step) part.push_back(lp);
        const int k = (int)part.size();
        if (k == 0) continue;
        // points whose products run in 3xTF32 first, the FP64 ones after them
        const bool tc_plan = precision == RCWA_PREC_MIXED && c.prod != 1;
        std::stable_partition(part.begin(), part.end(), [&](int lp) { return tc_plan && !c.fp64_pt[lp]; });
        int kt = 0;
        for (int lp : part) kt += (tc_plan && !c.fp64_pt[lp]) ? 1 : 0;
        // interfaces whose upper layer a is a patterned layer take the dense
        // LU route; those below the uniform superstrate (a = 0: Wa = I, Va
        // 2x2-block diagonal) take IE = Wb and the per-order 2x2 solve
        std::vector<const cplx*> csrc, csrcV;
        std::vector<cplx*> cdst, cdstV, lu, luV, rhs, rhsV;
        std::vector<HalfSolveItem> hs;
        std::vector<PhaseItem> ph;
        std::vector<const cplx*> fA(k), fB(k), fC(k), gA(k), gB(k), gC(k), sF(k), sG(k), tG(k), tT(k), tTau(k);
        std::vector<cplx*> fD(k), gD(k), sD(k), tauD(k), rD(k), tD(k), Sp(k);
        std::vector<int> ipoint, spoint(k);
        int kdt = 0;  // dense-route points with 3xTF32 solves
        for (int q = 0; q < k; ++q) {
          const int lp = part[q], p = c.points[lp];
          const int L = si[pts[p].stack].L;
          const int index = L - 1 - step, a = index - 1, b = index;
          cplx* IE = W_(c.IE) + nn * lp;
          cplx* IH = W_(c.IH) + nn * lp;
          cplx* WLU = W_(c.WLU) + nn * lp;
          cplx* VLU = W_(c.VLU) + nn * lp;
          csrc.push_back(layerW(lp, b)); cdst.push_back(IE);
          csrc.push_back(layerV(lp, b)); cdst.push_back(IH);
          if (a == 0 && !si[pts[p].stack].pat0) {
            HalfSolveItem h;
            h.X = IH;
            h.V0 = layerV(lp, 0);
            h.point = p;
            hs.push_back(h);
          } else {
            csrcV.push_back(layerW(lp, a)); cdstV.push_back(WLU);
            csrcV.push_back(layerV(lp, a)); cdstV.push_back(VLU);
            lu.push_back(WLU); luV.push_back(VLU);
            rhs.push_back(IE); rhsV.push_back(IH);
            ipoint.push_back(p);
            if (tc_plan && !c.fp64_pt[lp]) ++kdt;  // the dense list keeps part's order: 3xTF32 points first
          }
          spoint[q] = p;
          if (step > 0) {
            PhaseItem it;
            it.Rud = rud[lp];
            it.Tdd = tdd[lp];
            it.gamma = layerG(lp, b);
            it.thick = si[pts[p].stack].thick[b];
            ph.push_back(it);
          }
          cplx* F = W_(c.F) + nn * lp;
          fA[q] = IE; fB[q] = rud[lp]; fC[q] = IE; fD[q] = F;
          gA[q] = IH; gB[q] = rud[lp]; gC[q] = IH; gD[q] = gbuf[lp];
          sF[q] = F; sG[q] = gbuf[lp]; sD[q] = F; Sp[q] = F;
          cplx* tau = W_(c.tau) + nn * lp;
          tauD[q] = tau;
          // Rud = -2 G tau + I ; Tnew = 2 Tdd tau -> into the G buffer, then swap
          tG[q] = gbuf[lp]; tTau[q] = tau; rD[q] = rud[lp];
          tT[q] = tdd[lp]; tD[q] = gbuf[lp];
          std::swap(tdd[lp], gbuf[lp]);
        }
        // LU batch: the W's and then the V's of the dense-route points whose
        // solves run with 3xTF32 updates, then those of the FP64 points
        const int kd = (int)lu.size(), kh = (int)hs.size();
        csrc.insert(csrc.end(), csrcV.begin(), csrcV.end());
        cdst.insert(cdst.end(), cdstV.begin(), cdstV.end());
        {
          std::vector<cplx*> l2, r2;
          std::vector<int> i2;
          auto put = [&](int q0, int q1) {
            for (int q = q0; q < q1; ++q) { l2.push_back(lu[q]); r2.push_back(rhs[q]); i2.push_back(ipoint[q]); }
            for (int q = q0; q < q1; ++q) { l2.push_back(luV[q]); r2.push_back(rhsV[q]); i2.push_back(ipoint[q]); }
          };
          put(0, kdt);
          put(kdt, kd);
          lu = l2;
          rhs = r2;
          ipoint = i2;
        }
        const int ncopy = (int)csrc.size();
        const size_t ocs = meta.add_vec(csrc), ocd = meta.add_vec(cdst), olu = meta.add_vec(lu), orhs = meta.add_vec(rhs);
        const size_t oip = meta.add_vec(ipoint), osp = meta.add_vec(spoint), ohs = meta.add_vec(hs);
        const size_t oph = meta.add_vec(ph);
        const int nph = (int)ph.size();
        const size_t ofA = meta.add_vec(fA), ofB = meta.add_vec(fB), ofC = meta.add_vec(fC), ofD = meta.add_vec(fD);
        const size_t ogA = meta.add_vec(gA), ogB = meta.add_vec(gB), ogC = meta.add_vec(gC), ogD = meta.add_vec(gD);
        const size_t osF = meta.add_vec(sF), osG = meta.add_vec(sG), osD = meta.add_vec(sD), oSp = meta.add_vec(Sp);
        const size_t otau = meta.add_vec(tauD), otG = meta.add_vec(tG), otTau = meta.add_vec(tTau), orD = meta.add_vec(rD);
        const size_t otT = meta.add_vec(tT), otD = meta.add_vec(tD);
        int* pipiv = (int*)(wb + c.pipiv);
        int* pinfo = (int*)(wb + c.pinfo);
        int* status = P->dStatus;
        int* tcerr = P->dTcErr;
        int* tcscale = P->dTcScale;
        const int lu_if = c.lu_if, lu_tau = c.lu_tau;
        const int tile_n = c.prod == 2 ? 256 : 128;
        float* planes = (float*)(wb + c.planes);
        const size_t planes_bytes = c.planes_bytes;
        P->steps.push_back([=](cudaStream_t st, StageProf& pf) {
          // the cascade products: items [0, kt) in 3xTF32 on tcgen05, the
          // rest on the FP64 tensor path
          auto product = [&](const GemmArgs& ga) {
            cudaError_t x = cudaSuccess;
            if (kt > 0) {
              GemmArgs t = ga;
              t.batch = kt;
              x = zgemm_tf32x3_batched(t, tcscale, tcerr, st, tile_n, planes, planes_bytes);
            }
            if (x == cudaSuccess && kt < ga.batch) {
              GemmArgs f = ga;
              f.A = ga.A + kt;
              f.B = ga.B + kt;
              f.C = ga.C ? ga.C + kt : nullptr;
              f.D = ga.D + kt;
              f.batch = ga.batch - kt;
              x = zgemm_batched(f, st);
            }
            return x;
          };
          char* m = (char*)plan->meta.p;
          auto cpa = [m](size_t o) { return (const cplx* const*)(m + o); };
          auto pa = [m](size_t o) { return (cplx* const*)(m + o); };
          cudaError_t err;
          // interface matrices IE = Wa^-1 Wb, IH = Va^-1 Vb (rcwa/RCWASolver.cpp:537-543)
          if ((err = zcopy_batched(cpa(ocs), n, pa(ocd), n, n, n, ncopy, st)) != cudaSuccess) return err;
          pf.mark(st, kStInterface);
          // factorisations and solves: the first 2 kdt with 3xTF32 updates
          // between 128-wide blocks, the rest in FP64
          const TcProducts tcx{tcscale, tcerr, planes, planes_bytes};
          if (kdt > 0 && (err = zgetrf_blocked_batched(pa(olu), n, n, pipiv, pinfo, 2 * kdt, &tcx, st)) != cudaSuccess)
            return err;
          if (kd > kdt && (err = zgetrf_batched(pa(olu) + 2 * kdt, n, n, pipiv + (size_t)2 * kdt * n, pinfo + 2 * kdt,
                                                2 * (kd - kdt), st, lu_if)) != cudaSuccess)
            return err;
          if ((err = fold_info(pinfo, (const int*)(m + oip), 2 * kd, RCWA_ERR_SINGULAR, status, st)) != cudaSuccess)
            return err;
          pf.mark(st, kStInterfaceLU);
          if (kdt > 0 && (err = zgetrs_blocked_batched(cpa(olu), n, n, pipiv, pa(orhs), n, n, 2 * kdt, false, &tcx,
                                                       st)) != cudaSuccess)
            return err;
          if (kd > kdt && (err = zgetrs_batched(cpa(olu) + 2 * kdt, n, n, pipiv + (size_t)2 * kdt * n,
                                                pa(orhs) + 2 * kdt, n, n, 2 * (kd - kdt), st)) != cudaSuccess)
            return err;
          if ((err = halfspace_solve((const HalfSolveItem*)(m + ohs), kh, N, status, st)) != cudaSuccess) return err;
          pf.mark(st, kStInterface);
          if (nph > 0) {
            if ((err = apply_phase((const PhaseItem*)(m + oph), nph, n, st)) != cudaSuccess) return err;
            pf.mark(st, kStPhase);
          }
          GemmArgs g{};
          g.M = n; g.N = n; g.K = n;
          g.lda = n; g.ldb = n; g.ldc = n; g.ldd = n;
          g.batch = k;
          g.gammaI = mkc(0, 0);
          // F = IE + IE waveRud ; G = IH - IH waveRud   (:440-443)
          g.A = cpa(ofA); g.B = cpa(ofB); g.C = cpa(ofC); g.D = pa(ofD);
          g.alpha = mkc(1, 0); g.beta = mkc(1, 0);
          if ((err = product(g)) != cudaSuccess) return err;
          g.A = cpa(ogA); g.B = cpa(ogB); g.C = cpa(ogC); g.D = pa(ogD);
          g.alpha = mkc(-1, 0); g.beta = mkc(1, 0);
          if ((err = product(g)) != cudaSuccess) return err;
          pf.mark(st, kStCascadeGemm);
          // tau = (F + G)^-1  (:451-453)
          if ((err = zaxpby_batched(cpa(osF), cpa(osG), pa(osD), mkc(1, 0), mkc(1, 0), n, k, st)) != cudaSuccess)
            return err;
          pf.mark(st, kStTau);
          if (kt > 0 && (err = zgetrf_blocked_batched(pa(oSp), n, n, pipiv, pinfo, kt, &tcx, st)) != cudaSuccess)
            return err;
          if (k > kt && (err = zgetrf_batched(pa(oSp) + kt, n, n, pipiv + (size_t)kt * n, pinfo + kt, k - kt, st,
                                              lu_tau)) != cudaSuccess)
            return err;
          if ((err = fold_info(pinfo, (const int*)(m + osp), k, RCWA_ERR_SINGULAR, status, st)) != cudaSuccess)
            return err;
          pf.mark(st, kStTauLU);
          // tau = (F + G)^-1 in the getri order (PartialPivLU::inverse, :451-453)
          if (kt > 0 && (err = zgetrs_blocked_batched(cpa(oSp), n, n, pipiv, pa(otau), n, n, kt, true, &tcx, st)) !=
                            cudaSuccess)
            return err;
          if (k > kt && (err = zgetri_batched(cpa(oSp) + kt, n, n, pipiv + (size_t)kt * n, pa(otau) + kt, n, k - kt,
                                              st)) != cudaSuccess)
            return err;
          pf.mark(st, kStTau);
          // Rud = I - 2 G tau ; Tdd = 2 waveTdd tau  (:457-460)
          g.A = cpa(otG); g.B = cpa(otTau); g.C = nullptr; g.D = pa(orD);
          g.alpha = mkc(-2, 0); g.beta = mkc(0, 0); g.gammaI = mkc(1, 0);
          if ((err = product(g)) != cudaSuccess) return err;
          g.A = cpa(otT); g.B = cpa(otTau); g.C = nullptr; g.D = pa(otD);
          g.alpha = mkc(2, 0); g.beta = mkc(0, 0); g.gammaI = mkc(0, 0);
          err = product(g);
          pf.mark(st, kStCascadeGemm);
          return err;
        });
      }
      // ---------------- what rcwa_plan_field needs of every point
      if (P->field_pts.size() != (size_t)n_pts) P->field_pts.resize(n_pts);
      for (int lp = 0; lp < np; ++lp) {
        const int p = c.points[lp], s = pts[p].stack;
        const StackInfo& sk = si[s];
        FieldPoint& fp = P->field_pts[p];
        fp.N = N; fp.nx = nx; fp.ny = ny; fp.L = sk.L;
        fp.W.assign(sk.L, nullptr); fp.V.assign(sk.L, nullptr); fp.gamma.assign(sk.L, nullptr);
        fp.Einv.assign(sk.L, nullptr);
        for (int l = 0; l < sk.L; ++l) {
          fp.W[l] = layerW(lp, l);
          fp.V[l] = layerV(lp, l);
          fp.gamma[l] = layerG(lp, l);
          if (l > 0 && l + 1 < sk.L) fp.Einv[l] = W_(c.Einv) + NN * c.conv_index.at({s, l});
        }
        fp.thick = sk.thick;
        fp.Rud = rud[lp];
        fp.Tdd = tdd[lp];
        fp.ab = (const cplx*)(inb + ab_off[p]);
        fp.pat0 = sk.pat0 != 0;
        fp.k0 = 2 * kPi / pts[p].lambda;
        fp.kx0 = pts[p].kx0;
        fp.ky0 = pts[p].ky0;
        fp.x0 = sk.cx.front();
        fp.y0 = sk.cy.front();
        fp.Lx = sk.Lx;
        fp.Ly = sk.Ly;
      }

      // ---------------- responses of points with a patterned half-space
      // C = W_ref^-1 [e_inc, e_N+inc] (LU of a copy of W_ref), then
      // Rc = W_ref (Rud C), Tc = W_trn (Tdd C): the harmonics of
      // generateHorizontalPlaneWave's plane wave (rcwa/Layer.cpp:453-480)
      // scattered into both half-spaces (rcwa/RCWASolver.cpp:1806-1811).
      // Buffers of the finished cascade hold them: the W_ref copy in WLU, C
      // in F, Rud C in IE, Tdd C in IH, Rc in tau, Tc in VLU (n x 2 each).
      std::vector<int> qpts;
      for (int lp = 0; lp < np; ++lp) {
        const StackInfo& sl = si[pts[c.points[lp]].stack];
        if (sl.pat0 || sl.patL) qpts.push_back(lp);
      }
      std::vector<cplx*> rc_of(np, nullptr), tc_of(np, nullptr);
      if (!qpts.empty()) {
        const int nq = (int)qpts.size();
        const int inc = ny * ((nx - 1) / 2) + (ny - 1) / 2;
        std::vector<const cplx*> w0(nq), rA(nq), tA(nq), wt(nq);
        std::vector<cplx*> wlu(nq), cb(nq), r1(nq), t1(nq), rcp(nq), tcp(nq);
        std::vector<int> qpoint(nq);
        for (int q = 0; q < nq; ++q) {
          const int lp = qpts[q];
          const int L = si[pts[c.points[lp]].stack].L;
          w0[q] = layerW(lp, 0);
          wt[q] = layerW(lp, L - 1);
          wlu[q] = W_(c.WLU) + nn * lp;
          cb[q] = W_(c.F) + nn * lp;
          r1[q] = W_(c.IE) + nn * lp;
          t1[q] = W_(c.IH) + nn * lp;
          rcp[q] = W_(c.tau) + nn * lp;
          tcp[q] = W_(c.VLU) + nn * lp;
          rA[q] = rud[lp];
          tA[q] = tdd[lp];
          qpoint[q] = c.points[lp];
          rc_of[lp] = rcp[q];
          tc_of[lp] = tcp[q];
        }
        const size_t ow0 = meta.add_vec(w0), owt = meta.add_vec(wt), owlu = meta.add_vec(wlu);
        const size_t ocb = meta.add_vec(cb), or1 = meta.add_vec(r1), ot1 = meta.add_vec(t1);
        const size_t orc = meta.add_vec(rcp), otc = meta.add_vec(tcp), orA = meta.add_vec(rA), otA = meta.add_vec(tA);
        const size_t oqp = meta.add_vec(qpoint);
        int* pipiv = (int*)(wb + c.pipiv);
        int* pinfo = (int*)(wb + c.pinfo);
        int* status = P->dStatus;
        P->steps.push_back([=](cudaStream_t st, StageProf& pf) {
          char* m = (char*)plan->meta.p;
          auto cpa = [m](size_t o) { return (const cplx* const*)(m + o); };
          auto pa = [m](size_t o) { return (cplx* const*)(m + o); };
          cudaError_t err;
          if ((err = zcopy_batched(cpa(ow0), n, pa(owlu), n, n, n, nq, st)) != cudaSuccess) return err;
          if ((err = zgetrf_batched(pa(owlu), n, n, pipiv, pinfo, nq, st)) != cudaSuccess) return err;
          if ((err = fold_info(pinfo, (const int*)(m + oqp), nq, RCWA_ERR_SINGULAR, status, st)) != cudaSuccess)
            return err;
          // C = [e_inc, e_N+inc], then C = W_ref^-1 C
          if ((err = unit_columns(pa(ocb), n, inc, N + inc, nq, st)) != cudaSuccess) return err;
          if ((err = zgetrs_batched(cpa(owlu), n, n, pipiv, pa(ocb), 2, 2, nq, st)) != cudaSuccess) return err;
          GemmArgs g{};
          g.M = n; g.N = 2; g.K = n;
          g.lda = n; g.ldb = 2; g.ldc = 2; g.ldd = 2;
          g.alpha = mkc(1, 0); g.beta = mkc(0, 0); g.gammaI = mkc(0, 0);
          g.batch = nq;
          g.A = cpa(orA); g.B = cpa(ocb); g.D = pa(or1);
          if ((err = zgemm_batched(g, st)) != cudaSuccess) return err;
          g.A = cpa(otA); g.B = cpa(ocb); g.D = pa(ot1);
          if ((err = zgemm_batched(g, st)) != cudaSuccess) return err;
          g.A = cpa(ow0); g.B = cpa(or1); g.D = pa(orc);
          if ((err = zgemm_batched(g, st)) != cudaSuccess) return err;
          g.A = cpa(owt); g.B = cpa(ot1); g.D = pa(otc);
          err = zgemm_batched(g, st);
          pf.mark(st, kStScatter);
          return err;
        });
      }

      // ---------------- scatter
      std::vector<ScatterItem> sc;
      for (int lp = 0; lp < np; ++lp) {
        const int p = c.points[lp], s = pts[p].stack;
        const size_t cells = (size_t)(si[s].ncx - 1) * (si[s].ncy - 1);
        for (int x = 0; x < n_exc; ++x) {
          ScatterItem it;
          it.Rud = rud[lp];
          it.Tdd = tdd[lp];
          it.ab = (const cplx*)(inb + ab_off[p]);
          // k^2 = k0^2 eps mu of the half-spaces, and the transmitted flux
          // ratio |mu_ref / mu_trn| (rcwa/RCWASolver.cpp:1826-1830, 1905-1907)
          // (a patterned half-space: its values at (0, 0), Layer::eps(0, 0)
          // and Layer::mu(0, 0), rcwa/RCWASolver.cpp:1823-1827)
          const StackInfo& sk = si[s];
          const int Lt = sk.L - 1;
          const cplx mr = sk.pat0 && !sk.mu.empty() ? cell_value(sk, sk.mu, 0, 0.0, 0.0) : layer_mu0(sk, 0);
          const cplx mt = sk.patL && !sk.mu.empty() ? cell_value(sk, sk.mu, Lt, 0.0, 0.0) : layer_mu0(sk, Lt);
          const cplx er = sk.pat0 ? cell_value(sk, sk.eps, 0, 0.0, 0.0) : sk.eps[0];
          const cplx et = sk.patL ? cell_value(sk, sk.eps, Lt, 0.0, 0.0) : sk.eps[(size_t)Lt * cells];
          it.n2_ref = cmul(er, mr);
          it.n2_trn = cmul(et, mt);
          it.Rc = rc_of[lp];
          it.Tc = tc_of[lp];
          it.trn_scale = (mr.x == mt.x && mr.y == mt.y)
                             ? 1.0
                             : std::abs(std::complex<double>(mr.x, mr.y) / std::complex<double>(mt.x, mt.y));
          it.k0 = 2 * kPi / pts[p].lambda;
          const rcwa_cplx px = pxy[((size_t)p * n_exc + x) * 2], py = pxy[((size_t)p * n_exc + x) * 2 + 1];
          it.px = mkc(px.re, px.im);
          it.py = mkc(py.re, py.im);
          it.ref = P->dRef + P->order_offset[p] + (size_t)x * N;
          it.trn = P->dTrn + P->order_offset[p] + (size_t)x * N;
          it.R = P->dR + (size_t)p * n_exc + x;
          it.T = P->dT + (size_t)p * n_exc + x;
          it.point = p;
          sc.push_back(it);
        }
      }
      const size_t osc = meta.add_vec(sc);
      const int nsc = (int)sc.size();
      P->scatter_items = sc;
      P->scatter_meta = osc;
      P->scatter_N = N;
      P->scatter_nx = nx;
      P->scatter_ny = ny;
      int* status = P->dStatus;
      P->steps.push_back([=](cudaStream_t st, StageProf& pf) {
        cudaError_t err = scatter_efficiencies((const ScatterItem*)((char*)plan->meta.p + osc), nsc, N, nx, ny, status,
                                               st);
        pf.mark(st, kStScatter);
        return err;
      });
    }
  }
  P->chunks = (int)chunks.size();
  if (!P->meta.take(e, std::max<size_t>(meta.bytes.size(), 16))) return fail(e, RCWA_ERR_NOMEM, "metadata allocation failed");
  P->meta.bytes = meta.bytes.size();
  if (!meta.bytes.empty() &&
      cudaMemcpy(P->meta.p, meta.bytes.data(), meta.bytes.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(e, RCWA_ERR_CUDA, "metadata upload failed");
  // the uploads above ran on the legacy stream, which the plan's (non-blocking)
  // stream does not wait for
  if (cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess) return fail(e, RCWA_ERR_CUDA, "upload failed");
  *out = P.release();
  return RCWA_OK;
}
}  // namespace

namespace {
// The plan's launch sequence on stream st (status reset, then every step).
cudaError_t issue_plan(rcwa_plan* p, cudaStream_t st) {
  cudaError_t err = cudaMemsetAsync(p->dStatus, 0, sizeof(int) * p->n_pts, st);
  if (err == cudaSuccess) err = cudaMemsetAsync(p->dTcErr, 0, sizeof(int), st);
  p->prof->begin(st);
  for (size_t i = 0; err == cudaSuccess && i < p->steps.size(); ++i) err = p->steps[i](st, *p->prof);
  return err;
}
}  // namespace

// The first execution launches the kernels directly; from the second on the
// sequence is captured once into a CUDA graph (with the stage-timing event
// records when profiling is on) and the graph is launched, so repeated sweeps
// pay one launch instead of thousands.
extern "C" int rcwa_plan_execute(rcwa_plan* p, void* stream) {
  if (!p) return RCWA_ERR_INVALID;
  cudaStream_t st = stream ? (cudaStream_t)stream : p->e->stream;
  if (cudaSetDevice(p->e->device) != cudaSuccess) return fail(p->e, RCWA_ERR_CUDA, "cudaSetDevice failed");
  const long long launches0 = launch_counter();
  cudaError_t err = cudaSuccess;
  const bool graph = p->executions > 0;
  if (graph && p->graph_exec && p->graph_prof != p->prof->on) {
    // recapture with or without the stage-timing event nodes
    cudaDeviceSynchronize();
    cudaGraphExecDestroy(p->graph_exec);
    p->graph_exec = nullptr;
  }
  if (graph && !p->graph_exec) {
    p->graph_prof = p->prof->on;
    cudaGraph_t g = nullptr;
    // the previous execution's event records must have completed
    err = cudaStreamSynchronize(st);
    if (err == cudaSuccess) err = cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed);
    if (err == cudaSuccess) {
      cudaError_t ierr = issue_plan(p, st);
      err = cudaStreamEndCapture(st, &g);
      if (ierr != cudaSuccess) err = ierr;
    }
    if (err == cudaSuccess) err = cudaGraphInstantiate(&p->graph_exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (err != cudaSuccess) {
      p->graph_exec = nullptr;
      return fail(p->e, RCWA_ERR_CUDA, std::string("graph capture failed: ") + cudaGetErrorString(err));
    }
    p->graph_launches = launch_counter() - launches0;
  }
  if (graph) {
    err = cudaGraphLaunch(p->graph_exec, st);
    p->launches = p->graph_launches;
  } else {
    err = issue_plan(p, st);
    p->launches = launch_counter() - launches0;
  }
  ++p->executions;
  if (err != cudaSuccess) return fail(p->e, RCWA_ERR_CUDA, std::string("launch failed: ") + cudaGetErrorString(err));
  return RCWA_OK;
}

extern "C" int rcwa_plan_field_rows(const rcwa_plan* p, int point, int slice, int nres1, int* rows) {
  if (!p || !rows || point < 0 || point >= p->n_pts || slice < 0 || slice > 2 || nres1 < 1) return RCWA_ERR_INVALID;
  if (p->field_pts.size() != (size_t)p->n_pts) return RCWA_ERR_INVALID;
  *rows = field_rows(p->field_pts[point], slice, nres1);
  return RCWA_OK;
}

extern "C" int rcwa_plan_field(rcwa_plan* p, int point, rcwa_cplx px, rcwa_cplx py, int slice, double coord,
                               int component, int nres1, rcwa_cplx* field) {
  if (!p || !field || point < 0 || point >= p->n_pts) return RCWA_ERR_INVALID;
  if (p->chunks != 1) return fail(p->e, RCWA_ERR_UNSUPPORTED, "fields need a single-chunk plan");
  if (p->executions == 0) return fail(p->e, RCWA_ERR_INVALID, "execute the plan before asking for its fields");
  if (p->field_pts.size() != (size_t)p->n_pts || p->field_pts[point].L < 3)
    return fail(p->e, RCWA_ERR_INVALID, "fields need at least one interior layer");
  if (cudaSetDevice(p->e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  // the plan's last execution may still run on another stream
  if (cudaDeviceSynchronize() != cudaSuccess) return RCWA_ERR_CUDA;
  const int rc = field_slice(p->field_pts[point], mkc(px.re, px.im), mkc(py.re, py.im), slice, coord, component,
                             nres1, reinterpret_cast<cplx*>(field), p->e->stream);
  if (rc != RCWA_OK) return fail(p->e, rc, "field evaluation failed");
  return RCWA_OK;
}

extern "C" int rcwa_plan_rescatter(rcwa_plan* p, const rcwa_cplx* pxy) {
  if (!p || !pxy) return RCWA_ERR_INVALID;
  if (p->chunks != 1) return fail(p->e, RCWA_ERR_UNSUPPORTED, "rescatter needs a single-chunk plan");
  if (cudaSetDevice(p->e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  std::vector<ScatterItem> sc = p->scatter_items;
  for (size_t k = 0; k < sc.size(); ++k) {
    ScatterItem& it = sc[k];
    const size_t e = k % (size_t)p->n_exc;
    const rcwa_cplx px = pxy[((size_t)it.point * p->n_exc + e) * 2], py = pxy[((size_t)it.point * p->n_exc + e) * 2 + 1];
    it.px = mkc(px.re, px.im);
    it.py = mkc(py.re, py.im);
  }
  // the previous execution may still run on another stream
  if (cudaDeviceSynchronize() != cudaSuccess) return RCWA_ERR_CUDA;
  cudaStream_t st = p->e->stream;
  if (cudaMemcpyAsync((char*)p->meta.p + p->scatter_meta, sc.data(), sizeof(ScatterItem) * sc.size(),
                      cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemsetAsync(p->dStatus, 0, sizeof(int) * p->n_pts, st) != cudaSuccess)
    return RCWA_ERR_CUDA;
  if (scatter_efficiencies((const ScatterItem*)((char*)p->meta.p + p->scatter_meta), (int)sc.size(), p->scatter_N,
                           p->scatter_nx, p->scatter_ny, p->dStatus, st) != cudaSuccess)
    return RCWA_ERR_CUDA;
  // the host copy must outlive the asynchronous upload
  return cudaStreamSynchronize(st) == cudaSuccess ? RCWA_OK : RCWA_ERR_CUDA;
}

extern "C" int rcwa_plan_smatrix(rcwa_plan* p, int point, rcwa_cplx* Rud, rcwa_cplx* Tdd) {
  if (!p) return RCWA_ERR_INVALID;
  if (point < 0 || point >= p->n_pts) return fail(p->e, RCWA_ERR_INVALID, "point index out of range");
  if (p->chunks != 1) return fail(p->e, RCWA_ERR_UNSUPPORTED, "the S-matrix of a multi-chunk plan is not kept");
  if (cudaSetDevice(p->e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  const ScatterItem* it = nullptr;
  for (const ScatterItem& s : p->scatter_items)
    if (s.point == point) { it = &s; break; }
  if (!it) return fail(p->e, RCWA_ERR_INVALID, "point not found in the plan");
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(p->e, RCWA_ERR_CUDA, "execution failed");
  const size_t n = 2 * (size_t)p->point_N[point];
  if (Rud && cudaMemcpy(Rud, it->Rud, sizeof(cplx) * n * n, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(p->e, RCWA_ERR_CUDA, "download failed");
  if (Tdd && cudaMemcpy(Tdd, it->Tdd, sizeof(cplx) * n * n, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(p->e, RCWA_ERR_CUDA, "download failed");
  return RCWA_OK;
}

extern "C" int rcwa_plan_schedule(const rcwa_plan* p, int chunk, int* sched) {
  if (!p) return -1;
  if (chunk < 0 || !sched) return (int)p->sched.size();
  if (chunk >= (int)p->sched.size()) return -1;
  for (int k = 0; k < 6; ++k) sched[k] = p->sched[chunk][k];
  return (int)p->sched.size();
}

extern "C" long long rcwa_plan_launch_count(const rcwa_plan* p) { return p ? p->launches : 0; }

extern "C" int rcwa_plan_set_profiling(rcwa_plan* p, int on) {
  if (!p) return RCWA_ERR_INVALID;
  p->prof->on = on != 0;
  return RCWA_OK;
}

extern "C" int rcwa_plan_stage_times(rcwa_plan* p, double* ms, int max_stages) {
  if (!p || !ms) return RCWA_ERR_INVALID;
  // the events were recorded on whichever stream executed the plan
  if (p->prof->used > 0 && cudaEventSynchronize(p->prof->ev[p->prof->used - 1]) != cudaSuccess) return RCWA_ERR_CUDA;
  double t[kStCount];
  p->prof->collect(t);
  for (int i = 0; i < max_stages; ++i) ms[i] = i < kStCount ? t[i] : 0.0;
  return kStCount;
}

extern "C" const char* rcwa_stage_name(int stage) {
  static const char* names[kStCount] = {"conv_tables", "conv_gather", "conv_inverse", "pq_gemm", "assemble_pq",
                                        "hessenberg", "schur_qr", "trevc", "eig_backtransform", "eig_normalize",
                                        "modes_v", "halfspace", "interface_lu_solve", "phase", "cascade_gemm",
                                        "tau_inverse", "scatter", "interface_getrf", "tau_getrf"};
  return (stage >= 0 && stage < kStCount) ? names[stage] : "";
}

extern "C" int rcwa_plan_results(rcwa_plan* p, double* R, double* T, double* ref_orders, double* trn_orders,
                                 int* status) {
  if (!p) return RCWA_ERR_INVALID;
  if (cudaDeviceSynchronize() != cudaSuccess)
    return fail(p->e, RCWA_ERR_CUDA, std::string("execution failed: ") + cudaGetErrorString(cudaGetLastError()));
  const size_t ne = (size_t)p->n_pts * p->n_exc;
  // one download of the output block (R, T, orders, status, tensor-core flag)
  const char* base = (const char*)p->outputs.p;
  const size_t span = (size_t)((const char*)(p->dTcErr + 1) - base);
  std::vector<unsigned char> h(span);
  if (cudaMemcpy(h.data(), base, span, cudaMemcpyDeviceToHost) != cudaSuccess) return RCWA_ERR_CUDA;
  auto at = [&](const void* d) { return h.data() + ((const char*)d - base); };
  if (R) std::memcpy(R, at(p->dR), sizeof(double) * ne);
  if (T) std::memcpy(T, at(p->dT), sizeof(double) * ne);
  if (ref_orders) std::memcpy(ref_orders, at(p->dRef), sizeof(double) * p->total_orders);
  if (trn_orders) std::memcpy(trn_orders, at(p->dTrn), sizeof(double) * p->total_orders);
  std::vector<int> hs(p->n_pts);
  std::memcpy(hs.data(), at(p->dStatus), sizeof(int) * p->n_pts);
  if (status) std::memcpy(status, hs.data(), sizeof(int) * p->n_pts);
  int tcerr = 0;
  std::memcpy(&tcerr, at(p->dTcErr), sizeof(int));
  if (tcerr) return fail(p->e, RCWA_ERR_CUDA, "a tensor-core completion wait ran out; results are incomplete");
  for (int v : hs)
    if (v) return v;
  return RCWA_OK;
}

extern "C" void rcwa_plan_destroy(rcwa_plan* p) {
  if (!p) return;
  cudaSetDevice(p->e->device);
  delete p;
}

extern "C" int rcwa_engine_solve_tables(rcwa_engine* e, const rcwa_table_stack* stacks, int n_stacks,
                                        const rcwa_point* pts, int n_pts, int n_exc, const rcwa_cplx* pxy,
                                        int precision, double* R, double* T, double* ref_orders,
                                        double* trn_orders, int* status) {
  rcwa_plan* p = nullptr;
  int rc = rcwa_plan_create_tables(e, stacks, n_stacks, pts, n_pts, n_exc, pxy, precision, &p);
  if (rc) return rc;
  rc = rcwa_plan_execute(p, nullptr);
  if (rc == RCWA_OK) rc = rcwa_plan_results(p, R, T, ref_orders, trn_orders, status);
  rcwa_plan_destroy(p);
  return rc;
}

extern "C" int rcwa_engine_solve_batch(rcwa_engine* e, const rcwa_stack* stacks, int n_stacks, const rcwa_point* pts,
                                       int n_pts, int n_exc, const rcwa_cplx* pxy, int precision, double* R,
                                       double* T, double* ref_orders, double* trn_orders, int* status) {
  rcwa_plan* p = nullptr;
  int rc = rcwa_plan_create(e, stacks, n_stacks, pts, n_pts, n_exc, pxy, precision, &p);
  if (rc) return rc;
  rc = rcwa_plan_execute(p, nullptr);
  if (rc == RCWA_OK) rc = rcwa_plan_results(p, R, T, ref_orders, trn_orders, status);
  rcwa_plan_destroy(p);
  return rc;
}
