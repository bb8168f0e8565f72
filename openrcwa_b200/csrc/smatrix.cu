// Slab scattering matrices and the Redheffer star product, batched in FP64.
//
//   slab  dtmm::RCWAScatterMatrix::compute_v2 (rcwa/RCWAScatterMatrix.cpp:90-146)
//   star  the z-integrators' cascade update (core/RCWAIntegrator.cpp:57-67,
//         core/RedhefferIntegrator.cpp:136-146)
//
// Both are compositions of the engine's batched LU (getrf/getrs) and tile
// GEMM; the only dedicated kernel builds the slab's right-hand sides.  Every
// batch item is one independent problem; matrices are row-major n x n.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <map>
#include <string>
#include <vector>

#include "eig.cuh"
#include "engine_internal.cuh"
#include "linalg.cuh"
#include "rcwa_kernels.cuh"

namespace {

struct SlabRhsItem {
  const cplx* F0;     // W^-1 W0
  const cplx* G0;     // V^-1 V0
  const cplx* gamma;  // n slab propagation constants
  double ss;          // wz / k0
  cplx* A;            // out: F0 + G0
  cplx* R3;           // out: [B | X A | X B], n x 3n
};

// A = F0 + G0; R3 = [B | diag(X) A | diag(X) B] with B = F0 - G0 and
// X = exp(i gamma ss) (rcwa/RCWAScatterMatrix.cpp:114-117,128-134).
__global__ void slab_rhs_kernel(const SlabRhsItem* items, int n) {
  const SlabRhsItem it = items[blockIdx.y];
  const size_t nn = (size_t)n * n;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < nn;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx / n), c = (int)(idx % n);
    const cplx f = it.F0[idx], g = it.G0[idx];
    const cplx a = cadd(f, g), b = csub(f, g);
    const cplx gm = it.gamma[r];
    const cplx x = cexp_(mkc(-gm.y * it.ss, gm.x * it.ss));
    it.A[idx] = a;
    cplx* R = it.R3 + (size_t)r * 3 * n;
    R[c] = b;
    R[n + c] = cmul(x, a);
    R[2 * n + c] = cmul(x, b);
  }
}

// RAII device allocation.
struct Buf {
  void* p = nullptr;
  explicit Buf(size_t bytes) {
    if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) p = nullptr;
  }
  ~Buf() { if (p) cudaFree(p); }
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
  cplx* c() const { return (cplx*)p; }
};

// Pointer arrays for the batched primitives, collected on the host and
// uploaded as one block.
struct PtrBlob {
  std::vector<void*> h;
  Buf* d = nullptr;
  // batch pointers base + b*stride + off; returns the slot of the first one
  size_t add(cplx* base, size_t stride, size_t off, int batch) {
    const size_t at = h.size();
    for (int b = 0; b < batch; ++b) h.push_back(base + stride * b + off);
    return at;
  }
  size_t add_list(const std::vector<cplx*>& v) {
    const size_t at = h.size();
    for (cplx* q : v) h.push_back(q);
    return at;
  }
  size_t add_ints(const std::vector<int>& v) {
    // ints packed two per slot
    const size_t at = h.size();
    const size_t slots = (v.size() + 1) / 2;
    h.resize(at + slots, nullptr);
    std::memcpy(h.data() + at, v.data(), sizeof(int) * v.size());
    return at;
  }
  bool upload(cudaStream_t st) {
    d = new Buf(sizeof(void*) * h.size());
    return d->p && cudaMemcpyAsync(d->p, h.data(), sizeof(void*) * h.size(), cudaMemcpyHostToDevice, st) ==
                       cudaSuccess;
  }
  ~PtrBlob() { delete d; }
  cplx* const* at(size_t slot) const { return (cplx* const*)((void**)d->p + slot); }
  const cplx* const* cat(size_t slot) const { return (const cplx* const*)((void**)d->p + slot); }
  const int* ints(size_t slot) const { return (const int*)((void**)d->p + slot); }
};

int set_err(rcwa_engine* e, int code, const char* msg) {
  if (e) e->last_error = msg;
  return code;
}

GemmArgs gemm(int n, int batch) {
  GemmArgs g{};
  g.M = n; g.N = n; g.K = n;
  g.batch = batch;
  g.alpha = mkc(1, 0);
  g.beta = mkc(0, 0);
  g.gammaI = mkc(0, 0);
  return g;
}

// Uploads are ordered on the engine's (non-blocking) stream; pageable sources
// are staged by the driver before the call returns.
bool up(cplx* d, const rcwa_cplx* h, size_t count, cudaStream_t st) {
  return cudaMemcpyAsync(d, h, sizeof(cplx) * count, cudaMemcpyHostToDevice, st) == cudaSuccess;
}

// Copy the per-item status out and return the first error.
int finish_status(rcwa_engine* e, const int* dstatus, int batch, int* status) {
  std::vector<int> hs(batch);
  if (cudaMemcpy(hs.data(), dstatus, sizeof(int) * batch, cudaMemcpyDeviceToHost) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "status download failed");
  int first = RCWA_OK;
  for (int b = 0; b < batch; ++b) {
    if (status) status[b] = hs[b];
    if (first == RCWA_OK && hs[b] != RCWA_OK) first = hs[b];
  }
  if (first != RCWA_OK) set_err(e, first, "singular matrix in the S-matrix computation");
  return first;
}

// The slab S-matrices of rcwa_slab_smatrix_batched on device buffers: items
// contiguous with stride n*n (gamma: n).  W, V are factorised in place; F0,
// G0 hold copies of W0, V0 on entry and W^-1 W0, V^-1 V0 on return; R2[b]
// (n x 2n) receives [Rud | Tuu]; ss[b] (host) = wz lambda / 2pi; stat[b]
// (device) takes RCWA_ERR_SINGULAR.  Waits for its work before returning.
int slab_core(rcwa_engine* e, int n, int batch, cplx* Wd, cplx* Vd, cplx* F0, cplx* G0, const cplx* gam,
              const double* ss, cplx* R2, int* stat, cudaStream_t st) {
  const size_t nn = (size_t)n * n, tot = nn * batch;
  Buf dA(sizeof(cplx) * tot), dR3(sizeof(cplx) * 3 * tot), dM(sizeof(cplx) * tot),
      dpiv(sizeof(int) * 2 * n * batch), dinfo(sizeof(int) * 2 * batch), ditems(sizeof(SlabRhsItem) * batch);
  if (!dA.p || !dR3.p || !dM.p || !dpiv.p || !dinfo.p || !ditems.p)
    return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  std::vector<SlabRhsItem> items(batch);
  for (int b = 0; b < batch; ++b) {
    items[b].F0 = F0 + nn * b;
    items[b].G0 = G0 + nn * b;
    items[b].gamma = gam + (size_t)n * b;
    items[b].ss = ss[b];
    items[b].A = dA.c() + nn * b;
    items[b].R3 = dR3.c() + 3 * nn * b;
  }
  PtrBlob pb;
  const size_t pW = pb.add(Wd, nn, 0, batch), pV = pb.add(Vd, nn, 0, batch);
  const size_t pWV = pb.h.size();
  for (size_t k = 0; k < (size_t)2 * batch; ++k) pb.h.push_back(pb.h[k < (size_t)batch ? pW + k : pV + k - batch]);
  const size_t pF = pb.add(F0, nn, 0, batch), pG = pb.add(G0, nn, 0, batch);
  const size_t pFG = pb.h.size();
  for (size_t k = 0; k < (size_t)2 * batch; ++k) pb.h.push_back(pb.h[k < (size_t)batch ? pF + k : pG + k - batch]);
  const size_t pA = pb.add(dA.c(), nn, 0, batch);
  const size_t pR3 = pb.add(dR3.c(), 3 * nn, 0, batch);
  const size_t pR3a = pb.add(dR3.c(), 3 * nn, n, batch);      // invAXA block
  const size_t pR3b = pb.add(dR3.c(), 3 * nn, 2 * n, batch);  // invAXB block
  const size_t pM = pb.add(dM.c(), nn, 0, batch);
  const size_t pR2 = pb.add(R2, 2 * nn, 0, batch);
  const size_t pR2t = pb.add(R2, 2 * nn, n, batch);
  std::vector<int> item2(2 * batch), item1(batch);
  for (int b = 0; b < batch; ++b) item2[b] = item2[batch + b] = item1[b] = b;
  const size_t pI2 = pb.add_ints(item2), pI1 = pb.add_ints(item1);
  if (!pb.upload(st) ||
      cudaMemcpyAsync(ditems.p, items.data(), sizeof(SlabRhsItem) * batch, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "upload failed");
  int* piv = (int*)dpiv.p;
  int* info = (int*)dinfo.p;
  cudaError_t err = cudaSuccess;
  auto run = [&](cudaError_t x) { if (err == cudaSuccess) err = x; };
  // F0 = W^-1 W0, G0 = V^-1 V0 (:119-126)
  run(zgetrf_batched(pb.at(pWV), n, n, piv, info, 2 * batch, st));
  run(fold_info(info, pb.ints(pI2), 2 * batch, RCWA_ERR_SINGULAR, stat, st));
  run(zgetrs_batched(pb.cat(pWV), n, n, piv, pb.at(pFG), n, n, 2 * batch, st));
  // A, [B | XA | XB] (:128-134), then A^-1 applied to all three (:131-136)
  {
    dim3 grid((unsigned)std::min<size_t>(1024, (nn + 255) / 256), batch);
    slab_rhs_kernel<<<grid, 256, 0, st>>>((const SlabRhsItem*)ditems.p, n);
    ++launch_counter();
    run(cudaGetLastError());
  }
  run(zgetrf_batched(pb.at(pA), n, n, piv, info, batch, st));
  run(fold_info(info, pb.ints(pI1), batch, RCWA_ERR_SINGULAR, stat, st));
  run(zgetrs_batched(pb.cat(pA), n, n, piv, pb.at(pR3), 3 * n, 3 * n, batch, st));
  // M = I - invAXB^2 (:139)
  GemmArgs g = gemm(n, batch);
  g.A = pb.cat(pR3b); g.lda = 3 * n;
  g.B = pb.cat(pR3b); g.ldb = 3 * n;
  g.D = pb.at(pM); g.ldd = n;
  g.alpha = mkc(-1, 0); g.gammaI = mkc(1, 0);
  run(zgemm_batched(g, st));
  // [invAXB invAXA - invAB | invAXA - invAXB invAB] (:142,144)
  g = gemm(n, batch);
  g.A = pb.cat(pR3b); g.lda = 3 * n;
  g.B = pb.cat(pR3a); g.ldb = 3 * n;
  g.C = pb.cat(pR3); g.ldc = 3 * n; g.beta = mkc(-1, 0);
  g.D = pb.at(pR2); g.ldd = 2 * n;
  run(zgemm_batched(g, st));
  g.B = pb.cat(pR3);
  g.C = pb.cat(pR3a); g.beta = mkc(1, 0);
  g.alpha = mkc(-1, 0);
  g.D = pb.at(pR2t);
  run(zgemm_batched(g, st));
  // Rud, Tuu = M^-1 [..] (:143,145)
  run(zgetrf_batched(pb.at(pM), n, n, piv, info, batch, st));
  run(fold_info(info, pb.ints(pI1), batch, RCWA_ERR_SINGULAR, stat, st));
  run(zgetrs_batched(pb.cat(pM), n, n, piv, pb.at(pR2), 2 * n, 2 * n, batch, st));
  if (err != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "slab S-matrix kernels failed");
  return RCWA_OK;
}

// The star product of rcwa_star_product_batched over pointer lists: up[k][b]
// (k: Rud, Rdu, Tdd, Tuu) the running S-matrix of item b, updated in place;
// lo[k][b] the S-matrix below it; stat[stat_id[b]] takes RCWA_ERR_SINGULAR.
// Waits for its work before returning.
int star_core(rcwa_engine* e, int n, int batch, const std::vector<cplx*> up[4], const std::vector<cplx*> lo[4],
              int* stat, const std::vector<int>& stat_id, cudaStream_t st) {
  const size_t nn = (size_t)n * n, tot = nn * batch;
  // scratch: T0 (factorised), C1, K1, C2, T1, T2, T3, Tuu'
  enum { kRud, kRdu, kTdd, kTuu, krud, krdu, ktdd, ktuu, kT0, kC1, kK1, kC2, kT1, kT2, kT3, kTn, kCount };
  Buf dm(sizeof(cplx) * tot * (kCount - 8)), dpiv(sizeof(int) * n * batch), dinfo(sizeof(int) * batch);
  if (!dm.p || !dpiv.p || !dinfo.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  PtrBlob pb;
  size_t slot[kCount];
  for (int k = 0; k < 4; ++k) slot[k] = pb.add_list(up[k]);
  for (int k = 0; k < 4; ++k) slot[4 + k] = pb.add_list(lo[k]);
  for (int k = kT0; k < kCount; ++k) slot[k] = pb.add(dm.c() + tot * (k - kT0), nn, 0, batch);
  const size_t pI1 = pb.add_ints(stat_id);
  if (!pb.upload(st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
  int* piv = (int*)dpiv.p;
  int* info = (int*)dinfo.p;
  cudaError_t err = cudaSuccess;
  auto run = [&](cudaError_t x) { if (err == cudaSuccess) err = x; };
  // D = alpha A B + beta C + gammaI I, every operand one of the slots
  auto mm = [&](int a, int b, int d, double alpha, int c, double beta, double gI) {
    GemmArgs g = gemm(n, batch);
    g.lda = g.ldb = g.ldc = g.ldd = n;
    g.A = pb.cat(slot[a]);
    g.B = pb.cat(slot[b]);
    g.D = pb.at(slot[d]);
    g.alpha = mkc(alpha, 0);
    if (c >= 0) { g.C = pb.cat(slot[c]); g.beta = mkc(beta, 0); }
    g.gammaI = mkc(gI, 0);
    run(zgemm_batched(g, st));
  };
  // C1 = (I - rdu Rud)^-1 as an explicit inverse (core/RCWAIntegrator.cpp:57-60)
  mm(krdu, kRud, kT0, -1.0, -1, 0.0, 1.0);
  run(zgetrf_batched(pb.at(slot[kT0]), n, n, piv, info, batch, st));
  run(fold_info(info, pb.ints(pI1), batch, RCWA_ERR_SINGULAR, stat, st));
  run(zset_identity_batched(pb.at(slot[kC1]), n, n, batch, st));
  run(zgetrs_batched(pb.cat(slot[kT0]), n, n, piv, pb.at(slot[kC1]), n, n, batch, st));
  // C2 = I + Rud C1 rdu (:61-62); K1 = Rud C1 is kept for the new Rud
  mm(kRud, kC1, kK1, 1.0, -1, 0.0, 0.0);
  mm(kK1, krdu, kC2, 1.0, -1, 0.0, 1.0);
  // Rdu += Tdd rdu C2 Tuu (:64)
  mm(kTdd, krdu, kT1, 1.0, -1, 0.0, 0.0);
  mm(kT1, kC2, kT2, 1.0, -1, 0.0, 0.0);
  mm(kT2, kTuu, kRdu, 1.0, kRdu, 1.0, 0.0);
  // Tdd = Tdd C1 tdd (:65)
  mm(kTdd, kC1, kT3, 1.0, -1, 0.0, 0.0);
  mm(kT3, ktdd, kTdd, 1.0, -1, 0.0, 0.0);
  // Rud = rud + tuu Rud C1 tdd (:66)
  mm(ktuu, kK1, kT1, 1.0, -1, 0.0, 0.0);
  mm(kT1, ktdd, kRud, 1.0, krud, 1.0, 0.0);
  // Tuu = tuu C2 Tuu (:67)
  mm(ktuu, kC2, kT2, 1.0, -1, 0.0, 0.0);
  mm(kT2, kTuu, kTn, 1.0, -1, 0.0, 0.0);
  run(zcopy_batched(pb.cat(slot[kTn]), n, pb.at(slot[kTuu]), n, n, n, batch, st));
  if (err != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "star product kernels failed");
  return RCWA_OK;
}

}  // namespace

extern "C" int rcwa_slab_smatrix_batched(rcwa_engine* e, int n, int batch, const rcwa_cplx* W, const rcwa_cplx* V,
                                         const rcwa_cplx* gamma, const rcwa_cplx* W0, const rcwa_cplx* V0,
                                         const double* lambda, const double* wz, rcwa_cplx* Rud, rcwa_cplx* Tuu,
                                         int* status) {
  if (!e || n < 1 || batch < 1 || !W || !V || !gamma || !W0 || !V0 || !lambda || !wz || !Rud || !Tuu)
    return RCWA_ERR_INVALID;
  for (int b = 0; b < batch; ++b)
    if (!(lambda[b] > 0.0) || !std::isfinite(lambda[b]) || !std::isfinite(wz[b]))
      return set_err(e, RCWA_ERR_INVALID, "lambda must be positive and wz finite");
  if (cudaSetDevice(e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  const size_t nn = (size_t)n * n, tot = nn * batch;
  Buf dWV(sizeof(cplx) * 2 * tot), dFG(sizeof(cplx) * 2 * tot), dg(sizeof(cplx) * n * batch),
      dR2(sizeof(cplx) * 2 * tot), dstat(sizeof(int) * batch);
  if (!dWV.p || !dFG.p || !dg.p || !dR2.p || !dstat.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  cplx* Wd = dWV.c();
  cplx* Vd = Wd + tot;
  cplx* F0 = dFG.c();
  cplx* G0 = F0 + tot;
  cudaStream_t st = e->stream;
  if (!up(Wd, W, tot, st) || !up(Vd, V, tot, st) || !up(F0, W0, tot, st) || !up(G0, V0, tot, st) ||
      !up(dg.c(), gamma, n * batch, st) || cudaMemsetAsync(dstat.p, 0, sizeof(int) * batch, st) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "upload failed");
  std::vector<double> ss(batch);
  for (int b = 0; b < batch; ++b) ss[b] = lambda[b] / (2.0 * 3.14159265358979323846) * wz[b];
  const int rc = slab_core(e, n, batch, Wd, Vd, F0, G0, dg.c(), ss.data(), dR2.c(), (int*)dstat.p, st);
  if (rc != RCWA_OK) return rc;
  const size_t row = sizeof(cplx) * n;
  if (cudaMemcpy2D(Rud, row, dR2.c(), 2 * row, row, (size_t)n * batch, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy2D(Tuu, row, dR2.c() + n, 2 * row, row, (size_t)n * batch, cudaMemcpyDeviceToHost) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "download failed");
  return finish_status(e, (const int*)dstat.p, batch, status);
}

extern "C" int rcwa_star_product_batched(rcwa_engine* e, int n, int batch, rcwa_cplx* Rud, rcwa_cplx* Rdu,
                                         rcwa_cplx* Tdd, rcwa_cplx* Tuu, const rcwa_cplx* rud, const rcwa_cplx* rdu,
                                         const rcwa_cplx* tdd, const rcwa_cplx* tuu, int* status) {
  if (!e || n < 1 || batch < 1 || !Rud || !Rdu || !Tdd || !Tuu || !rud || !rdu || !tdd || !tuu)
    return RCWA_ERR_INVALID;
  if (cudaSetDevice(e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  const size_t nn = (size_t)n * n, tot = nn * batch;
  Buf dm(sizeof(cplx) * tot * 8), dstat(sizeof(int) * batch);
  if (!dm.p || !dstat.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  auto M = [&](int k) { return dm.c() + tot * k; };
  cudaStream_t st = e->stream;
  const rcwa_cplx* in[8] = {Rud, Rdu, Tdd, Tuu, rud, rdu, tdd, tuu};
  for (int k = 0; k < 8; ++k)
    if (!up(M(k), in[k], tot, st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
  if (cudaMemsetAsync(dstat.p, 0, sizeof(int) * batch, st) != cudaSuccess) return RCWA_ERR_CUDA;
  std::vector<cplx*> upl[4], lol[4];
  std::vector<int> ids(batch);
  for (int b = 0; b < batch; ++b) {
    ids[b] = b;
    for (int k = 0; k < 4; ++k) {
      upl[k].push_back(M(k) + nn * b);
      lol[k].push_back(M(4 + k) + nn * b);
    }
  }
  const int rc = star_core(e, n, batch, upl, lol, (int*)dstat.p, ids, st);
  if (rc != RCWA_OK) return rc;
  rcwa_cplx* out[4] = {Rud, Rdu, Tdd, Tuu};
  for (int k = 0; k < 4; ++k)
    if (cudaMemcpy(out[k], M(k), sizeof(cplx) * tot, cudaMemcpyDeviceToHost) != cudaSuccess)
      return set_err(e, RCWA_ERR_CUDA, "download failed");
  return finish_status(e, (const int*)dstat.p, batch, status);
}

namespace {

constexpr double kTwoPi = 2.0 * 3.14159265358979323846;

// keff = GammaSqrtOp(w) and V[:, c] = (Q W)[:, c] / keff[c] for every sample
// (rcwa/WaveEquationSolver.cpp:33-36).
__global__ void integrator_modes_kernel(const cplx* w, cplx* keff, cplx* V, int n) {
  const int b = blockIdx.y;
  const size_t nn = (size_t)n * n;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < nn; idx += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(idx % n);
    const cplx k = gamma_sqrt(w[(size_t)b * n + c]);
    V[b * nn + idx] = cmul(V[b * nn + idx], cdiv(mkc(1.0, 0.0), k));
    if (idx < (size_t)n) keff[(size_t)b * n + idx] = gamma_sqrt(w[(size_t)b * n + idx]);
  }
}

// WaveEquationSolver::solve (rcwa/WaveEquationSolver.cpp:24-37) for the
// samples P[b], Q[b] listed: W[b] the eigenvectors of P Q, keff[b] (n),
// V[b] = Q W keff^-1.  Waits for its work.
int sample_modes(rcwa_engine* e, int n, const std::vector<cplx*>& P, const std::vector<cplx*>& Q,
                 const std::vector<cplx*>& W, const std::vector<cplx*>& V, cplx* keff, cudaStream_t st) {
  const int count = (int)P.size();
  const size_t nn = (size_t)n * n;
  Buf dA(sizeof(cplx) * nn * count), dw(sizeof(cplx) * n * count), dwork(zgeev_workspace_bytes(n) * count),
      dinfo(sizeof(int) * count);
  if (!dA.p || !dw.p || !dwork.p || !dinfo.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  // the modes kernel scales V in place and needs it contiguous
  for (int b = 1; b < count; ++b)
    if (V[b] != V[0] + nn * b) return set_err(e, RCWA_ERR_INVALID, "sample modes need contiguous V");
  PtrBlob pb;
  const size_t pP = pb.add_list(P), pQ = pb.add_list(Q), pA = pb.add(dA.c(), nn, 0, count);
  const size_t pW = pb.add_list(W), pV = pb.add_list(V);
  if (!pb.upload(st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
  cudaError_t err = cudaSuccess;
  auto run = [&](cudaError_t x) { if (err == cudaSuccess) err = x; };
  GemmArgs g = gemm(n, count);
  g.lda = g.ldb = g.ldc = g.ldd = n;
  g.A = pb.cat(pP); g.B = pb.cat(pQ); g.D = pb.at(pA);
  run(zgemm_batched(g, st));
  run(zgeev_batched(pb.at(pA), n, n, dw.c(), pb.at(pW), n, dwork.p, (int*)dinfo.p, count, st));
  g.A = pb.cat(pQ); g.B = pb.cat(pW); g.D = pb.at(pV);
  run(zgemm_batched(g, st));
  dim3 grid((unsigned)std::min<size_t>(1024, (nn + 255) / 256), count);
  integrator_modes_kernel<<<grid, 256, 0, st>>>(dw.c(), keff, V[0], n);
  ++launch_counter();
  run(cudaGetLastError());
  if (err != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "mode kernels failed");
  std::vector<int> hinfo(count);
  if (cudaMemcpy(hinfo.data(), dinfo.p, sizeof(int) * count, cudaMemcpyDeviceToHost) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "download failed");
  for (int v : hinfo)
    if (v != 0) return set_err(e, v, "eigensolver failed on a sample");
  return RCWA_OK;
}

// S-matrices of a z-integrator, four matrices per item: Rud, Rdu, Tdd, Tuu.
struct SBank {
  Buf buf;
  size_t nn;
  SBank(int n, int count) : buf(sizeof(cplx) * 4 * (size_t)n * n * std::max(count, 1)), nn((size_t)n * n) {}
  cplx* at(int k, int i) const { return buf.c() + nn * ((size_t)4 * i + k); }
};

// S_0 * S_1 * ... * S_{count-1} (top to bottom) into item 0, pairwise: the
// star product is associative, so ceil(log2 count) batched levels replace
// the integrators' top-down fold.
int cascade_tree(rcwa_engine* e, int n, int count, const SBank& S, int* stat, cudaStream_t st) {
  std::vector<int> list(count);
  for (int i = 0; i < count; ++i) list[i] = i;
  while (list.size() > 1) {
    std::vector<cplx*> upl[4], lol[4];
    std::vector<int> ids, next;
    for (size_t j = 0; j + 1 < list.size(); j += 2) {
      for (int k = 0; k < 4; ++k) {
        upl[k].push_back(S.at(k, list[j]));
        lol[k].push_back(S.at(k, list[j + 1]));
      }
      ids.push_back(list[j]);
      next.push_back(list[j]);
    }
    if (list.size() % 2) next.push_back(list.back());
    const int rc = star_core(e, n, (int)ids.size(), upl, lol, stat, ids, st);
    if (rc != RCWA_OK) return rc;
    list = next;
  }
  return RCWA_OK;
}

// The integrators' last step (core/RCWAIntegrator.cpp:73-85,
// core/DifferentialIntegrator.cpp:116-133): the cascade S (item 0), built in
// the modes (Wb, Vb) at z1, brought into the modes (Wt, Vt) at z0:
//   A = (Wb^-1 Wt + Vb^-1 Vt)/2, B = (Wb^-1 Wt - Vb^-1 Vt)/2,
//   Rdu <- (A - Rdu B)^-1 (Rdu A - B), Tdd <- (A - Rdu B)^-1 Tdd,
//   Rud <- Tuu B Tdd + Rud, Tuu <- Tuu (B Rdu + A)  (new Tdd, Rdu);
// then the per-item statuses stat[0 .. nstat) are checked and the four
// blocks downloaded (NULL skips one).
int top_projection(rcwa_engine* e, int n, const SBank& S, const cplx* Wt, const cplx* Vt, const cplx* Wb,
                   const cplx* Vb, int* stat, int nstat, cudaStream_t st, rcwa_cplx* Rud, rcwa_cplx* Rdu,
                   rcwa_cplx* Tdd, rcwa_cplx* Tuu) {
  const size_t nn = (size_t)n * n;
  enum { kLW, kLV, kF, kG, kAm, kBm, kM, kX1, kX2, kT, kCnt };
  Buf dx(sizeof(cplx) * nn * kCnt), dpiv(sizeof(int) * 2 * n), dinf(sizeof(int) * 2);
  if (!dx.p || !dpiv.p || !dinf.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  auto X = [&](int k) { return dx.c() + nn * k; };
  PtrBlob pb;
  const size_t pLU = pb.add_list({X(kLW), X(kLV)});
  const size_t pFG = pb.add_list({X(kF), X(kG)});
  const size_t s0 = pb.add_list({(cplx*)Wb, (cplx*)Vb, (cplx*)Wt, (cplx*)Vt});
  const size_t d0 = pb.add_list({X(kLW), X(kLV), X(kF), X(kG)});
  auto one = [&](cplx* q) { return pb.add_list({q}); };
  const size_t pF = one(X(kF)), pG = one(X(kG)), pAm = one(X(kAm)), pBm = one(X(kBm)), pM = one(X(kM));
  const size_t pX1 = one(X(kX1)), pX2 = one(X(kX2)), pT = one(X(kT));
  const size_t pRud = one(S.at(0, 0)), pRdu = one(S.at(1, 0)), pTdd = one(S.at(2, 0)), pTuu = one(S.at(3, 0));
  const size_t pI = pb.add_ints({0, 0});
  if (!pb.upload(st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
  int* piv = (int*)dpiv.p;
  int* inf = (int*)dinf.p;
  cudaError_t err = cudaSuccess;
  auto run = [&](cudaError_t x) { if (err == cudaSuccess) err = x; };
  auto mm = [&](size_t a, size_t b, size_t d, double alpha, long c, double beta) {
    GemmArgs g = gemm(n, 1);
    g.lda = g.ldb = g.ldc = g.ldd = n;
    g.A = pb.cat(a); g.B = pb.cat(b); g.D = pb.at(d);
    g.alpha = mkc(alpha, 0);
    if (c >= 0) { g.C = pb.cat((size_t)c); g.beta = mkc(beta, 0); }
    run(zgemm_batched(g, st));
  };
  // [LW, LV, F, G] <- [Wb, Vb, Wt, Vt]; F = Wb^-1 Wt, G = Vb^-1 Vt
  run(zcopy_batched(pb.cat(s0), n, pb.at(d0), n, n, n, 4, st));
  run(zgetrf_batched(pb.at(pLU), n, n, piv, inf, 2, st));
  run(fold_info(inf, pb.ints(pI), 2, RCWA_ERR_SINGULAR, stat, st));
  run(zgetrs_batched(pb.cat(pLU), n, n, piv, pb.at(pFG), n, n, 2, st));
  run(zaxpby_batched(pb.cat(pF), pb.cat(pG), pb.at(pAm), mkc(0.5, 0), mkc(0.5, 0), n, 1, st));
  run(zaxpby_batched(pb.cat(pF), pb.cat(pG), pb.at(pBm), mkc(0.5, 0), mkc(-0.5, 0), n, 1, st));
  mm(pRdu, pBm, pM, -1.0, (long)pAm, 1.0);    // M = A - Rdu B
  mm(pRdu, pAm, pX1, 1.0, (long)pBm, -1.0);   // X1 = Rdu A - B
  run(zcopy_batched(pb.cat(pTdd), n, pb.at(pX2), n, n, n, 1, st));  // X2 = Tdd
  run(zgetrf_batched(pb.at(pM), n, n, piv, inf, 1, st));
  run(fold_info(inf, pb.ints(pI), 1, RCWA_ERR_SINGULAR, stat, st));
  run(zgetrs_batched(pb.cat(pM), n, n, piv, pb.at(pX1), n, n, 1, st));  // Rdu'
  run(zgetrs_batched(pb.cat(pM), n, n, piv, pb.at(pX2), n, n, 1, st));  // Tdd'
  mm(pBm, pX2, pT, 1.0, -1, 0.0);              // T = B Tdd'
  mm(pTuu, pT, pRud, 1.0, (long)pRud, 1.0);    // Rud' = Tuu T + Rud
  mm(pBm, pX1, pT, 1.0, (long)pAm, 1.0);       // T = B Rdu' + A
  mm(pTuu, pT, pM, 1.0, -1, 0.0);              // Tuu' (into M's storage)
  if (err != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "integrator kernels failed");
  std::vector<int> hs(nstat);
  if (cudaMemcpy(hs.data(), stat, sizeof(int) * nstat, cudaMemcpyDeviceToHost) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "download failed");
  for (int v : hs)
    if (v != RCWA_OK) return set_err(e, v, "singular matrix in the integrator");
  const size_t mb = sizeof(cplx) * nn;
  struct Out { rcwa_cplx* h; const void* d; } outs[] = {{Rud, S.at(0, 0)}, {Rdu, X(kX1)}, {Tdd, X(kX2)}, {Tuu, X(kM)}};
  for (const Out& o : outs)
    if (o.h && cudaMemcpy(o.h, o.d, mb, cudaMemcpyDeviceToHost) != cudaSuccess)
      return set_err(e, RCWA_ERR_CUDA, "download failed");
  return RCWA_OK;
}

// Downloads of the end modes (NULL skips one).
int download_modes(rcwa_engine* e, int n, const cplx* W, const cplx* V, const cplx* g, rcwa_cplx* Wh, rcwa_cplx* Vh,
                   rcwa_cplx* gh) {
  const size_t mb = sizeof(cplx) * n * n, vb = sizeof(cplx) * n;
  if ((Wh && cudaMemcpy(Wh, W, mb, cudaMemcpyDeviceToHost) != cudaSuccess) ||
      (Vh && cudaMemcpy(Vh, V, mb, cudaMemcpyDeviceToHost) != cudaSuccess) ||
      (gh && cudaMemcpy(gh, g, vb, cudaMemcpyDeviceToHost) != cudaSuccess))
    return set_err(e, RCWA_ERR_CUDA, "download failed");
  return RCWA_OK;
}

// D[b] = a X[b] + b Y[b] over `count` elements per item (any shape).
__global__ void axpby_elems_kernel(const cplx* const* X, const cplx* const* Y, cplx* const* D, cplx a, cplx bb,
                                   size_t count) {
  const int b = blockIdx.y;
  const cplx* x = X[b];
  const cplx* y = Y[b];
  cplx* d = D[b];
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    d[i] = cfma(a, x[i], cmul(bb, y[i]));
}

cudaError_t axpby_elems(const cplx* const* X, const cplx* const* Y, cplx* const* D, cplx a, cplx b, size_t count,
                        int batch, cudaStream_t st) {
  dim3 grid((unsigned)std::min<size_t>(1024, (count + 255) / 256), batch);
  axpby_elems_kernel<<<grid, 256, 0, st>>>(X, Y, D, a, b, count);
  ++launch_counter();
  return cudaGetLastError();
}

// RedhefferIntegrator::evaluatePerturbationAndDifference's combination step
// (core/RedhefferIntegrator.cpp:366-397) for one interval per blockIdx.y:
// from dA0, dB0 (left end) and dA2, dB2 (right end), with pf = exp(i L gam/k0)
// and c = i L/(12 k0):
//   tuu = c (pf dA0 + dA2 pf) + diag(pf), rud = -c (pf dB0 pf + dB2),
//   rdu = -c (dB0 + pf dB2 pf),          tdd = c (dA0 pf + pf dA2) + diag(pf);
// err = the largest |entry| of the four before the diagonal is added (bits
// of a non-negative double compare like the value).
struct PertItem {
  const cplx* dA0; const cplx* dB0; const cplx* dA2; const cplx* dB2;
  const cplx* gam;
  double L;  // interval length over k0
  cplx* tdd; cplx* tuu; cplx* rud; cplx* rdu;
  unsigned long long* err;
};

__global__ void perturbation_kernel(const PertItem* items, int n) {
  const PertItem it = items[blockIdx.y];
  const size_t nn = (size_t)n * n;
  const cplx c = mkc(0.0, it.L / 12.0), mc = mkc(0.0, -it.L / 12.0);
  double mx = 0.0;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < nn; idx += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx / n), q = (int)(idx % n);
    const cplx gr = it.gam[r], gq = it.gam[q];
    const cplx pr = cexp_(mkc(-gr.y * it.L, gr.x * it.L)), pq = cexp_(mkc(-gq.y * it.L, gq.x * it.L));
    const cplx a0 = it.dA0[idx], b0 = it.dB0[idx], a2 = it.dA2[idx], b2 = it.dB2[idx];
    const cplx tu = cmul(c, cadd(cmul(pr, a0), cmul(a2, pq)));
    const cplx ru = cmul(mc, cadd(cmul(cmul(pr, b0), pq), b2));
    const cplx rd = cmul(mc, cadd(b0, cmul(cmul(pr, b2), pq)));
    const cplx td = cmul(c, cadd(cmul(a0, pq), cmul(pr, a2)));
    mx = fmax(mx, fmax(fmax(cabs(tu), cabs(ru)), fmax(cabs(rd), cabs(td))));
    it.tuu[idx] = r == q ? cadd(tu, pr) : tu;
    it.rud[idx] = ru;
    it.rdu[idx] = rd;
    it.tdd[idx] = r == q ? cadd(td, pr) : td;
  }
  for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
  if ((threadIdx.x & 31) == 0) atomicMax(it.err, (unsigned long long)__double_as_longlong(mx));
}

bool integrator_args_ok(double lambda, double z0, double z1) {
  return lambda > 0.0 && std::isfinite(lambda) && std::isfinite(z0) && std::isfinite(z1);
}

}  // namespace

extern "C" int rcwa_rcwa_integrate(rcwa_engine* e, int n, int nslab, double lambda, double z0, double z1,
                                   const rcwa_cplx* P, const rcwa_cplx* Q, rcwa_cplx* Rud, rcwa_cplx* Rdu,
                                   rcwa_cplx* Tdd, rcwa_cplx* Tuu, rcwa_cplx* W0, rcwa_cplx* V0, rcwa_cplx* gam0,
                                   rcwa_cplx* W1, rcwa_cplx* V1, rcwa_cplx* gam1) {
  if (!e || n < 1 || nslab < 0 || !P || !Q) return RCWA_ERR_INVALID;
  if (!integrator_args_ok(lambda, z0, z1))
    return set_err(e, RCWA_ERR_INVALID, "lambda must be positive and z0, z1 finite");
  if (cudaSetDevice(e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  const int ns = nslab + 2;  // samples: z0, the slab midpoints, z1
  const size_t nn = (size_t)n * n;
  cudaStream_t st = e->stream;
  Buf dP(sizeof(cplx) * nn * ns), dQ(sizeof(cplx) * nn * ns), dW(sizeof(cplx) * nn * ns),
      dV(sizeof(cplx) * nn * ns), dk(sizeof(cplx) * n * ns), dstat(sizeof(int) * (nslab + 1));
  if (!dP.p || !dQ.p || !dW.p || !dV.p || !dk.p || !dstat.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  if (!up(dP.c(), P, nn * ns, st) || !up(dQ.c(), Q, nn * ns, st) ||
      cudaMemsetAsync(dstat.p, 0, sizeof(int) * (nslab + 1), st) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "upload failed");
  // modes of every sample (rcwa/WaveEquationSolver.cpp:24-37)
  {
    std::vector<cplx*> p(ns), q(ns), w(ns), v(ns);
    for (int b = 0; b < ns; ++b) {
      p[b] = dP.c() + nn * b; q[b] = dQ.c() + nn * b; w[b] = dW.c() + nn * b; v[b] = dV.c() + nn * b;
    }
    const int rc = sample_modes(e, n, p, q, w, v, dk.c(), st);
    if (rc != RCWA_OK) return rc;
  }
  cplx* Wt = dW.c();                  // modes at z0
  cplx* Vt = dV.c();
  cplx* Wb = dW.c() + nn * (ns - 1);  // modes at z1, the slabs' reference medium
  cplx* Vb = dV.c() + nn * (ns - 1);
  int* stat = (int*)dstat.p;
  cudaError_t err = cudaSuccess;
  auto run = [&](cudaError_t x) { if (err == cudaSuccess) err = x; };
  SBank S(n, nslab);
  if (!S.buf.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  if (nslab == 0) {
    // core/RCWAIntegrator.cpp:36-39: Tdd = Tuu = I, Rud = Rdu = 0
    PtrBlob pb;
    const size_t pR = pb.add_list({S.at(0, 0), S.at(1, 0)}), pT = pb.add_list({S.at(2, 0), S.at(3, 0)});
    if (!pb.upload(st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
    run(cascade_init(pb.at(pR), pb.at(pT), n, 2, st));
  } else {
    // the slabs' S-matrices against the modes at z1 (:41-50), each from its
    // own copies of W1, V1
    Buf dF(sizeof(cplx) * nn * nslab), dG(sizeof(cplx) * nn * nslab), dR2(sizeof(cplx) * 2 * nn * nslab);
    if (!dF.p || !dG.p || !dR2.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
    {
      PtrBlob pb;
      std::vector<cplx*> sw(nslab, Wb), sv(nslab, Vb);
      const size_t pSW = pb.add_list(sw), pSV = pb.add_list(sv);
      const size_t pF = pb.add(dF.c(), nn, 0, nslab), pG = pb.add(dG.c(), nn, 0, nslab);
      if (!pb.upload(st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
      run(zcopy_batched(pb.cat(pSW), n, pb.at(pF), n, n, n, nslab, st));
      run(zcopy_batched(pb.cat(pSV), n, pb.at(pG), n, n, n, nslab, st));
      if (err != cudaSuccess) return set_err(e, RCWA_ERR_CUDA, "copy failed");
      std::vector<double> ss(nslab, lambda / kTwoPi * ((z1 - z0) / nslab));
      const int rc = slab_core(e, n, nslab, dW.c() + nn, dV.c() + nn, dF.c(), dG.c(), dk.c() + n, ss.data(),
                               dR2.c(), stat, st);
      if (rc != RCWA_OK) return rc;
    }
    {
      // a slab is symmetric: rdu = rud, tdd = tuu (rcwa/RCWAScatterMatrix.h:40-47)
      PtrBlob pb;
      const size_t pRl = pb.add(dR2.c(), 2 * nn, 0, nslab), pTl = pb.add(dR2.c(), 2 * nn, n, nslab);
      std::vector<cplx*> d[4];
      for (int i = 0; i < nslab; ++i)
        for (int k = 0; k < 4; ++k) d[k].push_back(S.at(k, i));
      size_t pd[4];
      for (int k = 0; k < 4; ++k) pd[k] = pb.add_list(d[k]);
      if (!pb.upload(st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
      run(zcopy_batched(pb.cat(pRl), 2 * n, pb.at(pd[0]), n, n, n, nslab, st));
      run(zcopy_batched(pb.cat(pRl), 2 * n, pb.at(pd[1]), n, n, n, nslab, st));
      run(zcopy_batched(pb.cat(pTl), 2 * n, pb.at(pd[2]), n, n, n, nslab, st));
      run(zcopy_batched(pb.cat(pTl), 2 * n, pb.at(pd[3]), n, n, n, nslab, st));
      if (err != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
        return set_err(e, RCWA_ERR_CUDA, "copy failed");
    }
    // the cascade from the top down (:41-68)
    const int rc = cascade_tree(e, n, nslab, S, stat, st);
    if (rc != RCWA_OK) return rc;
  }
  int rc = top_projection(e, n, S, Wt, Vt, Wb, Vb, stat, nslab + 1, st, Rud, Rdu, Tdd, Tuu);
  if (rc == RCWA_OK) rc = download_modes(e, n, Wt, Vt, dk.c(), W0, V0, gam0);
  if (rc == RCWA_OK) rc = download_modes(e, n, Wb, Vb, dk.c() + (size_t)n * (ns - 1), W1, V1, gam1);
  return rc;
}

extern "C" int rcwa_differential_integrate(rcwa_engine* e, int n, int nslab, double lambda, double z0, double z1,
                                           const rcwa_cplx* P, const rcwa_cplx* Q, rcwa_cplx* Rud, rcwa_cplx* Rdu,
                                           rcwa_cplx* Tdd, rcwa_cplx* Tuu, rcwa_cplx* W0, rcwa_cplx* V0,
                                           rcwa_cplx* gam0, rcwa_cplx* W1, rcwa_cplx* V1, rcwa_cplx* gam1) {
  if (!e || n < 1 || nslab < 1 || !P || !Q) return RCWA_ERR_INVALID;
  if (!integrator_args_ok(lambda, z0, z1))
    return set_err(e, RCWA_ERR_INVALID, "lambda must be positive and z0, z1 finite");
  if (cudaSetDevice(e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  const int N = nslab;
  const int ns = 2 * N + 1;  // samples at z0 + k dz/2
  const size_t nn = (size_t)n * n;
  cudaStream_t st = e->stream;
  Buf dP(sizeof(cplx) * nn * ns), dQ(sizeof(cplx) * nn * ns), dW(sizeof(cplx) * nn * 2), dV(sizeof(cplx) * nn * 2),
      dk(sizeof(cplx) * n * 2), dstat(sizeof(int) * (N + 1));
  if (!dP.p || !dQ.p || !dW.p || !dV.p || !dk.p || !dstat.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  if (!up(dP.c(), P, nn * ns, st) || !up(dQ.c(), Q, nn * ns, st) ||
      cudaMemsetAsync(dstat.p, 0, sizeof(int) * (N + 1), st) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "upload failed");
  auto Ps = [&](int k) { return dP.c() + nn * k; };
  auto Qs = [&](int k) { return dQ.c() + nn * k; };
  // modes at z0 (sample 0) and z1 (sample 2N)  (:26-29, :115-116)
  {
    const int rc = sample_modes(e, n, {Ps(0), Ps(2 * N)}, {Qs(0), Qs(2 * N)}, {dW.c(), dW.c() + nn},
                                {dV.c(), dV.c() + nn}, dk.c(), st);
    if (rc != RCWA_OK) return rc;
  }
  cplx* Wt = dW.c();
  cplx* Vt = dV.c();
  cplx* Wb = dW.c() + nn;
  cplx* Vb = dV.c() + nn;
  int* stat = (int*)dstat.p;
  cudaError_t err = cudaSuccess;
  auto run = [&](cudaError_t x) { if (err == cudaSuccess) err = x; };
  // W1^-1 and V1^-1 once (the reference solves with their LU per slab,
  // :31-34, :73-76)
  Buf dinv(sizeof(cplx) * nn * 4), dpiv(sizeof(int) * 2 * n), dinf(sizeof(int) * 2);
  if (!dinv.p || !dpiv.p || !dinf.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  cplx* iW = dinv.c();
  cplx* iV = dinv.c() + nn;
  {
    PtrBlob pb;
    const size_t src = pb.add_list({Wb, Vb}), pLU = pb.add_list({dinv.c() + 2 * nn, dinv.c() + 3 * nn});
    const size_t pInv = pb.add_list({iW, iV});
    const size_t pI = pb.add_ints({0, 0});
    if (!pb.upload(st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
    run(zcopy_batched(pb.cat(src), n, pb.at(pLU), n, n, n, 2, st));
    run(zgetrf_batched(pb.at(pLU), n, n, (int*)dpiv.p, (int*)dinf.p, 2, st));
    run(fold_info((int*)dinf.p, pb.ints(pI), 2, RCWA_ERR_SINGULAR, stat, st));
    run(zset_identity_batched(pb.at(pInv), n, n, 2, st));
    run(zgetrs_batched(pb.cat(pLU), n, n, (int*)dpiv.p, pb.at(pInv), n, n, 2, st));
    if (err != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
      return set_err(e, RCWA_ERR_CUDA, "integrator kernels failed");
  }
  // per slab, all slabs at once: the transfer blocks L (:55-66), A (:73-81),
  // T (:83-86) and the slab S-matrix (:93-97)
  enum { t1, t2, t3, t4, t5, t6, kL11, kL12, kL21, kL22, kX1, kX2, kY1, kY2, kA11, kA12, kA21, kA22, kU1, kU2, kU3,
         kU4, kT11, kT12, kT21, kT22, kCnt };
  Buf dw(sizeof(cplx) * nn * kCnt * N), dp2(sizeof(int) * n * N), dinfo(sizeof(int) * N);
  if (!dw.p || !dp2.p || !dinfo.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  auto Wk = [&](int k, int i) { return dw.c() + nn * ((size_t)kCnt * i + k); };
  SBank S(n, N);
  if (!S.buf.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  PtrBlob pb;
  auto list = [&](const std::function<cplx*(int)>& f) {
    std::vector<cplx*> v(N);
    for (int i = 0; i < N; ++i) v[i] = f(i);
    return pb.add_list(v);
  };
  const size_t P0 = list([&](int i) { return Ps(2 * i); }), P1 = list([&](int i) { return Ps(2 * i + 1); }),
               P2 = list([&](int i) { return Ps(2 * i + 2); });
  const size_t Q0 = list([&](int i) { return Qs(2 * i); }), Q1 = list([&](int i) { return Qs(2 * i + 1); }),
               Q2 = list([&](int i) { return Qs(2 * i + 2); });
  size_t w[kCnt];
  for (int k = 0; k < kCnt; ++k) w[k] = list([&](int i) { return Wk(k, i); });
  const size_t iWl = list([&](int) { return iW; }), iVl = list([&](int) { return iV; });
  const size_t Wbl = list([&](int) { return Wb; }), Vbl = list([&](int) { return Vb; });
  size_t Sk[4];
  for (int k = 0; k < 4; ++k) Sk[k] = list([&](int i) { return S.at(k, i); });
  std::vector<int> ids(N);
  for (int i = 0; i < N; ++i) ids[i] = i;
  const size_t pIds = pb.add_ints(ids);
  if (!pb.upload(st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
  const double k0 = kTwoPi / lambda, dz = (z1 - z0) / N;
  const double c = dz * dz / (k0 * k0);
  const cplx beta = mkc(0.0, dz / (6.0 * k0));
  const cplx one = mkc(1, 0);
  // D = alpha A B + bC C + gI I (n x n, batch N)
  auto mm = [&](size_t a, size_t b, size_t d, cplx alpha, long cC, double bC, double gI) {
    GemmArgs g = gemm(n, N);
    g.lda = g.ldb = g.ldc = g.ldd = n;
    g.A = pb.cat(a); g.B = pb.cat(b); g.D = pb.at(d);
    g.alpha = alpha;
    if (cC >= 0) { g.C = pb.cat((size_t)cC); g.beta = mkc(bC, 0); }
    g.gammaI = mkc(gI, 0);
    run(zgemm_batched(g, st));
  };
  // D = a X + b Y elementwise
  auto ax = [&](size_t x, size_t y, size_t d, cplx a, cplx b) {
    run(axpby_elems(pb.cat(x), pb.cat(y), pb.at(d), a, b, nn, N, st));
  };
  mm(P1, Q0, w[t1], one, -1, 0, 0);   // P1 Q0
  mm(P2, Q1, w[t2], one, -1, 0, 0);   // P2 Q1
  mm(P1, Q1, w[t3], one, -1, 0, 0);   // P1 Q1
  mm(Q1, P1, w[t4], one, -1, 0, 0);   // Q1 P1
  mm(Q2, P1, w[t5], one, -1, 0, 0);   // Q2 P1
  mm(Q1, P0, w[t6], one, -1, 0, 0);   // Q1 P0
  const double c2 = c / 6.0, c4 = c / 4.0;
  const cplx mc2 = mkc(-c2, 0.0), bh = cscale(beta, -0.5 * c), b4 = cscale(beta, 4.0);
  // L11 = I - c/6 (P1Q0 + P1Q1 + P2Q1 - c/4 P2Q1 P1Q0)
  mm(w[t2], w[t1], w[kL11], mkc(c2 * c4, 0), -1, 0, 1.0);
  ax(w[kL11], w[t1], w[kL11], one, mc2);
  ax(w[kL11], w[t3], w[kL11], one, mc2);
  ax(w[kL11], w[t2], w[kL11], one, mc2);
  // L12 = i dz/(6 k0) (P0 + 4 P1 + P2 - c/2 (P1Q1 P0 + P2Q1 P1))
  mm(w[t3], P0, w[kL12], bh, -1, 0, 0);
  mm(w[t2], P1, w[kL12], bh, (long)w[kL12], 1.0, 0);
  ax(w[kL12], P0, w[kL12], one, beta);
  ax(w[kL12], P1, w[kL12], one, b4);
  ax(w[kL12], P2, w[kL12], one, beta);
  // L21 = i dz/(6 k0) (Q0 + 4 Q1 + Q2 - c/2 (Q1P1 Q0 + Q2P1 Q1))
  mm(w[t4], Q0, w[kL21], bh, -1, 0, 0);
  mm(w[t5], Q1, w[kL21], bh, (long)w[kL21], 1.0, 0);
  ax(w[kL21], Q0, w[kL21], one, beta);
  ax(w[kL21], Q1, w[kL21], one, b4);
  ax(w[kL21], Q2, w[kL21], one, beta);
  // L22 = I - c/6 (Q1P0 + Q1P1 + Q2P1 - c/4 Q2P1 Q1P0)
  mm(w[t5], w[t6], w[kL22], mkc(c2 * c4, 0), -1, 0, 1.0);
  ax(w[kL22], w[t6], w[kL22], one, mc2);
  ax(w[kL22], w[t4], w[kL22], one, mc2);
  ax(w[kL22], w[t5], w[kL22], one, mc2);
  // A11 = (W1^-1 L11 + V1^-1 L21)/2, A12 = (W1^-1 L12 + V1^-1 L22)/2,
  // A21, A22 the differences (:73-81)
  mm(iWl, w[kL11], w[kX1], one, -1, 0, 0);
  mm(iWl, w[kL12], w[kX2], one, -1, 0, 0);
  mm(iVl, w[kL21], w[kY1], one, -1, 0, 0);
  mm(iVl, w[kL22], w[kY2], one, -1, 0, 0);
  const cplx h = mkc(0.5, 0), mh = mkc(-0.5, 0);
  ax(w[kX1], w[kY1], w[kA11], h, h);
  ax(w[kX2], w[kY2], w[kA12], h, h);
  ax(w[kX1], w[kY1], w[kA21], h, mh);
  ax(w[kX2], w[kY2], w[kA22], h, mh);
  // T11 = A11 W1 + A12 V1, T12 = A11 W1 - A12 V1, T21, T22 likewise (:83-86)
  mm(w[kA11], Wbl, w[kU1], one, -1, 0, 0);
  mm(w[kA12], Vbl, w[kU2], one, -1, 0, 0);
  mm(w[kA21], Wbl, w[kU3], one, -1, 0, 0);
  mm(w[kA22], Vbl, w[kU4], one, -1, 0, 0);
  ax(w[kU1], w[kU2], w[kT11], one, one);
  ax(w[kU1], w[kU2], w[kT12], one, mkc(-1, 0));
  ax(w[kU3], w[kU4], w[kT21], one, one);
  ax(w[kU3], w[kU4], w[kT22], one, mkc(-1, 0));
  // tdd = T22^-1, rdu = -T22^-1 T21, rud = T12 tdd, tuu = T11 + T12 rdu
  // (:93-97), into the bank (Rud, Rdu, Tdd, Tuu)
  run(zset_identity_batched(pb.at(Sk[2]), n, n, N, st));
  run(zcopy_batched(pb.cat(w[kT21]), n, pb.at(Sk[1]), n, n, n, N, st));
  run(zgetrf_batched(pb.at(w[kT22]), n, n, (int*)dp2.p, (int*)dinfo.p, N, st));
  run(fold_info((int*)dinfo.p, pb.ints(pIds), N, RCWA_ERR_SINGULAR, stat, st));
  run(zgetrs_batched(pb.cat(w[kT22]), n, n, (int*)dp2.p, pb.at(Sk[2]), n, n, N, st));
  run(zgetrs_batched(pb.cat(w[kT22]), n, n, (int*)dp2.p, pb.at(Sk[1]), n, n, N, st));
  ax(Sk[1], Sk[1], Sk[1], mkc(-1, 0), mkc(0, 0));
  mm(w[kT12], Sk[2], Sk[0], one, -1, 0, 0);
  mm(w[kT12], Sk[1], Sk[3], one, (long)w[kT11], 1.0, 0);
  if (err != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "integrator kernels failed");
  // the cascade from the top down (:98-114), then the modes at z0 on top
  int rc = cascade_tree(e, n, N, S, stat, st);
  if (rc == RCWA_OK) rc = top_projection(e, n, S, Wt, Vt, Wb, Vb, stat, N + 1, st, Rud, Rdu, Tdd, Tuu);
  if (rc == RCWA_OK) rc = download_modes(e, n, Wt, Vt, dk.c(), W0, V0, gam0);
  if (rc == RCWA_OK) rc = download_modes(e, n, Wb, Vb, dk.c() + n, W1, V1, gam1);
  return rc;
}

namespace {

// Modes, explicit inverses and samples of the Redheffer integrator's
// reference depths; every block of device memory is kept until the call ends.
struct RedRef {
  cplx* P; cplx* Q;            // the sample at the reference depth
  cplx* W; cplx* V; cplx* iW; cplx* iV; cplx* gam;
};
struct RedSample { cplx* P; cplx* Q; };
struct RedInterval {
  double za, zb;
  RedSample a, b;  // end samples
  int ref;         // the midpoint's modes
};

// A <- ..., one batched projection of items onto their own modes from the
// modes left of them (core/RedhefferIntegrator.cpp:278-288, the top-side
// projection): F = iW leftW, G = iV leftV, A = (F + G)/2, B = (F - G)/2,
//   M = A - rdu B, rdu <- M^-1 (rdu A - B), tdd <- M^-1 tdd,
//   rud <- tuu B tdd + rud, tuu <- tuu (A + B rdu)   (new tdd, rdu).
int project_items(rcwa_engine* e, int n, const std::vector<cplx*> iW, const std::vector<cplx*> iV,
                  const std::vector<cplx*> lW, const std::vector<cplx*> lV, const SBank& S, int* stat,
                  cudaStream_t st) {
  const int m = (int)iW.size();
  const size_t nn = (size_t)n * n;
  enum { kF, kG, kA, kB, kM, kX1, kT, kCnt };
  Buf dx(sizeof(cplx) * nn * kCnt * m), dpiv(sizeof(int) * n * m), dinf(sizeof(int) * m);
  if (!dx.p || !dpiv.p || !dinf.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  PtrBlob pb;
  auto X = [&](int k) { return pb.add(dx.c() + nn * k, nn * kCnt, 0, m); };
  const size_t pF = X(kF), pG = X(kG), pA = X(kA), pB = X(kB), pM = X(kM), pX1 = X(kX1), pT = X(kT);
  const size_t piW = pb.add_list(iW), piV = pb.add_list(iV), plW = pb.add_list(lW), plV = pb.add_list(lV);
  size_t Sk[4];
  for (int k = 0; k < 4; ++k) {
    std::vector<cplx*> v(m);
    for (int i = 0; i < m; ++i) v[i] = S.at(k, i);
    Sk[k] = pb.add_list(v);
  }
  std::vector<int> ids(m);
  for (int i = 0; i < m; ++i) ids[i] = 0;
  const size_t pI = pb.add_ints(ids);
  if (!pb.upload(st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
  cudaError_t err = cudaSuccess;
  auto run = [&](cudaError_t x) { if (err == cudaSuccess) err = x; };
  auto mm = [&](size_t a, size_t b, size_t d, double alpha, long c, double beta) {
    GemmArgs g = gemm(n, m);
    g.lda = g.ldb = g.ldc = g.ldd = n;
    g.A = pb.cat(a); g.B = pb.cat(b); g.D = pb.at(d);
    g.alpha = mkc(alpha, 0);
    if (c >= 0) { g.C = pb.cat((size_t)c); g.beta = mkc(beta, 0); }
    run(zgemm_batched(g, st));
  };
  enum { kRud, kRdu, kTdd, kTuu };
  mm(piW, plW, pF, 1.0, -1, 0.0);
  mm(piV, plV, pG, 1.0, -1, 0.0);
  run(axpby_elems(pb.cat(pF), pb.cat(pG), pb.at(pA), mkc(0.5, 0), mkc(0.5, 0), nn, m, st));
  run(axpby_elems(pb.cat(pF), pb.cat(pG), pb.at(pB), mkc(0.5, 0), mkc(-0.5, 0), nn, m, st));
  mm(Sk[kRdu], pB, pM, -1.0, (long)pA, 1.0);     // M = A - rdu B
  mm(Sk[kRdu], pA, pX1, 1.0, (long)pB, -1.0);    // X1 = rdu A - B
  run(zgetrf_batched(pb.at(pM), n, n, (int*)dpiv.p, (int*)dinf.p, m, st));
  run(fold_info((int*)dinf.p, pb.ints(pI), m, RCWA_ERR_SINGULAR, stat, st));
  run(zgetrs_batched(pb.cat(pM), n, n, (int*)dpiv.p, pb.at(pX1), n, n, m, st));          // rdu'
  run(zgetrs_batched(pb.cat(pM), n, n, (int*)dpiv.p, pb.at(Sk[kTdd]), n, n, m, st));     // tdd'
  run(zcopy_batched(pb.cat(pX1), n, pb.at(Sk[kRdu]), n, n, n, m, st));
  mm(pB, Sk[kTdd], pT, 1.0, -1, 0.0);                  // T = B tdd'
  mm(Sk[kTuu], pT, Sk[kRud], 1.0, (long)Sk[kRud], 1.0);  // rud' = tuu T + rud
  mm(pB, Sk[kRdu], pT, 1.0, (long)pA, 1.0);            // T = A + B rdu'
  mm(Sk[kTuu], pT, pM, 1.0, -1, 0.0);                  // tuu'
  run(zcopy_batched(pb.cat(pM), n, pb.at(Sk[kTuu]), n, n, n, m, st));
  if (err != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "projection kernels failed");
  return RCWA_OK;
}

}  // namespace

extern "C" int rcwa_redheffer_integrate(rcwa_engine* e, int n, double lambda, double z0, double z1, double pe,
                                        int max_intervals, rcwa_sampler sample, void* user, rcwa_cplx* Rud,
                                        rcwa_cplx* Rdu, rcwa_cplx* Tdd, rcwa_cplx* Tuu, rcwa_cplx* W0,
                                        rcwa_cplx* V0, rcwa_cplx* gam0, rcwa_cplx* W1, rcwa_cplx* V1,
                                        rcwa_cplx* gam1, int* n_intervals, int* n_eig) {
  if (!e || n < 1 || !sample || max_intervals < 1 || !(pe > 0.0) || !std::isfinite(pe)) return RCWA_ERR_INVALID;
  if (!integrator_args_ok(lambda, z0, z1) || !(z1 > z0))
    return set_err(e, RCWA_ERR_INVALID, "lambda must be positive and z0 < z1 finite");
  if (cudaSetDevice(e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  const size_t nn = (size_t)n * n;
  const double k0 = kTwoPi / lambda;
  cudaStream_t st = e->stream;
  std::vector<std::unique_ptr<Buf>> keep;  // device blocks alive until the end
  auto alloc = [&](size_t bytes) -> cplx* {
    keep.emplace_back(new Buf(bytes));
    return keep.back()->c();
  };
  Buf dstat(sizeof(int));
  if (!dstat.p || cudaMemsetAsync(dstat.p, 0, sizeof(int), st) != cudaSuccess)
    return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  int* stat = (int*)dstat.p;
  std::map<double, RedSample> samples;
  std::vector<RedRef> refs;
  int n_eig_solves = 0;
  // the sampler at every depth in zs not seen yet, uploaded as one block
  std::vector<rcwa_cplx> hP(nn), hQ(nn);
  auto fetch = [&](const std::vector<double>& zs) -> int {
    std::vector<double> fresh;
    for (double z : zs)
      if (!samples.count(z) && std::find(fresh.begin(), fresh.end(), z) == fresh.end()) fresh.push_back(z);
    if (fresh.empty()) return RCWA_OK;
    cplx* blk = alloc(sizeof(cplx) * 2 * nn * fresh.size());
    if (!blk) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
    for (size_t i = 0; i < fresh.size(); ++i) {
      if (sample(user, fresh[i], hP.data(), hQ.data()) != 0) return set_err(e, RCWA_ERR_INVALID, "sampler failed");
      RedSample sm{blk + 2 * nn * i, blk + 2 * nn * i + nn};
      // ordered on the engine's stream ahead of the kernels that read them
      // (pageable sources are staged before the call returns)
      if (!up(sm.P, hP.data(), nn, st) || !up(sm.Q, hQ.data(), nn, st))
        return set_err(e, RCWA_ERR_CUDA, "upload failed");
      samples[fresh[i]] = sm;
    }
    return RCWA_OK;
  };
  // modes (and, with inv, explicit inverses of W and V) at the depths zs,
  // appended to refs
  auto make_refs = [&](const std::vector<double>& zs, bool inv) -> int {
    const int m = (int)zs.size();
    if (m == 0) return RCWA_OK;
    cplx* blk = alloc(sizeof(cplx) * ((size_t)4 * nn * m + (size_t)n * m));
    if (!blk) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
    std::vector<cplx*> p(m), q(m), w(m), v(m);
    const int base = (int)refs.size();
    for (int i = 0; i < m; ++i) {
      const RedSample& sm = samples.at(zs[i]);
      RedRef r{sm.P, sm.Q, blk + nn * i, blk + nn * (m + i), blk + nn * (2 * m + i), blk + nn * (3 * m + i),
               blk + 4 * nn * m + (size_t)n * i};
      refs.push_back(r);
      p[i] = r.P; q[i] = r.Q; w[i] = r.W; v[i] = r.V;
    }
    int rc = sample_modes(e, n, p, q, w, v, refs[base].gam, st);
    if (rc != RCWA_OK) return rc;
    n_eig_solves += m;
    if (!inv) return RCWA_OK;
    Buf lu(sizeof(cplx) * 2 * nn * m), piv(sizeof(int) * 2 * n * m), inf(sizeof(int) * 2 * m);
    if (!lu.p || !piv.p || !inf.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
    PtrBlob pb;
    std::vector<cplx*> src, idv;
    for (int i = 0; i < m; ++i) { src.push_back(w[i]); idv.push_back(refs[base + i].iW); }
    for (int i = 0; i < m; ++i) { src.push_back(v[i]); idv.push_back(refs[base + i].iV); }
    const size_t pS = pb.add_list(src), pL = pb.add(lu.c(), nn, 0, 2 * m), pInv = pb.add_list(idv);
    const size_t pI = pb.add_ints(std::vector<int>(2 * m, 0));
    if (!pb.upload(st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
    cudaError_t err = cudaSuccess;
    auto run = [&](cudaError_t x) { if (err == cudaSuccess) err = x; };
    run(zcopy_batched(pb.cat(pS), n, pb.at(pL), n, n, n, 2 * m, st));
    run(zgetrf_batched(pb.at(pL), n, n, (int*)piv.p, (int*)inf.p, 2 * m, st));
    run(fold_info((int*)inf.p, pb.ints(pI), 2 * m, RCWA_ERR_SINGULAR, stat, st));
    run(zset_identity_batched(pb.at(pInv), n, n, 2 * m, st));
    run(zgetrs_batched(pb.cat(pL), n, n, (int*)piv.p, pb.at(pInv), n, n, 2 * m, st));
    if (err != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
      return set_err(e, RCWA_ERR_CUDA, "inverse kernels failed");
    return RCWA_OK;
  };
  // the ends and the first midpoint (:197-211)
  const double zm = 0.5 * (z0 + z1);
  int rc = fetch({z0, z1, zm});
  if (rc == RCWA_OK) rc = make_refs({z0, z1}, false);
  if (rc == RCWA_OK) rc = make_refs({zm}, true);
  if (rc != RCWA_OK) return rc;
  const RedRef top = refs[0], bottom = refs[1];
  std::vector<RedInterval> pending{{z0, z1, samples.at(z0), samples.at(z1), 2}};
  struct Accepted { double za; int ref; cplx* S; };  // S: Rud, Rdu, Tdd, Tuu contiguous
  std::vector<Accepted> acc;
  for (int level = 0; !pending.empty(); ++level) {
    if (level > 40) return set_err(e, RCWA_ERR_NOCONV, "interval subdivision did not settle");
    // perturbation S-matrices of the pending intervals, 64 at a time
    std::vector<RedInterval> next;
    std::vector<double> split_z, ref_z;
    for (size_t c0 = 0; c0 < pending.size(); c0 += 64) {
      const int m = (int)std::min<size_t>(64, pending.size() - c0);
      enum { kD0, kE0, kD2, kE2, kX0, kY0, kX2, kY2, kx0, ky0, kx2, ky2, kA0, kB0, kA2, kB2, kCnt };
      Buf dt(sizeof(cplx) * nn * kCnt * m), derr(sizeof(unsigned long long) * m), ditems(sizeof(PertItem) * m);
      cplx* Sblk = alloc(sizeof(cplx) * 4 * nn * m);
      if (!dt.p || !derr.p || !ditems.p || !Sblk) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
      auto T = [&](int k, int i) { return dt.c() + nn * ((size_t)kCnt * i + k); };
      PtrBlob pb;
      auto lst = [&](const std::function<cplx*(int)>& f) {
        std::vector<cplx*> v(m);
        for (int i = 0; i < m; ++i) v[i] = f(i);
        return pb.add_list(v);
      };
      const RedInterval* iv = pending.data() + c0;
      const size_t Pa = lst([&](int i) { return iv[i].a.P; }), Qa = lst([&](int i) { return iv[i].a.Q; });
      const size_t Pb = lst([&](int i) { return iv[i].b.P; }), Qb = lst([&](int i) { return iv[i].b.Q; });
      auto ref_of = [&](int i) -> const RedRef& { return refs[iv[i].ref]; };
      const size_t Pr = lst([&](int i) { return ref_of(i).P; }), Qr = lst([&](int i) { return ref_of(i).Q; });
      const size_t Wr = lst([&](int i) { return ref_of(i).W; }), Vr = lst([&](int i) { return ref_of(i).V; });
      const size_t iWr = lst([&](int i) { return ref_of(i).iW; }), iVr = lst([&](int i) { return ref_of(i).iV; });
      size_t t[kCnt];
      for (int k = 0; k < kCnt; ++k) t[k] = lst([&](int i) { return T(k, i); });
      if (!pb.upload(st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
      std::vector<PertItem> items(m);
      for (int i = 0; i < m; ++i) {
        PertItem& it = items[i];
        it.dA0 = T(kA0, i); it.dB0 = T(kB0, i); it.dA2 = T(kA2, i); it.dB2 = T(kB2, i);
        it.gam = refs[iv[i].ref].gam;
        it.L = (iv[i].zb - iv[i].za) / k0;
        cplx* S = Sblk + 4 * nn * i;
        it.rud = S; it.rdu = S + nn; it.tdd = S + 2 * nn; it.tuu = S + 3 * nn;
        it.err = (unsigned long long*)derr.p + i;
      }
      cudaError_t err = cudaSuccess;
      auto run = [&](cudaError_t x) { if (err == cudaSuccess) err = x; };
      auto mm = [&](size_t a, size_t b, size_t d) {
        GemmArgs g = gemm(n, m);
        g.lda = g.ldb = g.ldc = g.ldd = n;
        g.A = pb.cat(a); g.B = pb.cat(b); g.D = pb.at(d);
        run(zgemm_batched(g, st));
      };
      const cplx one = mkc(1, 0), mone = mkc(-1, 0);
      run(axpby_elems(pb.cat(Pa), pb.cat(Pr), pb.at(t[kD0]), one, mone, nn, m, st));   // P0 - Pr
      run(axpby_elems(pb.cat(Qa), pb.cat(Qr), pb.at(t[kE0]), one, mone, nn, m, st));   // Q0 - Qr
      run(axpby_elems(pb.cat(Pb), pb.cat(Pr), pb.at(t[kD2]), one, mone, nn, m, st));   // P1 - Pr
      run(axpby_elems(pb.cat(Qb), pb.cat(Qr), pb.at(t[kE2]), one, mone, nn, m, st));   // Q1 - Qr
      mm(t[kD0], Vr, t[kX0]);  mm(t[kE0], Wr, t[kY0]);
      mm(t[kD2], Vr, t[kX2]);  mm(t[kE2], Wr, t[kY2]);
      mm(iWr, t[kX0], t[kx0]); mm(iVr, t[kY0], t[ky0]);
      mm(iWr, t[kX2], t[kx2]); mm(iVr, t[kY2], t[ky2]);
      run(axpby_elems(pb.cat(t[kx0]), pb.cat(t[ky0]), pb.at(t[kA0]), one, one, nn, m, st));
      run(axpby_elems(pb.cat(t[kx0]), pb.cat(t[ky0]), pb.at(t[kB0]), one, mone, nn, m, st));
      run(axpby_elems(pb.cat(t[kx2]), pb.cat(t[ky2]), pb.at(t[kA2]), one, one, nn, m, st));
      run(axpby_elems(pb.cat(t[kx2]), pb.cat(t[ky2]), pb.at(t[kB2]), one, mone, nn, m, st));
      run(cudaMemsetAsync(derr.p, 0, sizeof(unsigned long long) * m, st));
      run(cudaMemcpyAsync(ditems.p, items.data(), sizeof(PertItem) * m, cudaMemcpyHostToDevice, st));
      {
        dim3 grid((unsigned)std::min<size_t>(256, (nn + 255) / 256), m);
        perturbation_kernel<<<grid, 256, 0, st>>>((const PertItem*)ditems.p, n);
        ++launch_counter();
        run(cudaGetLastError());
      }
      std::vector<unsigned long long> herr(m);
      if (err != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess ||
          cudaMemcpy(herr.data(), derr.p, sizeof(unsigned long long) * m, cudaMemcpyDeviceToHost) != cudaSuccess)
        return set_err(e, RCWA_ERR_CUDA, "perturbation kernels failed");
      for (int i = 0; i < m; ++i) {
        double ev;
        std::memcpy(&ev, &herr[i], sizeof(double));
        if (!std::isfinite(ev)) return set_err(e, RCWA_ERR_NONFINITE, "non-finite perturbation");
        const RedInterval& I = iv[i];
        if (ev <= pe) {
          if ((int)acc.size() >= max_intervals) return set_err(e, RCWA_ERR_NOCONV, "more intervals than allowed");
          acc.push_back({I.za, I.ref, Sblk + 4 * nn * i});
        } else {
          // thirds (:293-327): the middle one keeps the parent's modes
          const double zm0 = 2. / 3. * I.za + 1. / 3. * I.zb, zm1 = 1. / 3. * I.za + 2. / 3. * I.zb;
          split_z.insert(split_z.end(), {0.5 * (I.za + zm0), zm0, zm1, 0.5 * (zm1 + I.zb)});
          ref_z.insert(ref_z.end(), {0.5 * (I.za + zm0), 0.5 * (zm1 + I.zb)});
          next.push_back({I.za, zm0, I.a, {}, -1});      // samples and modes filled below
          next.push_back({zm0, zm1, {}, {}, I.ref});
          next.push_back({zm1, I.zb, {}, I.b, -1});
        }
      }
    }
    if (next.empty()) break;
    rc = fetch(split_z);
    if (rc != RCWA_OK) return rc;
    const int base = (int)refs.size();
    rc = make_refs(ref_z, true);
    if (rc != RCWA_OK) return rc;
    for (size_t j = 0; j < next.size(); j += 3) {
      RedInterval& c1 = next[j];
      RedInterval& c2 = next[j + 1];
      RedInterval& c3 = next[j + 2];
      c1.b = samples.at(c1.zb);
      c1.ref = base + (int)(2 * (j / 3));
      c2.a = samples.at(c2.za);
      c2.b = samples.at(c2.zb);
      c3.a = samples.at(c3.za);
      c3.ref = base + (int)(2 * (j / 3)) + 1;
    }
    pending = next;
  }
  // the accepted intervals from the top down (the reference's depth-first
  // order): each projected from the modes of the one above it (the top
  // modes for the first), then cascaded
  std::sort(acc.begin(), acc.end(), [](const Accepted& a, const Accepted& b) { return a.za < b.za; });
  const int na = (int)acc.size();
  SBank S(n, na);
  // statuses of the projection, cascade and bottom steps, one per accepted
  // interval (the cascade's star products report by interval)
  Buf dcstat(sizeof(int) * na);
  if (!S.buf.p || !dcstat.p || cudaMemsetAsync(dcstat.p, 0, sizeof(int) * na, st) != cudaSuccess)
    return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  int* cstat = (int*)dcstat.p;
  {
    std::vector<cplx*> src, dst;
    for (int i = 0; i < na; ++i)
      for (int k = 0; k < 4; ++k) { src.push_back(acc[i].S + nn * k); dst.push_back(S.at(k, i)); }
    PtrBlob pb;
    const size_t ps = pb.add_list(src), pd = pb.add_list(dst);
    if (!pb.upload(st) || zcopy_batched(pb.cat(ps), n, pb.at(pd), n, n, n, 4 * na, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return set_err(e, RCWA_ERR_CUDA, "copy failed");
  }
  {
    std::vector<cplx*> iW(na), iV(na), lW(na), lV(na);
    for (int i = 0; i < na; ++i) {
      iW[i] = refs[acc[i].ref].iW;
      iV[i] = refs[acc[i].ref].iV;
      lW[i] = i ? refs[acc[i - 1].ref].W : top.W;
      lV[i] = i ? refs[acc[i - 1].ref].V : top.V;
    }
    rc = project_items(e, n, iW, iV, lW, lV, S, cstat, st);
    if (rc == RCWA_OK) rc = cascade_tree(e, n, na, S, cstat, st);
    if (rc != RCWA_OK) return rc;
  }
  // the bottom into the modes at z1 (:235-245): F = iW_last W1,
  // G = iV_last V1, A, B; M = A - Rud B; Tuu <- M^-1 Tuu;
  // Rud <- M^-1 (Rud A - B); Rdu <- Rdu + Tdd B Tuu; Tdd <- Tdd (B Rud + A)
  {
    const RedRef& last = refs[acc.back().ref];
    enum { kF, kG, kA, kB, kM, kX1, kT, kCnt };
    Buf dx(sizeof(cplx) * nn * kCnt), dpiv(sizeof(int) * n), dinf(sizeof(int));
    if (!dx.p || !dpiv.p || !dinf.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
    PtrBlob pb;
    auto one = [&](cplx* q) { return pb.add_list({q}); };
    auto X = [&](int k) { return one(dx.c() + nn * k); };
    const size_t pF = X(kF), pG = X(kG), pA = X(kA), pB = X(kB), pM = X(kM), pX1 = X(kX1), pT = X(kT);
    const size_t piW = one(last.iW), piV = one(last.iV), pW1 = one(bottom.W), pV1 = one(bottom.V);
    const size_t pRud = one(S.at(0, 0)), pRdu = one(S.at(1, 0)), pTdd = one(S.at(2, 0)), pTuu = one(S.at(3, 0));
    const size_t pI = pb.add_ints({0, 0});
    if (!pb.upload(st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
    cudaError_t err = cudaSuccess;
    auto run = [&](cudaError_t x) { if (err == cudaSuccess) err = x; };
    auto mm = [&](size_t a, size_t b, size_t d, double alpha, long c, double beta) {
      GemmArgs g = gemm(n, 1);
      g.lda = g.ldb = g.ldc = g.ldd = n;
      g.A = pb.cat(a); g.B = pb.cat(b); g.D = pb.at(d);
      g.alpha = mkc(alpha, 0);
      if (c >= 0) { g.C = pb.cat((size_t)c); g.beta = mkc(beta, 0); }
      run(zgemm_batched(g, st));
    };
    mm(piW, pW1, pF, 1.0, -1, 0.0);
    mm(piV, pV1, pG, 1.0, -1, 0.0);
    run(axpby_elems(pb.cat(pF), pb.cat(pG), pb.at(pA), mkc(0.5, 0), mkc(0.5, 0), nn, 1, st));
    run(axpby_elems(pb.cat(pF), pb.cat(pG), pb.at(pB), mkc(0.5, 0), mkc(-0.5, 0), nn, 1, st));
    mm(pRud, pB, pM, -1.0, (long)pA, 1.0);     // M = A - Rud B
    mm(pRud, pA, pX1, 1.0, (long)pB, -1.0);    // X1 = Rud A - B
    run(zgetrf_batched(pb.at(pM), n, n, (int*)dpiv.p, (int*)dinf.p, 1, st));
    run(fold_info((int*)dinf.p, pb.ints(pI), 1, RCWA_ERR_SINGULAR, cstat, st));
    run(zgetrs_batched(pb.cat(pM), n, n, (int*)dpiv.p, pb.at(pTuu), n, n, 1, st));  // Tuu'
    run(zgetrs_batched(pb.cat(pM), n, n, (int*)dpiv.p, pb.at(pX1), n, n, 1, st));   // Rud'
    mm(pB, pTuu, pT, 1.0, -1, 0.0);                  // T = B Tuu'
    mm(pTdd, pT, pRdu, 1.0, (long)pRdu, 1.0);        // Rdu' = Rdu + Tdd T
    mm(pB, pX1, pT, 1.0, (long)pA, 1.0);             // T = B Rud' + A
    mm(pTdd, pT, pM, 1.0, -1, 0.0);                  // Tdd'
    if (err != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
      return set_err(e, RCWA_ERR_CUDA, "integrator kernels failed");
    std::vector<int> hs(na + 1);
    if (cudaMemcpy(hs.data(), stat, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(hs.data() + 1, cstat, sizeof(int) * na, cudaMemcpyDeviceToHost) != cudaSuccess)
      return set_err(e, RCWA_ERR_CUDA, "download failed");
    for (int v : hs)
      if (v != RCWA_OK) return set_err(e, v, "singular matrix in the integrator");
    const size_t mb = sizeof(cplx) * nn;
    struct Out { rcwa_cplx* h; const void* d; } outs[] = {
        {Rud, dx.c() + nn * kX1}, {Rdu, S.at(1, 0)}, {Tdd, dx.c() + nn * kM}, {Tuu, S.at(3, 0)}};
    for (const Out& o : outs)
      if (o.h && cudaMemcpy(o.h, o.d, mb, cudaMemcpyDeviceToHost) != cudaSuccess)
        return set_err(e, RCWA_ERR_CUDA, "download failed");
  }
  rc = download_modes(e, n, top.W, top.V, top.gam, W0, V0, gam0);
  if (rc == RCWA_OK) rc = download_modes(e, n, bottom.W, bottom.V, bottom.gam, W1, V1, gam1);
  if (n_intervals) *n_intervals = na;
  if (n_eig) *n_eig = n_eig_solves;
  return rc;
}
