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

}  // namespace

extern "C" int rcwa_rcwa_integrate(rcwa_engine* e, int n, int nslab, double lambda, double z0, double z1,
                                   const rcwa_cplx* P, const rcwa_cplx* Q, rcwa_cplx* Rud, rcwa_cplx* Rdu,
                                   rcwa_cplx* Tdd, rcwa_cplx* Tuu, rcwa_cplx* W0, rcwa_cplx* V0, rcwa_cplx* gam0,
                                   rcwa_cplx* W1, rcwa_cplx* V1, rcwa_cplx* gam1) {
  if (!e || n < 1 || nslab < 0 || !P || !Q) return RCWA_ERR_INVALID;
  if (!(lambda > 0.0) || !std::isfinite(lambda) || !std::isfinite(z0) || !std::isfinite(z1))
    return set_err(e, RCWA_ERR_INVALID, "lambda must be positive and z0, z1 finite");
  if (cudaSetDevice(e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  const int ns = nslab + 2;  // samples: z0, the slab midpoints, z1
  const size_t nn = (size_t)n * n;
  cudaStream_t st = e->stream;
  Buf dP(sizeof(cplx) * nn * ns), dQ(sizeof(cplx) * nn * ns), dA(sizeof(cplx) * nn * ns),
      dW(sizeof(cplx) * nn * ns), dV(sizeof(cplx) * nn * ns), dw(sizeof(cplx) * n * ns), dk(sizeof(cplx) * n * ns),
      dwork(zgeev_workspace_bytes(n) * ns), dinfo(sizeof(int) * ns), dstat(sizeof(int) * (nslab + 1));
  if (!dP.p || !dQ.p || !dA.p || !dW.p || !dV.p || !dw.p || !dk.p || !dwork.p || !dinfo.p || !dstat.p)
    return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  if (!up(dP.c(), P, nn * ns, st) || !up(dQ.c(), Q, nn * ns, st) ||
      cudaMemsetAsync(dstat.p, 0, sizeof(int) * (nslab + 1), st) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "upload failed");
  cudaError_t err = cudaSuccess;
  auto run = [&](cudaError_t x) { if (err == cudaSuccess) err = x; };
  // modes of every sample: W, keff, V = Q W keff^-1 (rcwa/WaveEquationSolver.cpp:24-37)
  {
    PtrBlob pb;
    const size_t pP = pb.add(dP.c(), nn, 0, ns), pQ = pb.add(dQ.c(), nn, 0, ns), pA = pb.add(dA.c(), nn, 0, ns);
    const size_t pW = pb.add(dW.c(), nn, 0, ns), pV = pb.add(dV.c(), nn, 0, ns);
    if (!pb.upload(st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
    GemmArgs g = gemm(n, ns);
    g.lda = g.ldb = g.ldc = g.ldd = n;
    g.A = pb.cat(pP); g.B = pb.cat(pQ); g.D = pb.at(pA);
    run(zgemm_batched(g, st));
    run(zgeev_batched(pb.at(pA), n, n, dw.c(), pb.at(pW), n, dwork.p, (int*)dinfo.p, ns, st));
    g.A = pb.cat(pQ); g.B = pb.cat(pW); g.D = pb.at(pV);
    run(zgemm_batched(g, st));
    dim3 grid((unsigned)std::min<size_t>(1024, (nn + 255) / 256), ns);
    integrator_modes_kernel<<<grid, 256, 0, st>>>(dw.c(), dk.c(), dV.c(), n);
    ++launch_counter();
    run(cudaGetLastError());
    if (err != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
      return set_err(e, RCWA_ERR_CUDA, "integrator mode kernels failed");
  }
  std::vector<int> hinfo(ns);
  if (cudaMemcpy(hinfo.data(), dinfo.p, sizeof(int) * ns, cudaMemcpyDeviceToHost) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "download failed");
  for (int k = 0; k < ns; ++k)
    if (hinfo[k] != 0) return set_err(e, hinfo[k], "eigensolver failed on a sample");
  cplx* Wt = dW.c();                     // modes at z0
  cplx* Vt = dV.c();
  cplx* Wb = dW.c() + nn * (ns - 1);     // modes at z1, the slabs' reference medium
  cplx* Vb = dV.c() + nn * (ns - 1);
  // the running S-matrix of the whole region: 4 matrices per slab, cascaded
  // pairwise (the star product is associative) in ceil(log2 N) batched levels
  const int nS = std::max(nslab, 1);
  Buf dS(sizeof(cplx) * 4 * nn * nS);
  if (!dS.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  auto Sm = [&](int k, int i) { return dS.c() + nn * ((size_t)4 * i + k); };  // k: Rud, Rdu, Tdd, Tuu
  int* stat = (int*)dstat.p;
  if (nslab == 0) {
    // core/RCWAIntegrator.cpp:36-39: Tdd = Tuu = I, Rud = Rdu = 0
    PtrBlob pb;
    const size_t pR = pb.add_list({Sm(0, 0), Sm(1, 0)}), pT = pb.add_list({Sm(2, 0), Sm(3, 0)});
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
      const double dz = (z1 - z0) / nslab;
      std::vector<double> ss(nslab, lambda / (2.0 * 3.14159265358979323846) * dz);
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
        for (int k = 0; k < 4; ++k) d[k].push_back(Sm(k, i));
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
    // the cascade from the top down (:41-68): S_1 * S_2 * ... * S_N
    std::vector<int> list(nslab);
    for (int i = 0; i < nslab; ++i) list[i] = i;
    while (list.size() > 1) {
      std::vector<cplx*> upl[4], lol[4];
      std::vector<int> ids, next;
      for (size_t j = 0; j + 1 < list.size(); j += 2) {
        for (int k = 0; k < 4; ++k) {
          upl[k].push_back(Sm(k, list[j]));
          lol[k].push_back(Sm(k, list[j + 1]));
        }
        ids.push_back(list[j]);
        next.push_back(list[j]);
      }
      if (list.size() % 2) next.push_back(list.back());
      const int rc = star_core(e, n, (int)ids.size(), upl, lol, stat, ids, st);
      if (rc != RCWA_OK) return rc;
      list = next;
    }
  }
  // the modes at z0 on top (:70-85): A = (W1^-1 W0 + V1^-1 V0)/2,
  // B = (W1^-1 W0 - V1^-1 V0)/2, then
  //   Rdu <- (A - Rdu B)^-1 (Rdu A - B), Tdd <- (A - Rdu B)^-1 Tdd,
  //   Rud <- Tuu B Tdd + Rud, Tuu <- Tuu (B Rdu + A)  (new Tdd, Rdu)
  enum { kLW, kLV, kF, kG, kAm, kBm, kM, kX1, kX2, kT, kCnt };
  Buf dx(sizeof(cplx) * nn * kCnt), dpiv(sizeof(int) * 2 * n), dinf(sizeof(int) * 2);
  if (!dx.p || !dpiv.p || !dinf.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  auto X = [&](int k) { return dx.c() + nn * k; };
  cplx* SRud = Sm(0, 0);
  cplx* SRdu = Sm(1, 0);
  cplx* STdd = Sm(2, 0);
  cplx* STuu = Sm(3, 0);
  {
    PtrBlob pb;
    const size_t pLU = pb.add_list({X(kLW), X(kLV)});
    const size_t pFG = pb.add_list({X(kF), X(kG)});
    auto one = [&](cplx* q) { return pb.add_list({q}); };
    const size_t pF = one(X(kF)), pG = one(X(kG)), pAm = one(X(kAm)), pBm = one(X(kBm)), pM = one(X(kM));
    const size_t pX1 = one(X(kX1)), pX2 = one(X(kX2)), pT = one(X(kT));
    const size_t pRud = one(SRud), pRdu = one(SRdu), pTdd = one(STdd), pTuu = one(STuu);
    const size_t pI = pb.add_ints({0, 0});
    if (!pb.upload(st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
    int* piv = (int*)dpiv.p;
    int* inf = (int*)dinf.p;
    {
      // [LW, LV, F, G] <- [W1, V1, W0, V0]
      PtrBlob cp;
      const size_t s0 = cp.add_list({Wb, Vb, Wt, Vt}), d0 = cp.add_list({X(kLW), X(kLV), X(kF), X(kG)});
      if (!cp.upload(st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
      run(zcopy_batched(cp.cat(s0), n, cp.at(d0), n, n, n, 4, st));
      // F = W1^-1 W0, G = V1^-1 V0
      run(zgetrf_batched(pb.at(pLU), n, n, piv, inf, 2, st));
      run(fold_info(inf, pb.ints(pI), 2, RCWA_ERR_SINGULAR, stat, st));
      run(zgetrs_batched(pb.cat(pLU), n, n, piv, pb.at(pFG), n, n, 2, st));
      run(zaxpby_batched(pb.cat(pF), pb.cat(pG), pb.at(pAm), mkc(0.5, 0), mkc(0.5, 0), n, 1, st));
      run(zaxpby_batched(pb.cat(pF), pb.cat(pG), pb.at(pBm), mkc(0.5, 0), mkc(-0.5, 0), n, 1, st));
      auto mm = [&](size_t a, size_t b, size_t d, double alpha, long c, double beta) {
        GemmArgs g = gemm(n, 1);
        g.lda = g.ldb = g.ldc = g.ldd = n;
        g.A = pb.cat(a); g.B = pb.cat(b); g.D = pb.at(d);
        g.alpha = mkc(alpha, 0);
        if (c >= 0) { g.C = pb.cat((size_t)c); g.beta = mkc(beta, 0); }
        run(zgemm_batched(g, st));
      };
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
      std::vector<int> hs(nslab + 1);
      if (cudaMemcpy(hs.data(), stat, sizeof(int) * (nslab + 1), cudaMemcpyDeviceToHost) != cudaSuccess)
        return set_err(e, RCWA_ERR_CUDA, "download failed");
      for (int v : hs)
        if (v != RCWA_OK) return set_err(e, v, "singular matrix in the integrator");
      const size_t mb = sizeof(cplx) * nn, vb = sizeof(cplx) * n;
      struct Out { rcwa_cplx* h; const void* d; size_t bytes; } outs[] = {
          {Rud, SRud, mb}, {Rdu, X(kX1), mb}, {Tdd, X(kX2), mb}, {Tuu, X(kM), mb},
          {W0, Wt, mb}, {V0, Vt, mb}, {gam0, dk.c(), vb},
          {W1, Wb, mb}, {V1, Vb, mb}, {gam1, dk.c() + (size_t)n * (ns - 1), vb}};
      for (const Out& o : outs)
        if (o.h && cudaMemcpy(o.h, o.d, o.bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
          return set_err(e, RCWA_ERR_CUDA, "download failed");
    }
  }
  return RCWA_OK;
}
