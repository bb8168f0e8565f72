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
  // W, V are factorised in place; W0, V0 become F0, G0 in place
  Buf dWV(sizeof(cplx) * 2 * tot), dFG(sizeof(cplx) * 2 * tot), dg(sizeof(cplx) * n * batch),
      dA(sizeof(cplx) * tot), dR3(sizeof(cplx) * 3 * tot), dM(sizeof(cplx) * tot), dR2(sizeof(cplx) * 2 * tot),
      dpiv(sizeof(int) * 2 * n * batch), dinfo(sizeof(int) * 2 * batch), dstat(sizeof(int) * batch),
      ditems(sizeof(SlabRhsItem) * batch);
  if (!dWV.p || !dFG.p || !dg.p || !dA.p || !dR3.p || !dM.p || !dR2.p || !dpiv.p || !dinfo.p || !dstat.p ||
      !ditems.p)
    return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  cplx* Wd = dWV.c();
  cplx* Vd = Wd + tot;
  cplx* F0 = dFG.c();
  cplx* G0 = F0 + tot;
  cudaStream_t st = e->stream;
  if (!up(Wd, W, tot, st) || !up(Vd, V, tot, st) || !up(F0, W0, tot, st) || !up(G0, V0, tot, st) ||
      !up(dg.c(), gamma, n * batch, st) || cudaMemsetAsync(dstat.p, 0, sizeof(int) * batch, st) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "upload failed");
  std::vector<SlabRhsItem> items(batch);
  for (int b = 0; b < batch; ++b) {
    items[b].F0 = F0 + nn * b;
    items[b].G0 = G0 + nn * b;
    items[b].gamma = dg.c() + (size_t)n * b;
    items[b].ss = lambda[b] / (2.0 * 3.14159265358979323846) * wz[b];
    items[b].A = dA.c() + nn * b;
    items[b].R3 = dR3.c() + 3 * nn * b;
  }
  PtrBlob pb;
  const size_t pWV = pb.add(Wd, nn, 0, 2 * batch);     // W then V
  const size_t pFG = pb.add(F0, nn, 0, 2 * batch);     // W0 then V0
  const size_t pA = pb.add(dA.c(), nn, 0, batch);
  const size_t pR3 = pb.add(dR3.c(), 3 * nn, 0, batch);
  const size_t pR3a = pb.add(dR3.c(), 3 * nn, n, batch);      // invAXA block
  const size_t pR3b = pb.add(dR3.c(), 3 * nn, 2 * n, batch);  // invAXB block
  const size_t pM = pb.add(dM.c(), nn, 0, batch);
  const size_t pR2 = pb.add(dR2.c(), 2 * nn, 0, batch);
  const size_t pR2t = pb.add(dR2.c(), 2 * nn, n, batch);
  std::vector<int> item2(2 * batch), item1(batch);
  for (int b = 0; b < batch; ++b) item2[b] = item2[batch + b] = item1[b] = b;
  const size_t pI2 = pb.add_ints(item2), pI1 = pb.add_ints(item1);
  if (!pb.upload(st) ||
      cudaMemcpyAsync(ditems.p, items.data(), sizeof(SlabRhsItem) * batch, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "upload failed");
  int* piv = (int*)dpiv.p;
  int* info = (int*)dinfo.p;
  int* stat = (int*)dstat.p;
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
  const size_t row = sizeof(cplx) * n;
  if (cudaMemcpy2D(Rud, row, dR2.c(), 2 * row, row, (size_t)n * batch, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy2D(Tuu, row, dR2.c() + n, 2 * row, row, (size_t)n * batch, cudaMemcpyDeviceToHost) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "download failed");
  return finish_status(e, stat, batch, status);
}

extern "C" int rcwa_star_product_batched(rcwa_engine* e, int n, int batch, rcwa_cplx* Rud, rcwa_cplx* Rdu,
                                         rcwa_cplx* Tdd, rcwa_cplx* Tuu, const rcwa_cplx* rud, const rcwa_cplx* rdu,
                                         const rcwa_cplx* tdd, const rcwa_cplx* tuu, int* status) {
  if (!e || n < 1 || batch < 1 || !Rud || !Rdu || !Tdd || !Tuu || !rud || !rdu || !tdd || !tuu)
    return RCWA_ERR_INVALID;
  if (cudaSetDevice(e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  const size_t nn = (size_t)n * n, tot = nn * batch;
  // 8 operands, then scratch: T0 (factorised), C1, K1, C2, T1, T2, T3, Tuu'
  enum { kRud, kRdu, kTdd, kTuu, krud, krdu, ktdd, ktuu, kT0, kC1, kK1, kC2, kT1, kT2, kT3, kTn, kCount };
  Buf dm(sizeof(cplx) * tot * kCount), dpiv(sizeof(int) * n * batch), dinfo(sizeof(int) * batch),
      dstat(sizeof(int) * batch);
  if (!dm.p || !dpiv.p || !dinfo.p || !dstat.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  auto M = [&](int k) { return dm.c() + tot * k; };
  cudaStream_t st = e->stream;
  const rcwa_cplx* in[8] = {Rud, Rdu, Tdd, Tuu, rud, rdu, tdd, tuu};
  for (int k = 0; k < 8; ++k)
    if (!up(M(k), in[k], tot, st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
  if (cudaMemsetAsync(dstat.p, 0, sizeof(int) * batch, st) != cudaSuccess) return RCWA_ERR_CUDA;
  PtrBlob pb;
  size_t slot[kCount];
  for (int k = 0; k < kCount; ++k) slot[k] = pb.add(M(k), nn, 0, batch);
  std::vector<int> item1(batch);
  for (int b = 0; b < batch; ++b) item1[b] = b;
  const size_t pI1 = pb.add_ints(item1);
  if (!pb.upload(st)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
  int* piv = (int*)dpiv.p;
  int* info = (int*)dinfo.p;
  int* stat = (int*)dstat.p;
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
  if (err != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "star product kernels failed");
  rcwa_cplx* out[4] = {Rud, Rdu, Tdd, Tuu};
  const int src[4] = {kRud, kRdu, kTdd, kTn};
  for (int k = 0; k < 4; ++k)
    if (cudaMemcpy(out[k], M(src[k]), sizeof(cplx) * tot, cudaMemcpyDeviceToHost) != cudaSuccess)
      return set_err(e, RCWA_ERR_CUDA, "download failed");
  return finish_status(e, stat, batch, status);
}
