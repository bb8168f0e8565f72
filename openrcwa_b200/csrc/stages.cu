// Stage entry points of the C ABI: single-call device versions of the
// reference's FourierSolver1D/2D, Layer::solve and the zgeev wrapper, with
// host buffers in and out.  They run the same kernels as the batched solve.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "eig.cuh"
#include "engine_internal.cuh"
#include "fourier.cuh"
#include "gemm_tc.cuh"
#include "linalg.cuh"
#include "rcwa_kernels.cuh"


namespace {

// RAII device allocation for the stage calls.
struct Dev {
  void* p = nullptr;
  explicit Dev(size_t bytes) {
    if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) p = nullptr;
  }
  ~Dev() { if (p) cudaFree(p); }
  template <class T> T* as() const { return (T*)p; }
};

int set_err(rcwa_engine* e, int code, const char* msg) {
  if (e) e->last_error = msg;
  return code;
}

bool ascending(const double* x, int n) {
  for (int i = 0; i + 1 < n; ++i)
    if (!(x[i + 1] >= x[i])) return false;
  return n >= 2 && x[n - 1] > x[0];
}

// A pageable host-to-device cudaMemcpy may return before its DMA lands, and the
// engine's stream does not wait for the legacy stream, so each upload waits
// for the legacy stream before kernels on the engine's stream read the data.
template <class T>
bool up(void* dst, const T* src, size_t count) {
  return cudaMemcpy(dst, src, sizeof(T) * count, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaStreamSynchronize(cudaStreamLegacy) == cudaSuccess;
}

// Convolution matrices of one layer into device buffers fe11/fe22/fe33 (N x N).
int conv_one(rcwa_engine* e, const double* cx, int ncx, const double* cy, int ncy, const rcwa_cplx* eps, int nx,
             int ny, cplx* fe11, cplx* fe22, cplx* fe33) {
  const size_t cells = (size_t)(ncx - 1) * (ncy - 1);
  const size_t tab = conv_table_elems(nx, ny, ncx, ncy);
  const int strips = std::max(ncx - 1, ncy - 1);
  Dev dcx(sizeof(double) * ncx), dcy(sizeof(double) * ncy), deps(sizeof(cplx) * cells), dtab(sizeof(cplx) * tab);
  Dev djob(sizeof(ConvJob)), dptr(sizeof(void*) * 4 * strips), dipiv(sizeof(int) * strips * std::max(nx, ny)),
      dinfo(sizeof(int) * strips);
  if (!dcx.p || !dcy.p || !deps.p || !dtab.p || !djob.p || !dptr.p || !dipiv.p || !dinfo.p)
    return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  std::vector<cplx> he(cells);
  for (size_t i = 0; i < cells; ++i) he[i] = mkc(eps[i].re, eps[i].im);
  if (!up(dcx.p, cx, ncx) || !up(dcy.p, cy, ncy) || !up(deps.p, he.data(), cells))
    return set_err(e, RCWA_ERR_CUDA, "upload failed");
  ConvJob J;
  J.cx = dcx.as<double>();
  J.cy = dcy.as<double>();
  J.eps = deps.as<cplx>();
  J.ncx = ncx;
  J.ncy = ncy;
  J.fe11 = fe11;
  J.fe22 = fe22;
  J.fe33 = fe33;
  J.tab = dtab.as<cplx>();
  if (!up(djob.p, &J, 1)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
  ConvLaunch L;
  L.jobs = djob.as<ConvJob>();
  L.njobs = 1;
  L.nx = nx;
  L.ny = ny;
  L.max_ncx = ncx;
  L.max_ncy = ncy;
  cplx** tp = dptr.as<cplx*>();
  L.tx_ptrs = tp;
  L.txinv_ptrs = tp + (ncy - 1);
  L.ty_ptrs = tp + 2 * (ncy - 1);
  L.tyinv_ptrs = tp + 2 * (ncy - 1) + (ncx - 1);
  L.ipiv = dipiv.as<int>();
  L.info = dinfo.as<int>();
  if (conv_matrices(L, e->stream) != cudaSuccess || cudaStreamSynchronize(e->stream) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "convolution kernels failed");
  return RCWA_OK;
}

}  // namespace

extern "C" int rcwa_fourier1d(rcwa_engine* e, const double* x, int nxe, double d, const rcwa_cplx* f, int M,
                              rcwa_cplx* Ff) {
  if (!e || !x || !f || !Ff || nxe < 2 || M < 1 || !(d > 0)) return RCWA_ERR_INVALID;
  if (cudaSetDevice(e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  Dev dx(sizeof(double) * nxe), df(sizeof(cplx) * (nxe - 1)), dF(sizeof(cplx) * M);
  if (!dx.p || !df.p || !dF.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  if (!up(dx.p, x, nxe) || !up(df.p, (const cplx*)f, nxe - 1)) return RCWA_ERR_CUDA;
  if (fourier1d_device(dx.as<double>(), nxe, d, df.as<cplx>(), M, dF.as<cplx>(), e->stream) != cudaSuccess ||
      cudaStreamSynchronize(e->stream) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "fourier1d kernel failed");
  return cudaMemcpy(Ff, dF.p, sizeof(cplx) * M, cudaMemcpyDeviceToHost) == cudaSuccess ? RCWA_OK : RCWA_ERR_CUDA;
}

extern "C" int rcwa_fourier2d(rcwa_engine* e, const double* cx, int ncx, const double* cy, int ncy,
                              const rcwa_cplx* f, int nx, int ny, int opt, rcwa_cplx* Ff) {
  if (!e || !cx || !cy || !f || !Ff || nx < 1 || ny < 1) return RCWA_ERR_INVALID;
  if (!ascending(cx, ncx) || !ascending(cy, ncy)) return set_err(e, RCWA_ERR_INVALID, "edges must ascend");
  if (opt < RCWA_CONTINUOUS_XY || opt > RCWA_DISCONTINUOUS_Y) return RCWA_ERR_INVALID;
  if (cudaSetDevice(e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  const size_t NN = (size_t)nx * ny * nx * ny;
  Dev out(sizeof(cplx) * NN);
  if (!out.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  cplx* o = out.as<cplx>();
  int rc = conv_one(e, cx, ncx, cy, ncy, f, nx, ny, opt == RCWA_DISCONTINUOUS_X ? o : nullptr,
                    opt == RCWA_DISCONTINUOUS_Y ? o : nullptr, opt == RCWA_CONTINUOUS_XY ? o : nullptr);
  if (rc) return rc;
  return cudaMemcpy(Ff, o, sizeof(cplx) * NN, cudaMemcpyDeviceToHost) == cudaSuccess ? RCWA_OK : RCWA_ERR_CUDA;
}

extern "C" int rcwa_layer_solve(rcwa_engine* e, const double* cx, int ncx, const double* cy, int ncy,
                                const rcwa_cplx* eps, int nx, int ny, const double* alpha, const double* beta,
                                double lambda, rcwa_cplx* W, rcwa_cplx* V, rcwa_cplx* gamma,
                                rcwa_cplx* eigenvalues) {
  if (!e || !cx || !cy || !eps || !alpha || !beta || nx < 1 || ny < 1 || !(lambda > 0)) return RCWA_ERR_INVALID;
  if (!ascending(cx, ncx) || !ascending(cy, ncy)) return set_err(e, RCWA_ERR_INVALID, "edges must ascend");
  if (cudaSetDevice(e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  const int N = nx * ny, n = 2 * N;
  const size_t NN = (size_t)N * N, nn = (size_t)n * n;
  Dev fe11(sizeof(cplx) * NN), fe22(sizeof(cplx) * NN), fe33(sizeof(cplx) * NN), Einv(sizeof(cplx) * NN),
      X1(sizeof(cplx) * NN), X2(sizeof(cplx) * NN), M(sizeof(cplx) * nn), Wd(sizeof(cplx) * nn),
      Vd(sizeof(cplx) * nn), mu(sizeof(cplx) * n), g(sizeof(cplx) * n), ab(sizeof(cplx) * n),
      work(zgeev_workspace_bytes(n)), ipiv(sizeof(int) * N), info(sizeof(int) * 2), ptrs(sizeof(void*) * 16),
      item(sizeof(LayerItem)), status(sizeof(int));
  if (!fe11.p || !fe22.p || !fe33.p || !Einv.p || !X1.p || !X2.p || !M.p || !Wd.p || !Vd.p || !mu.p || !g.p ||
      !ab.p || !work.p || !ipiv.p || !info.p || !ptrs.p || !item.p || !status.p)
    return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  int rc = conv_one(e, cx, ncx, cy, ncy, eps, nx, ny, fe11.as<cplx>(), fe22.as<cplx>(), fe33.as<cplx>());
  if (rc) return rc;
  std::vector<cplx> hab(n);
  for (int i = 0; i < N; ++i) { hab[i] = mkc(alpha[i], 0.0); hab[N + i] = mkc(beta[i], 0.0); }
  if (!up(ab.p, hab.data(), n)) return RCWA_ERR_CUDA;
  const double k0 = 2 * 3.1415926535897932 / lambda;
  // pointer table: [fe33] [Einv] [Einv Einv] [fe11 fe22] [ab ab+N] [X1 X2] [M] [W]
  //                [fe22 fe11] [Wb Wt] [Vt Vb]
  void* hp[16] = {fe33.p, Einv.p, Einv.p, Einv.p, fe11.p, fe22.p, ab.p, ab.as<cplx>() + N, X1.p, X2.p, M.p, Wd.p,
                  fe22.p, fe11.p, Wd.as<cplx>() + (size_t)N * n, Wd.p};
  void* hp2[2] = {Vd.p, Vd.as<cplx>() + (size_t)N * n};
  Dev ptr2(sizeof(void*) * 2);
  if (!ptr2.p || !up(ptrs.p, hp, 16) || !up(ptr2.p, hp2, 2)) return RCWA_ERR_CUDA;
  void** P = ptrs.as<void*>();
  LayerItem it;
  it.fe11 = fe11.as<cplx>();
  it.fe22 = fe22.as<cplx>();
  it.X1 = X1.as<cplx>();
  it.X2 = X2.as<cplx>();
  it.ab = ab.as<cplx>();
  it.M = M.as<cplx>();
  it.W = Wd.as<cplx>();
  it.V = Vd.as<cplx>();
  it.mu = mu.as<cplx>();
  it.gamma = g.as<cplx>();
  it.k0 = k0;
  it.point = 0;
  if (!up(item.p, &it, 1)) return RCWA_ERR_CUDA;
  cudaStream_t st = e->stream;
  cudaMemsetAsync(status.p, 0, sizeof(int), st);
  bool ok = zgetrf_batched((cplx* const*)&P[0], N, N, ipiv.as<int>(), info.as<int>(), 1, st) == cudaSuccess &&
            zset_identity_batched((cplx* const*)&P[1], N, N, 1, st) == cudaSuccess &&
            zgetrs_batched((const cplx* const*)&P[0], N, N, ipiv.as<int>(), (cplx* const*)&P[1], N, N, 1, st) ==
                cudaSuccess;
  GemmArgs ga{};
  ga.A = (const cplx* const*)&P[2];
  ga.B = (const cplx* const*)&P[4];
  ga.s = (const cplx* const*)&P[6];
  ga.D = (cplx* const*)&P[8];
  ga.M = N; ga.N = N; ga.K = N;
  ga.lda = N; ga.ldb = N; ga.ldc = N; ga.ldd = N;
  ga.alpha = mkc(1, 0); ga.beta = mkc(0, 0); ga.gammaI = mkc(0, 0);
  ga.batch = 2;
  ok = ok && zgemm_batched(ga, st) == cudaSuccess;
  ok = ok && assemble_m(item.as<LayerItem>(), 1, N, st) == cudaSuccess;
  ok = ok && zgeev_batched((cplx* const*)&P[10], n, n, mu.as<cplx>(), (cplx* const*)&P[11], n, work.p,
                           info.as<int>() + 1, 1, st) == cudaSuccess;
  GemmArgs gv{};
  gv.A = (const cplx* const*)&P[12];
  gv.B = (const cplx* const*)&P[14];
  gv.D = (cplx* const*)ptr2.p;
  gv.M = N; gv.N = n; gv.K = N;
  gv.lda = N; gv.ldb = n; gv.ldc = n; gv.ldd = n;
  gv.alpha = mkc(1, 0); gv.beta = mkc(0, 0); gv.gammaI = mkc(0, 0);
  gv.batch = 2;
  ok = ok && zgemm_batched(gv, st) == cudaSuccess;
  ok = ok && finish_modes(item.as<LayerItem>(), 1, N, status.as<int>(), st) == cudaSuccess;
  ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
  if (!ok) return set_err(e, RCWA_ERR_CUDA, "layer solve kernels failed");
  int hinfo[2], hstat = 0;
  cudaMemcpy(hinfo, info.p, sizeof(int) * 2, cudaMemcpyDeviceToHost);
  cudaMemcpy(&hstat, status.p, sizeof(int), cudaMemcpyDeviceToHost);
  if (W && cudaMemcpy(W, Wd.p, sizeof(cplx) * nn, cudaMemcpyDeviceToHost) != cudaSuccess) return RCWA_ERR_CUDA;
  if (V && cudaMemcpy(V, Vd.p, sizeof(cplx) * nn, cudaMemcpyDeviceToHost) != cudaSuccess) return RCWA_ERR_CUDA;
  if (gamma && cudaMemcpy(gamma, g.p, sizeof(cplx) * n, cudaMemcpyDeviceToHost) != cudaSuccess) return RCWA_ERR_CUDA;
  if (eigenvalues) {
    std::vector<cplx> hm(n);
    if (cudaMemcpy(hm.data(), mu.p, sizeof(cplx) * n, cudaMemcpyDeviceToHost) != cudaSuccess) return RCWA_ERR_CUDA;
    for (int i = 0; i < n; ++i) eigenvalues[i] = rcwa_cplx{hm[i].x * k0 * k0, hm[i].y * k0 * k0};
  }
  if (hinfo[0]) return set_err(e, RCWA_ERR_SINGULAR, "fe33 is singular");
  if (hinfo[1]) return set_err(e, hinfo[1], "eigensolver failed");
  return hstat;
}

extern "C" int rcwa_zgeev_batched(rcwa_engine* e, int n, int batch, const rcwa_cplx* A, rcwa_cplx* w,
                                  rcwa_cplx* VR, int* info) {
  if (!e || n < 1 || batch < 1 || !A || !w || !VR) return RCWA_ERR_INVALID;
  if (cudaSetDevice(e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  const size_t nn = (size_t)n * n;
  Dev dA(sizeof(cplx) * nn * batch), dV(sizeof(cplx) * nn * batch), dw(sizeof(cplx) * n * batch),
      dwork(zgeev_workspace_bytes(n) * batch), dinfo(sizeof(int) * batch), dpa(sizeof(void*) * batch),
      dpv(sizeof(void*) * batch);
  if (!dA.p || !dV.p || !dw.p || !dwork.p || !dinfo.p || !dpa.p || !dpv.p)
    return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  std::vector<void*> pa(batch), pv(batch);
  for (int b = 0; b < batch; ++b) {
    pa[b] = dA.as<cplx>() + nn * b;
    pv[b] = dV.as<cplx>() + nn * b;
  }
  if (!up(dA.p, (const cplx*)A, nn * batch) || !up(dpa.p, pa.data(), batch) || !up(dpv.p, pv.data(), batch))
    return RCWA_ERR_CUDA;
  if (zgeev_batched(dpa.as<cplx*>(), n, n, dw.as<cplx>(), dpv.as<cplx*>(), n, dwork.p, dinfo.as<int>(), batch,
                    e->stream) != cudaSuccess ||
      cudaStreamSynchronize(e->stream) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "eigensolver kernel failed");
  std::vector<int> hinfo(batch);
  if (cudaMemcpy(w, dw.p, sizeof(cplx) * n * batch, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(VR, dV.p, sizeof(cplx) * nn * batch, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(hinfo.data(), dinfo.p, sizeof(int) * batch, cudaMemcpyDeviceToHost) != cudaSuccess)
    return RCWA_ERR_CUDA;
  int first = 0;
  for (int b = 0; b < batch; ++b) {
    if (info) info[b] = hinfo[b];
    if (!first && hinfo[b]) first = hinfo[b];
  }
  return first;
}

extern "C" int rcwa_zgemm_batched(rcwa_engine* e, int M, int N, int K, int batch, const rcwa_cplx* A,
                                  const rcwa_cplx* B, const rcwa_cplx* C, rcwa_cplx alpha, rcwa_cplx beta,
                                  int precision, rcwa_cplx* D) {
  if (!e || M < 1 || N < 1 || K < 1 || batch < 1 || !A || !B || !D) return RCWA_ERR_INVALID;
  if ((beta.re != 0.0 || beta.im != 0.0) && !C) return RCWA_ERR_INVALID;
  if (precision != RCWA_PREC_FP64 && precision != RCWA_PREC_MIXED) return RCWA_ERR_INVALID;
  if (cudaSetDevice(e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  const size_t mk = (size_t)M * K, kn = (size_t)K * N, mn = (size_t)M * N;
  Dev dA(sizeof(cplx) * mk * batch), dB(sizeof(cplx) * kn * batch), dC(sizeof(cplx) * mn * batch),
      dD(sizeof(cplx) * mn * batch), dp(sizeof(void*) * 2 * batch), derr(sizeof(int)),
      dscale(sizeof(int) * 2 * batch);
  if (!dA.p || !dB.p || !dC.p || !dD.p || !dp.p || !derr.p || !dscale.p)
    return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  const bool useC = beta.re != 0.0 || beta.im != 0.0;
  if (!up(dA.p, (const cplx*)A, mk * batch) || !up(dB.p, (const cplx*)B, kn * batch) ||
      (useC && !up(dC.p, (const cplx*)C, mn * batch)))
    return set_err(e, RCWA_ERR_CUDA, "upload failed");
  std::vector<void*> hp(2 * batch);
  for (int b = 0; b < batch; ++b) {
    hp[b] = dC.as<cplx>() + mn * b;
    hp[batch + b] = dD.as<cplx>() + mn * b;
  }
  const int zero = 0;
  if (!up(dp.p, hp.data(), 2 * batch) || !up(derr.p, &zero, 1)) return set_err(e, RCWA_ERR_CUDA, "upload failed");
  GemmArgs g{};
  g.A0 = dA.as<cplx>(); g.sA = mk;
  g.B0 = dB.as<cplx>(); g.sB = kn;
  g.C = useC ? (const cplx* const*)dp.p : nullptr;
  g.D = (cplx* const*)dp.p + batch;
  g.M = M; g.N = N; g.K = K;
  g.lda = K; g.ldb = N; g.ldc = N; g.ldd = N;
  g.alpha = mkc(alpha.re, alpha.im);
  g.beta = mkc(beta.re, beta.im);
  g.gammaI = mkc(0.0, 0.0);
  g.batch = batch;
  const size_t pbytes = precision == RCWA_PREC_MIXED ? zgemm_tf32x3_planes_bytes(M, N, K, batch) : 0;
  Dev dplanes(pbytes);
  if (!dplanes.p) return set_err(e, RCWA_ERR_NOMEM, "allocation failed");
  cudaError_t err = precision == RCWA_PREC_MIXED
                        ? zgemm_tf32x3_batched(g, dscale.as<int>(), derr.as<int>(), e->stream, 128,
                                               dplanes.as<float>(), pbytes)
                        : zgemm_batched(g, e->stream);
  if (err != cudaSuccess || cudaStreamSynchronize(e->stream) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "GEMM kernel failed");
  int herr = 0;
  if (cudaMemcpy(&herr, derr.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(D, dD.p, sizeof(cplx) * mn * batch, cudaMemcpyDeviceToHost) != cudaSuccess)
    return set_err(e, RCWA_ERR_CUDA, "download failed");
  if (herr) return set_err(e, RCWA_ERR_CUDA, "tensor-core completion wait ran out");
  return RCWA_OK;
}
