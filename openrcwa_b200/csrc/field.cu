// Fields inside a solved stack (see field.cuh).
//
// The mode amplitudes follow RCWASolver::evaluateIntermediateField
// (rcwa/RCWASolver.cpp:1505-1644): the interface matrices IE = Wa^-1 Wb,
// IH = Va^-1 Vb and the RTCM recursion Rud_{i+1} = I - 2 G tau_i are
// recomputed for the point, and the amplitudes are propagated top-down.  The
// reference forms each interface's scattering blocks from t11 = (IE + IH)/2,
// t12 = (IE - IH)/2 (S11 = t11 - t12 t11^-1 t12, S12 = t12 t11^-1,
// S21 = -t11^-1 t12, S22 = t11^-1) and solves with S11; here only vectors
// meet them, through S11^-1 = (IE^-1 + IH^-1)/2 (the Schur complement of
// [[t11, t12], [t12, t11]], whose halves IE and IH decouple) and
// S21 x + S22 y = t11^-1 (y - t12 x), so an interface costs three LU
// factorisations instead of explicit blocks.  The same amplitudes to
// rounding.
#include <cmath>

#include "field.cuh"
#include "linalg.cuh"

namespace {

constexpr double kPi = 3.1415926535897932;

__device__ __forceinline__ cplx cexp_i(double z, cplx g) {  // exp(i z g)
  const double m = exp(-z * g.y);
  double s, c;
  sincos(z * g.x, &s, &c);
  return mkc(m * c, m * s);
}

// out = a x + b y (vectors)
__global__ void vaxpby_kernel(cplx a, const cplx* x, cplx b, const cplx* y, cplx* out, int len) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x)
    out[i] = cfma(a, x[i], cmul(b, y[i]));
}

// out = ph A ph, ph = exp(i gamma d) (ones when d_is_zero): the waveRud of
// the recursion (rcwa/RCWASolver.cpp:423-433)
__global__ void sandwich_kernel(const cplx* A, const cplx* gamma, double d, int ones, cplx* out, int n) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)n * n; e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / n), c = (int)(e % n);
    out[e] = ones ? A[e] : cmul(cmul(cexp_i(d, gamma[r]), A[e]), cexp_i(d, gamma[c]));
  }
}

// d = exp(i gamma t) * c (the amplitudes carried through a layer)
__global__ void vphase_kernel(const cplx* c, const cplx* gamma, double t, cplx* out, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = cmul(cexp_i(t, gamma[i]), c[i]);
}

// column k of U (n x nz, row-major): c_p exp(i zp gamma) + sgn c_m exp(-i zm gamma)
__global__ void modes_at_z_kernel(const cplx* cp, const cplx* cm, const cplx* gamma, double zp, double zm, double sgn,
                                  cplx* U, int n, int nz, int k) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const cplx up = cmul(cp[i], cexp_i(zp, gamma[i]));
    const cplx dm = cmul(cm[i], cexp_i(-zm, gamma[i]));
    U[(size_t)i * nz + k] = mkc(up.x + sgn * dm.x, up.y + sgn * dm.y);
  }
}

// Hz = i/k0^2 (alpha Ey - beta Ex), or the right-hand side of Ez,
// alpha Hy - beta Hx (scale = 1): from [Fx; Fy] (2N x nz) into h (N x nz)
__global__ void curl_z_kernel(const cplx* F, const cplx* ab, int N, int nz, cplx scale, cplx* h) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)N * nz; e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / nz), k = (int)(e % nz);
    const cplx v = csub(cmul(ab[r], F[(size_t)(N + r) * nz + k]), cmul(ab[N + r], F[(size_t)r * nz + k]));
    h[e] = cmul(scale, v);
  }
}

// field[i][j] = sum over harmonics (m, q) of h[(m, q)][col] exp(i (kx_m x + ky_q y)),
// kx_m = 2 pi m / Lx + kx0, ky_q = 2 pi q / Ly + ky0, with (x, y, col) from
// the slice: XY (x = x0 + dx (j + 1/2), y = y0 + dy (i + 1/2), col 0), XZ
// (x from j, y = coord, col i), YZ (x = coord, y = y0 + dy (j + 1/2), col i)
__global__ void synth_kernel(const cplx* h, int nx, int ny, int ncol, int slice, double coord, double x0, double dx,
                             double y0, double dy, double Lx, double Ly, double kx0, double ky0, int nres1, int nres2,
                             cplx* field) {
  const int mx = (nx - 1) / 2, my = (ny - 1) / 2;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)nres1 * nres2;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e / nres1), j = (int)(e % nres1);
    double x, y;
    int col;
    if (slice == 0) { x = x0 + dx * (j + 0.5); y = y0 + dy * (i + 0.5); col = 0; }
    else if (slice == 1) { x = x0 + dx * (j + 0.5); y = coord; col = i; }
    else { x = coord; y = y0 + dx * (j + 0.5); col = i; }
    cplx acc = mkc(0.0, 0.0);
    for (int m = 0; m < nx; ++m) {
      const double px = (2.0 * kPi * (m - mx) / Lx + kx0) * x;
      for (int q = 0; q < ny; ++q) {
        const double ph = px + (2.0 * kPi * (q - my) / Ly + ky0) * y;
        double s, c;
        sincos(ph, &s, &c);
        acc = cfma(h[(size_t)(m * ny + q) * ncol + col], mkc(c, s), acc);
      }
    }
    field[e] = acc;
  }
}

dim3 grid_for(size_t elems) {
  size_t b = (elems + 255) / 256;
  if (b > 2048) b = 2048;
  if (b < 1) b = 1;
  return dim3((unsigned)b);
}

// device memory of one call, freed on every exit
struct Scratch {
  char* base = nullptr;
  size_t off = 0, cap = 0;
  ~Scratch() {
    if (base) cudaFree(base);
  }
  template <class T>
  T* take(size_t count) {
    const size_t bytes = (sizeof(T) * count + 255) & ~(size_t)255;
    T* p = reinterpret_cast<T*>(base + off);
    off += bytes;
    return p;
  }
};

}  // namespace

int field_rows(const FieldPoint& fp, int slice, int nres1) {
  double L1 = fp.Lx, L2 = 0.0;
  if (slice == 1 || slice == 2) {
    if (slice == 2) L1 = fp.Ly;
    for (int l = 1; l + 1 < fp.L; ++l) L2 += fp.thick[l];
  } else {
    L2 = fp.Ly;
  }
  const int r = (int)(nres1 * L2 / L1);
  return r < 1 ? 1 : r;
}

int field_slice(const FieldPoint& fp, cplx px, cplx py, int slice, double coord, int component, int nres1,
                cplx* out, cudaStream_t st) {
  const int N = fp.N, n = 2 * N, L = fp.L, nI = L - 2, ns = L - 1;
  if (nI < 1 || slice < 0 || slice > 2 || component < 0 || component > 5 || nres1 < 1) return RCWA_ERR_INVALID;
  const size_t nn = (size_t)n * n;
  const int nres2 = field_rows(fp, slice, nres1);
  const int nz = slice == 0 ? 1 : nres2;
  // depth samples and their interior layer (first layer whose span holds z)
  std::vector<double> zs(nz);
  std::vector<int> zl(nz, -1);
  std::vector<double> ztop(L, 0.0);
  {
    double z0 = 0.0;
    for (int l = 1; l + 1 < L; ++l) { ztop[l] = z0; z0 += fp.thick[l]; }
    const double L2 = z0;
    for (int k = 0; k < nz; ++k) {
      const double z = slice == 0 ? coord : (L2 / nres2) * (k + 0.5);
      zs[k] = z;
      for (int l = 1; l + 1 < L; ++l)
        if (ztop[l] <= z && z <= ztop[l] + fp.thick[l]) { zl[k] = l; break; }
      if (zl[k] < 0) return RCWA_ERR_INVALID;  // outside the interior layers
    }
  }
  Scratch S;
  // per step: IE, IH, LU(IE), LU(IH), LU(t11); per step REF; work F, G, tau, wRud, WLU, VLU;
  // vectors; harmonics U, Hm (n x nz) and h (N x nz); pointer pool
  const size_t mats = (size_t)ns * 5 + ns + 6;
  const size_t vecs = (size_t)2 * nI + nI + 16;
  const size_t bytes = mats * ((sizeof(cplx) * nn + 255) & ~(size_t)255) + vecs * ((sizeof(cplx) * n + 255) & ~(size_t)255) +
                       3 * ((sizeof(cplx) * n * nz + 255) & ~(size_t)255) +
                       ((sizeof(int) * n * (3 * ns + 3) + 255) & ~(size_t)255) + sizeof(int) * (3 * ns + 264) +
                       sizeof(void*) * 4096 +
                       ((sizeof(cplx) * (size_t)nres1 * nres2 + 255) & ~(size_t)255) + 4096;
  if (cudaMalloc(&S.base, bytes) != cudaSuccess) {
    cudaGetLastError();
    return RCWA_ERR_NOMEM;
  }
  S.cap = bytes;
  std::vector<cplx*> IE(ns), IH(ns), LIE(ns), LIH(ns), LT(ns), REF(ns);
  for (int i = 0; i < ns; ++i) {
    IE[i] = S.take<cplx>(nn); IH[i] = S.take<cplx>(nn);
    LIE[i] = S.take<cplx>(nn); LIH[i] = S.take<cplx>(nn); LT[i] = S.take<cplx>(nn);
    REF[i] = S.take<cplx>(nn);
  }
  cplx* F = S.take<cplx>(nn);
  cplx* G = S.take<cplx>(nn);
  cplx* tau = S.take<cplx>(nn);
  cplx* wR = S.take<cplx>(nn);
  cplx* WLU = S.take<cplx>(nn);
  cplx* VLU = S.take<cplx>(nn);
  std::vector<cplx*> cm(nI), cp(nI), dv(nI);
  for (int k = 0; k < nI; ++k) { cm[k] = S.take<cplx>(n); cp[k] = S.take<cplx>(n); dv[k] = S.take<cplx>(n); }
  cplx* inp = S.take<cplx>(n);
  cplx* Rv = S.take<cplx>(n);
  cplx* Tv = S.take<cplx>(n);
  cplx* v1 = S.take<cplx>(n);
  cplx* v2 = S.take<cplx>(n);
  cplx* v3 = S.take<cplx>(n);
  cplx* v4 = S.take<cplx>(n);
  cplx* U = S.take<cplx>((size_t)n * nz);
  cplx* Hm = S.take<cplx>((size_t)n * nz);
  cplx* h = S.take<cplx>((size_t)n * nz);
  int* ipiv = S.take<int>((size_t)n * (3 * ns + 3));
  int* info = S.take<int>((size_t)3 * ns + 8);
  cplx* dfield = S.take<cplx>((size_t)nres1 * nres2);
  void** pool = S.take<void*>(4096);
  std::vector<void*> hp;
  auto P = [&](std::initializer_list<const void*> ps) {
    const size_t o = hp.size();
    for (const void* q : ps) hp.push_back(const_cast<void*>(q));
    return (cplx* const*)(pool + o);
  };
  // all pointer arrays first (their device addresses are known), one upload
  std::vector<cplx* const*> pIEH(ns), pLT(ns);
  cplx* const* pLU0 = nullptr;
  cplx* const* pInp = nullptr;
  for (int i = 0; i < ns; ++i) {
    pIEH[i] = P({IE[i], IH[i]});
    pLT[i] = P({LT[i]});
  }
  // the interfaces' independent work as batches: copies of Wa, Va (into the
  // LIE, LIH buffers, free until the amplitude factors), Wb, Vb (into IE,
  // IH); LU of every Wa, Va; the solves; later the LU of every IE, IH, t11
  std::vector<const void*> csrc, cdst, luA, rhsA, luC;
  for (int i = 0; i < ns; ++i) {
    const int index = L - 1 - i, a = index - 1, b = index;
    csrc.insert(csrc.end(), {fp.W[a], fp.V[a], fp.W[b], fp.V[b]});
    cdst.insert(cdst.end(), {LIE[i], LIH[i], IE[i], IH[i]});
    luA.insert(luA.end(), {LIE[i], LIH[i]});
    rhsA.insert(rhsA.end(), {IE[i], IH[i]});
    luC.insert(luC.end(), {LIE[i], LIH[i], LT[i]});
  }
  auto Pv = [&](const std::vector<const void*>& v) {
    const size_t o = hp.size();
    for (const void* q : v) hp.push_back(const_cast<void*>(q));
    return (cplx* const*)(pool + o);
  };
  cplx* const* pCs = Pv(csrc);
  cplx* const* pCd = Pv(cdst);
  cplx* const* pLA = Pv(luA);
  cplx* const* pRA = Pv(rhsA);
  cplx* const* pLC = Pv(luC);
  cplx* const* pW = P({WLU});
  cplx* const* pF = P({F});
  cplx* const* pTauD = P({tau});
  pLU0 = P({WLU});
  pInp = P({inp});
  std::vector<cplx* const*> pv(ns * 6);
  for (int i = 0; i < ns; ++i) {
    pv[6 * i + 0] = P({LIE[i]});
    pv[6 * i + 1] = P({LIH[i]});
    pv[6 * i + 2] = P({v1});
    pv[6 * i + 3] = P({v2});
    pv[6 * i + 4] = P({v3});
    pv[6 * i + 5] = P({IE[i]});
  }
  cplx* const* pv1 = P({v1});
  cplx* const* pv2 = P({v2});
  cplx* const* pv3 = P({v3});
  cplx* const* pv4 = P({v4});
  if (hp.size() > 4096) return RCWA_ERR_INVALID;
  if (cudaMemcpyAsync(pool, hp.data(), sizeof(void*) * hp.size(), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return RCWA_ERR_CUDA;
  (void)pW; (void)pF; (void)pTauD; (void)pv;

  auto ok = [](cudaError_t e) { return e == cudaSuccess; };
  auto gemm = [&](const cplx* A, int lda, const cplx* B, int ldb, cplx* D, int ldd, int M, int Nc, int K, cplx alpha,
                  cplx gammaI) {
    GemmArgs g{};
    g.A0 = A; g.B0 = B; g.D0 = D;
    g.M = M; g.N = Nc; g.K = K;
    g.lda = lda; g.ldb = ldb; g.ldd = ldd; g.ldc = ldd;
    g.alpha = alpha; g.beta = mkc(0, 0); g.gammaI = gammaI;
    g.batch = 1;
    return zgemm_batched(g, st);
  };
  // F = C + alpha A B with C given as a pointer array (beta = 1)
  auto gemm_acc = [&](const cplx* A, const cplx* B, cplx* const* Cp, cplx* D, cplx alpha) {
    GemmArgs g{};
    g.A0 = A; g.B0 = B; g.D0 = D; g.C = (const cplx* const*)Cp;
    g.M = n; g.N = n; g.K = n;
    g.lda = n; g.ldb = n; g.ldd = n; g.ldc = n;
    g.alpha = alpha; g.beta = mkc(1, 0); g.gammaI = mkc(0, 0);
    g.batch = 1;
    return zgemm_batched(g, st);
  };
  auto vax = [&](cplx a, const cplx* x, cplx b, const cplx* y, cplx* o) {
    vaxpby_kernel<<<grid_for(n), 256, 0, st>>>(a, x, b, y, o, n);
    ++launch_counter();
    return cudaGetLastError();
  };
  auto copy = [&](const cplx* s, cplx* d) { return cudaMemcpyAsync(d, s, sizeof(cplx) * nn, cudaMemcpyDeviceToDevice, st); };
  const cplx one = mkc(1, 0), zero = mkc(0, 0), half = mkc(0.5, 0);
  cudaError_t e = cudaSuccess;
  int* ip_run = ipiv + (size_t)2 * n;         // n: LU of F + G, W_ref
  int* ip_st = ipiv + (size_t)3 * n;          // 3 n per step: IE, IH, t11 (first Wa, Va)
  // ---- interfaces IE = Wa^-1 Wb, IH = Va^-1 Vb of every step at once
  // (rcwa/RCWASolver.cpp:537-543)
  e = zcopy_batched((const cplx* const*)pCs, n, pCd, n, n, n, 4 * ns, st);
  if (ok(e)) e = zgetrf_batched(pLA, n, n, ip_st, info, 2 * ns, st);
  if (ok(e)) e = zgetrs_batched((const cplx* const*)pLA, n, n, ip_st, pRA, n, n, 2 * ns, st);
  // ---- the recursion, step by step
  for (int i = 0; i < ns && ok(e); ++i) {
    const int index = L - 1 - i, b = index;
    // waveRud, F = IE + IE waveRud, G = IH - IH waveRud, tau = (F + G)^-1,
    // Rud = I - 2 G tau  (:423-460)
    const cplx* Rprev = i == 0 ? nullptr : REF[i - 1];
    if (ok(e)) {
      if (Rprev) {
        sandwich_kernel<<<grid_for(nn), 256, 0, st>>>(Rprev, fp.gamma[b], fp.thick[b], 0, wR, n);
        ++launch_counter();
        e = cudaGetLastError();
      } else {
        e = cudaMemsetAsync(wR, 0, sizeof(cplx) * nn, st);
      }
    }
    if (ok(e)) e = gemm_acc(IE[i], wR, pIEH[i], F, one);
    if (ok(e)) e = gemm_acc(IH[i], wR, pIEH[i] + 1, G, mkc(-1, 0));
    if (ok(e)) {
      // S = F + G (into F), then its inverse into tau
      vaxpby_kernel<<<grid_for(nn), 256, 0, st>>>(one, F, one, G, F, (int)nn);
      ++launch_counter();
      e = cudaGetLastError();
    }
    if (ok(e)) e = zgetrf_batched(pF, n, n, ip_run, info, 1, st);
    if (ok(e)) e = zgetri_batched((const cplx* const*)pF, n, n, ip_run, pTauD, n, 1, st);
    if (ok(e)) e = gemm(G, n, tau, n, REF[i], n, n, n, n, mkc(-2, 0), one);
  }
  // ---- factors for the amplitudes, every step at once: LU of IE, IH and
  // t11 = (IE + IH)/2 (item 3i + k's pivots at ip_st + (3i + k) n)
  for (int i = 0; i < ns && ok(e); ++i) {
    if (ok(e)) e = copy(IE[i], LIE[i]);
    if (ok(e)) e = copy(IH[i], LIH[i]);
    if (ok(e)) {
      vaxpby_kernel<<<grid_for(nn), 256, 0, st>>>(half, IE[i], half, IH[i], LT[i], (int)nn);
      ++launch_counter();
      e = cudaGetLastError();
    }
  }
  if (ok(e)) e = zgetrf_batched(pLC, n, n, ip_st, info, 3 * ns, st);
  if (!ok(e)) return RCWA_ERR_CUDA;
  // ---- the input: modal amplitudes of the incidence layer for the plane
  // wave (px, py) (generateHorizontalPlaneWave, rcwa/Layer.cpp:453-480)
  const int inc = fp.ny * ((fp.nx - 1) / 2) + (fp.ny - 1) / 2;
  {
    std::vector<cplx> s((size_t)n, mkc(0, 0));
    s[inc] = px;
    s[N + inc] = py;
    if (!ok(cudaMemcpyAsync(inp, s.data(), sizeof(cplx) * n, cudaMemcpyHostToDevice, st))) return RCWA_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return RCWA_ERR_CUDA;
  }
  if (fp.pat0) {
    if (ok(e)) e = copy(fp.W[0], WLU);
    if (ok(e)) e = zgetrf_batched(pLU0, n, n, ip_run, info, 1, st);
    if (ok(e)) e = zgetrs_batched((const cplx* const*)pLU0, n, n, ip_run, pInp, 1, 1, 1, st);
  }
  // R = Rud inp, T = Tdd inp  (:1602-1607)
  if (ok(e)) e = gemm(fp.Rud, n, inp, 1, Rv, 1, n, 1, n, one, zero);
  if (ok(e)) e = gemm(fp.Tdd, n, inp, 1, Tv, 1, n, 1, n, one, zero);
  // t12 x = (IE x - IH x)/2 into o (o != x)
  auto t12 = [&](int i, const cplx* x, cplx* o) {
    cudaError_t r = gemm(IE[i], n, x, 1, o, 1, n, 1, n, half, zero);
    if (r == cudaSuccess) r = gemm(IH[i], n, x, 1, v4, 1, n, 1, n, half, zero);
    if (r == cudaSuccess) r = vax(one, o, mkc(-1, 0), v4, o);
    return r;
  };
  // one step of the top-down amplitudes: given x (c_m of the layer above or
  // R) and y (its forward amplitude, or the input) at interface step s:
  // temp = S11^-1 (x - t12 t11^-1 y), c_p = t11^-1 (y - t12 temp)
  auto amp_step = [&](int s, const cplx* x, const cplx* y, cplx* c_p_out) {
    const int* ipE = ip_st + (size_t)3 * n * s;
    cudaError_t r = cudaMemcpyAsync(v1, y, sizeof(cplx) * n, cudaMemcpyDeviceToDevice, st);
    if (r == cudaSuccess) r = zgetrs_batched((const cplx* const*)pLT[s], n, n, ipE + 2 * n, pv1, 1, 1, 1, st);
    if (r == cudaSuccess) r = t12(s, v1, v2);                       // v2 = t12 t11^-1 y
    if (r == cudaSuccess) r = vax(one, x, mkc(-1, 0), v2, v2);      // v2 = x - S12 y
    if (r == cudaSuccess) r = cudaMemcpyAsync(v3, v2, sizeof(cplx) * n, cudaMemcpyDeviceToDevice, st);
    if (r == cudaSuccess) r = zgetrs_batched((const cplx* const*)pv[6 * s + 0], n, n, ipE, pv2, 1, 1, 1, st);
    if (r == cudaSuccess) r = zgetrs_batched((const cplx* const*)pv[6 * s + 1], n, n, ipE + n, pv3, 1, 1, 1, st);
    if (r == cudaSuccess) r = vax(half, v2, half, v3, v1);          // v1 = temp
    if (r == cudaSuccess) r = t12(s, v1, v2);                       // v2 = t12 temp
    if (r == cudaSuccess) r = vax(one, y, mkc(-1, 0), v2, c_p_out); // y - t12 temp
    if (r == cudaSuccess) {
      r = cudaMemcpyAsync(v1, c_p_out, sizeof(cplx) * n, cudaMemcpyDeviceToDevice, st);
      if (r == cudaSuccess) r = zgetrs_batched((const cplx* const*)pLT[s], n, n, ipE + 2 * n, pv1, 1, 1, 1, st);
      if (r == cudaSuccess) r = cudaMemcpyAsync(c_p_out, v1, sizeof(cplx) * n, cudaMemcpyDeviceToDevice, st);
    }
    return r;
  };
  // c_m of the bottom interior layer = S12[0] t11_0 T = t12_0 T  (:1615)
  if (ok(e)) e = t12(0, Tv, cm[nI - 1]);
  // c_p of the top interior layer, from R and the input at the top interface
  if (ok(e)) e = amp_step(L - 2, Rv, inp, cp[0]);
  auto carry = [&](int k, int s, cplx* out) {  // d = phase of stack layer (L - 1 - s) * c_p[k]
    const int li = L - 1 - s;
    vphase_kernel<<<grid_for(n), 256, 0, st>>>(cp[k], fp.gamma[li], fp.thick[li], out, n);
    ++launch_counter();
    return cudaGetLastError();
  };
  if (ok(e)) e = carry(0, L - 2, dv[nI - 1]);
  for (int i = nI - 2; i >= 0 && ok(e); --i) {
    // c_m = REF[i + 2] d[i + 1]; the reference's REF[k] is Rud after k steps
    e = gemm(REF[i + 1], n, dv[i + 1], 1, cm[nI - i - 2], 1, n, 1, n, one, zero);
    if (ok(e)) e = amp_step(i + 1, cm[nI - i - 2], dv[i + 1], cp[nI - i - 1]);
    if (ok(e)) e = carry(nI - i - 1, i + 1, dv[i]);
  }
  if (!ok(e)) return RCWA_ERR_CUDA;
  // ---- harmonics of the component at every depth sample
  // (SET_HARMONICS_2D of rcwa/RCWASolver.cpp:785-900)
  const bool useH = component >= 3 && component <= 4;
  const bool fromH = useH || component == 2;  // Ez comes from H
  for (int k = 0; k < nz && ok(e); ++k) {
    const int l = zl[k], ki = l - 1;
    const double zp = zs[k] - ztop[l], zm = zs[k] - (ztop[l] + fp.thick[l]);
    modes_at_z_kernel<<<grid_for(n), 256, 0, st>>>(cp[ki], cm[ki], fp.gamma[l], zp, zm, fromH ? -1.0 : 1.0, U, n, nz, k);
    ++launch_counter();
    e = cudaGetLastError();
  }
  // [Fx; Fy] = W U (E) or V U (H), layer by layer over its depth samples
  for (int k0 = 0; k0 < nz && ok(e);) {
    int k1 = k0;
    while (k1 < nz && zl[k1] == zl[k0]) ++k1;
    const int l = zl[k0];
    e = gemm(fromH ? fp.V[l] : fp.W[l], n, U + k0, nz, Hm + k0, nz, n, k1 - k0, n, one, zero);
    k0 = k1;
  }
  if (!ok(e)) return RCWA_ERR_CUDA;
  const cplx* hsrc = nullptr;
  if (component == 0 || component == 3) hsrc = Hm;
  else if (component == 1 || component == 4) hsrc = Hm + (size_t)N * nz;
  else if (component == 5) {
    // Hz = i/k0^2 (kx Ey - ky Ex)  (:852-866)
    curl_z_kernel<<<grid_for((size_t)N * nz), 256, 0, st>>>(Hm, fp.ab, N, nz, mkc(0.0, 1.0 / (fp.k0 * fp.k0)), h);
    ++launch_counter();
    e = cudaGetLastError();
    hsrc = h;
  } else {
    // Ez = i [[eps]]^-1 (kx Hy - ky Hx)  (:867-885), layer by layer
    curl_z_kernel<<<grid_for((size_t)N * nz), 256, 0, st>>>(Hm, fp.ab, N, nz, mkc(0.0, 1.0), U);
    ++launch_counter();
    e = cudaGetLastError();
    for (int k0 = 0; k0 < nz && ok(e);) {
      int k1 = k0;
      while (k1 < nz && zl[k1] == zl[k0]) ++k1;
      e = gemm(fp.Einv[zl[k0]], N, U + k0, nz, h + k0, nz, N, k1 - k0, N, one, zero);
      k0 = k1;
    }
    hsrc = h;
  }
  if (!ok(e)) return RCWA_ERR_CUDA;
  // ---- Fourier synthesis on the slice (:905-1008)
  double x0 = fp.x0, dx = fp.Lx / nres1, y0 = fp.y0, dy = fp.Ly / nres2;
  if (slice == 2) dx = fp.Ly / nres1;
  synth_kernel<<<grid_for((size_t)nres1 * nres2), 256, 0, st>>>(hsrc, fp.nx, fp.ny, nz, slice, coord, x0, dx, y0, dy,
                                                               fp.Lx, fp.Ly, fp.kx0, fp.ky0, nres1, nres2, dfield);
  ++launch_counter();
  if (cudaGetLastError() != cudaSuccess) return RCWA_ERR_CUDA;
  if (cudaMemcpyAsync(out, dfield, sizeof(cplx) * nres1 * nres2, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return RCWA_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return RCWA_ERR_CUDA;
  return RCWA_OK;
}
