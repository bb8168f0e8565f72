// Batched complex eigensolver, one CTA per matrix, FP64 throughout:
//   1. Householder reduction to upper Hessenberg form, Q accumulated backwards;
//   2. single-shift complex QR iteration (Wilkinson shifts, exceptional shifts
//      every 10 sweeps, Ahues-Tisseur deflation test) producing the Schur form
//      T with Schur vectors Z.  The bulge is chased by one warp inside a
//      32 x 32 window held in shared memory; the window's rotations are then
//      applied to the rest of T and to Z by the whole CTA, each thread
//      streaming one row or column through the whole rotation sequence;
//   3. eigenvectors of T by back-substitution (protected small divisors),
//      back-transformed with Z by the tile GEMM and normalised to unit 2-norm.
// This replaces LAPACK zgeev('N','V') behind MKLEigenSolver
// (rcwa/MKLEigenSolver.hpp:102-179).  Balancing is not applied.
#include "eig.cuh"
#include "linalg.cuh"
#include "tile.cuh"

namespace {

constexpr int kEigThreads = kTileThreads;  // 256
constexpr int kWin = 32;
constexpr int kItsPerEig = 300;

__host__ __device__ inline size_t workspace_bytes(int n) {
  const size_t nn = (size_t)n * n;
  size_t bytes = (2 * nn + 4 * (size_t)n) * sizeof(cplx) + (size_t)n * sizeof(double);
  return (bytes + 255) & ~(size_t)255;
}

struct Scratch {
  cplx* Z;     // n*n, column-major: Z(r, c) = Z[c*n + r]
  cplx* X;     // n*n, row-major upper-triangular eigenvector matrix of T
  cplx* v;     // n: current Householder vector
  cplx* wv;    // n
  cplx* uv;    // n
  cplx* v0;    // n: leading element of each stored reflector
  double* tau; // n
};

__device__ Scratch scratch_for(void* work, int n, int b) {
  const size_t nn = (size_t)n * n;
  char* base = (char*)work + (size_t)b * workspace_bytes(n);
  Scratch s;
  s.Z = (cplx*)base;
  s.X = s.Z + nn;
  s.v = s.X + nn;
  s.wv = s.v + n;
  s.uv = s.wv + n;
  s.v0 = s.uv + n;
  s.tau = (double*)(s.v0 + n);
  return s;
}

__device__ double block_sum(double v, double* red) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  return t;
}

__device__ cplx block_sum_c(cplx v, double* red) {
  const double re = block_sum(v.x, red);
  const double im = block_sum(v.y, red);
  return mkc(re, im);
}

__device__ int block_max_int(int v, int* red) {
  for (int off = 16; off > 0; off >>= 1) v = max(v, __shfl_down_sync(0xffffffffu, v, off));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  int t = red[0];
  for (int w = 1; w < (int)(blockDim.x >> 5); ++w) t = max(t, red[w]);
  return t;
}

__device__ __forceinline__ cplx& at(cplx* M, int ld, int r, int c) { return M[(size_t)r * ld + c]; }

// ---------------------------------------------------------------- Hessenberg
__device__ void hessenberg(cplx* A, int n, int lda, const Scratch& s, double* red) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  for (int k = 0; k + 2 < n; ++k) {
    double sig = 0.0;
    for (int i = k + 2 + tid; i < n; i += blockDim.x) sig += cnorm2(at(A, lda, i, k));
    sig = block_sum(sig, red);
    const cplx alpha = at(A, lda, k + 1, k);
    if (sig == 0.0) {
      if (tid == 0) { s.tau[k] = 0.0; s.v0[k] = mkc(1.0, 0.0); }
      __syncthreads();
      continue;
    }
    const double aa = cabs(alpha);
    const double xnorm = sqrt(aa * aa + sig);
    const cplx ph = aa > 0.0 ? cscale(alpha, 1.0 / aa) : mkc(1.0, 0.0);
    const cplx beta = cscale(ph, -xnorm);
    const cplx v0 = cscale(ph, aa + xnorm);
    const double tau = 2.0 / (cnorm2(v0) + sig);
    for (int i = k + 1 + tid; i < n; i += blockDim.x) s.v[i] = (i == k + 1) ? v0 : at(A, lda, i, k);
    __syncthreads();
    // w_j = sum_{i>k} conj(v_i) A(i,j), j > k   (thread per column)
    for (int j = k + 1 + tid; j < n; j += blockDim.x) {
      cplx acc = mkc(0.0, 0.0);
      for (int i = k + 1; i < n; ++i) acc = cfmaconj(s.v[i], at(A, lda, i, j), acc);
      s.wv[j] = acc;
    }
    // u_i = sum_{j>k} A(i,j) v_j, all rows   (warp per row)
    for (int i = wid; i < n; i += nw) {
      cplx acc = mkc(0.0, 0.0);
      for (int j = k + 1 + lane; j < n; j += 32) acc = cfma(at(A, lda, i, j), s.v[j], acc);
      for (int off = 16; off > 0; off >>= 1) {
        acc.x += __shfl_down_sync(0xffffffffu, acc.x, off);
        acc.y += __shfl_down_sync(0xffffffffu, acc.y, off);
      }
      if (lane == 0) s.uv[i] = acc;
    }
    __syncthreads();
    cplx wdotv = mkc(0.0, 0.0);
    for (int j = k + 1 + tid; j < n; j += blockDim.x) wdotv = cfma(s.wv[j], s.v[j], wdotv);
    wdotv = block_sum_c(wdotv, red);
    // A <- H A H, H = I - tau v v^H (rows/cols > k), column k handled below
    const int ncol = n - k - 1;
    for (size_t idx = tid; idx < (size_t)n * ncol; idx += blockDim.x) {
      const int i = (int)(idx / ncol), j = k + 1 + (int)(idx % ncol);
      cplx u = s.uv[i];
      cplx a = at(A, lda, i, j);
      if (i > k) {
        u = cfma(cscale(s.v[i], -tau), wdotv, u);
        a = cfma(cscale(s.v[i], -tau), s.wv[j], a);
      }
      a = cfma(cscale(u, -tau), cconj(s.v[j]), a);
      at(A, lda, i, j) = a;
    }
    if (tid == 0) {
      at(A, lda, k + 1, k) = beta;  // rows k+2.. keep the reflector tail v_i = x_i
      s.tau[k] = tau;
      s.v0[k] = v0;
    }
    __syncthreads();
  }
  // Z = H_0 H_1 ... H_{n-3}, accumulated backwards (column-major Z)
  for (size_t idx = tid; idx < (size_t)n * n; idx += blockDim.x)
    s.Z[idx] = mkc((idx / n) == (idx % n) ? 1.0 : 0.0, 0.0);
  __syncthreads();
  for (int k = n - 3; k >= 0; --k) {
    const double tau = s.tau[k];
    if (tau == 0.0) continue;
    const cplx v0 = s.v0[k];
    for (int j = k + 1 + wid; j < n; j += nw) {
      cplx* zc = s.Z + (size_t)j * n;
      cplx d = mkc(0.0, 0.0);
      for (int i = k + 1 + lane; i < n; i += 32) {
        const cplx vi = (i == k + 1) ? v0 : at(A, lda, i, k);
        d = cfmaconj(vi, zc[i], d);
      }
      for (int off = 16; off > 0; off >>= 1) {
        d.x += __shfl_xor_sync(0xffffffffu, d.x, off);
        d.y += __shfl_xor_sync(0xffffffffu, d.y, off);
      }
      d = cscale(d, -tau);
      for (int i = k + 1 + lane; i < n; i += 32) {
        const cplx vi = (i == k + 1) ? v0 : at(A, lda, i, k);
        zc[i] = cfma(vi, d, zc[i]);
      }
    }
    __syncthreads();
  }
  for (size_t idx = tid; idx < (size_t)n * n; idx += blockDim.x) {
    const int i = (int)(idx / n), j = (int)(idx % n);
    if (i > j + 1) at(A, lda, i, j) = mkc(0.0, 0.0);
  }
  __syncthreads();
}

// ---------------------------------------------------------------- QR
__device__ __forceinline__ void givens(cplx x, cplx y, double& c, cplx& s) {
  const double ax = cabs(x), ay = cabs(y);
  if (ay == 0.0) { c = 1.0; s = mkc(0.0, 0.0); }
  else if (ax == 0.0) { c = 0.0; s = mkc(1.0, 0.0); }
  else {
    const double nrm = hypot(ax, ay);
    c = ax / nrm;
    s = cscale(cmul(cscale(x, 1.0 / ax), cconj(y)), 1.0 / nrm);
  }
}

// Negligible subdiagonal T(k,k-1) inside the active block [l, i]:
// the standard relative test refined by the criterion of Ahues and Tisseur
// (LAPACK Working Note 122, 1997).
__device__ bool negligible(const cplx* T, int ldt, int k, int l, int i, double ulp, double smlnum) {
  const cplx h = T[(size_t)k * ldt + k - 1];
  const double ah = cabs1(h);
  if (ah <= smlnum) return true;
  const cplx hkk = T[(size_t)k * ldt + k], hk1 = T[(size_t)(k - 1) * ldt + k - 1];
  double tst = cabs1(hk1) + cabs1(hkk);
  if (tst == 0.0) {
    if (k - 2 >= l) tst += cabs1(T[(size_t)(k - 1) * ldt + k - 2]);
    if (k + 1 <= i) tst += cabs1(T[(size_t)(k + 1) * ldt + k]);
  }
  if (ah <= ulp * tst) {
    const double up = cabs1(T[(size_t)(k - 1) * ldt + k]);
    const double ab = fmax(ah, up), ba = fmin(ah, up);
    const double d1 = cabs1(hkk), d2 = cabs1(csub(hk1, hkk));
    const double aa = fmax(d1, d2), bb = fmin(d1, d2);
    const double sc = aa + ab;
    if (ba * (ab / sc) <= fmax(smlnum, ulp * (bb * (aa / sc)))) return true;
  }
  return false;
}

// Eigenvalue of the trailing 2x2 [[a, b], [c, d]] closest to d:
// d - b*c / (delta + r), delta = (a - d)/2, r = sqrt(delta^2 + b*c) taken on
// the side of delta so that the denominator does not cancel.
__device__ cplx wilkinson_shift(cplx a, cplx b, cplx c, cplx d) {
  const cplx bc = cmul(b, c);
  const double sbc = cabs1(bc);
  if (sbc == 0.0) return d;
  const cplx delta = cscale(csub(a, d), 0.5);
  const double sc = fmax(cabs1(delta), sqrt(sbc));
  const cplx ds = cscale(delta, 1.0 / sc);
  cplx r = csqrt_principal(cadd(cmul(ds, ds), cscale(bc, 1.0 / (sc * sc))));
  r = cscale(r, sc);
  if (delta.x * r.x + delta.y * r.y < 0.0) r = cneg(r);
  const cplx den = cadd(delta, r);
  if (den.x == 0.0 && den.y == 0.0) return d;
  return csub(d, cdiv(bc, den));
}

__device__ void qr_sweep(cplx* T, int ldt, cplx* Z, int n, int l, int i, cplx shift,
                         cplx (*Wt)[kWin + 1], double* rc, cplx* rs) {
  const int tid = threadIdx.x;
  int k = l, ws = l;
  while (k <= i - 1) {
    const int we = min(ws + kWin - 1, i);
    const int ke = (we == i) ? i - 1 : we - 2;
    const int w = we - ws + 1;
    for (int idx = tid; idx < w * w; idx += blockDim.x)
      Wt[idx / w][idx % w] = T[(size_t)(ws + idx / w) * ldt + ws + idx % w];
    __syncthreads();
    if (tid < 32) {
      const int lane = tid;
      for (int r = k; r <= ke; ++r) {
        cplx x, y;
        if (r == l) {
          x = csub(Wt[r - ws][r - ws], shift);
          y = Wt[r + 1 - ws][r - ws];
        } else {
          x = Wt[r - ws][r - 1 - ws];
          y = Wt[r + 1 - ws][r - 1 - ws];
        }
        double c;
        cplx sn;
        givens(x, y, c, sn);
        const int j0 = (r == l) ? r : r - 1;
        const int jj = j0 - ws + lane;
        if (jj < w) {
          const cplx a = Wt[r - ws][jj], b = Wt[r + 1 - ws][jj];
          Wt[r - ws][jj] = cfma(sn, b, cscale(a, c));
          Wt[r + 1 - ws][jj] = cfma(cneg(cconj(sn)), a, cscale(b, c));
        }
        __syncwarp();
        if (lane == 0 && r > l) Wt[r + 1 - ws][r - 1 - ws] = mkc(0.0, 0.0);
        const int iend = min(r + 2, i) - ws;
        if (lane <= iend) {
          const cplx a = Wt[lane][r - ws], b = Wt[lane][r + 1 - ws];
          Wt[lane][r - ws] = cfma(cconj(sn), b, cscale(a, c));
          Wt[lane][r + 1 - ws] = cfma(cneg(sn), a, cscale(b, c));
        }
        __syncwarp();
        if (lane == 0) { rc[r - k] = c; rs[r - k] = sn; }
      }
    }
    __syncthreads();
    for (int idx = tid; idx < w * w; idx += blockDim.x)
      T[(size_t)(ws + idx / w) * ldt + ws + idx % w] = Wt[idx / w][idx % w];
    // deferred application of rotations k..ke outside the window
    const int nrot = ke - k + 1;
    const int nright = n - 1 - we;
    const int nup = ws;
    const int ntask = nright + nup + n;
    for (int t = tid; t < ntask; t += blockDim.x) {
      if (t < nright) {
        const int j = we + 1 + t;
        cplx x = T[(size_t)k * ldt + j];
        for (int q = 0; q < nrot; ++q) {
          const cplx y = T[(size_t)(k + q + 1) * ldt + j];
          const double c = rc[q];
          const cplx sn = rs[q];
          T[(size_t)(k + q) * ldt + j] = cfma(sn, y, cscale(x, c));
          x = cfma(cneg(cconj(sn)), x, cscale(y, c));
        }
        T[(size_t)(k + nrot) * ldt + j] = x;
      } else if (t < nright + nup) {
        const int ii = t - nright;
        cplx* row = T + (size_t)ii * ldt;
        cplx x = row[k];
        for (int q = 0; q < nrot; ++q) {
          const cplx y = row[k + q + 1];
          const double c = rc[q];
          const cplx sn = rs[q];
          row[k + q] = cfma(cconj(sn), y, cscale(x, c));
          x = cfma(cneg(sn), x, cscale(y, c));
        }
        row[k + nrot] = x;
      } else {
        const int ii = t - nright - nup;
        cplx x = Z[(size_t)k * n + ii];
        for (int q = 0; q < nrot; ++q) {
          const cplx y = Z[(size_t)(k + q + 1) * n + ii];
          const double c = rc[q];
          const cplx sn = rs[q];
          Z[(size_t)(k + q) * n + ii] = cfma(cconj(sn), y, cscale(x, c));
          x = cfma(cneg(sn), x, cscale(y, c));
        }
        Z[(size_t)(k + nrot) * n + ii] = x;
      }
    }
    __syncthreads();
    ws = ke;
    k = ke + 1;
  }
}

// Returns 0 or RCWA_ERR_NOCONV.
__device__ int schur(cplx* T, int ldt, cplx* Z, int n, cplx (*Wt)[kWin + 1], double* rc, cplx* rs,
                     int* redi) {
  const double ulp = 2.0 * RCWA_DBL_EPS;
  const double smlnum = RCWA_DBL_MIN * ((double)n / ulp);
  int i = n - 1;
  long long total = 0;
  const long long itmax_total = 30LL * max(10, n);
  while (i >= 0) {
    int l = 0;
    bool conv = false;
    for (int its = 0; its <= kItsPerEig; ++its) {
      int best = l;
      for (int k = l + 1 + threadIdx.x; k <= i; k += blockDim.x)
        if (negligible(T, ldt, k, l, i, ulp, smlnum)) best = max(best, k);
      l = block_max_int(best, redi);
      if (l > 0 && threadIdx.x == 0) T[(size_t)l * ldt + l - 1] = mkc(0.0, 0.0);
      __syncthreads();
      if (l >= i) { conv = true; break; }
      cplx shift;
      if (its == 10 || its == 30) {
        shift = cadd(T[(size_t)l * ldt + l], mkc(0.75 * cabs1(T[(size_t)(l + 1) * ldt + l]), 0.0));
      } else if (its == 20 || its == 40) {
        shift = cadd(T[(size_t)i * ldt + i], mkc(0.75 * cabs1(T[(size_t)i * ldt + i - 1]), 0.0));
      } else {
        shift = wilkinson_shift(T[(size_t)(i - 1) * ldt + i - 1], T[(size_t)(i - 1) * ldt + i],
                                T[(size_t)i * ldt + i - 1], T[(size_t)i * ldt + i]);
      }
      __syncthreads();
      qr_sweep(T, ldt, Z, n, l, i, shift, Wt, rc, rs);
      if (++total > itmax_total) break;
    }
    if (!conv) return RCWA_ERR_NOCONV;
    i = l - 1;
  }
  return 0;
}

// ---------------------------------------------------------------- eigenvectors
__device__ void trevc(const cplx* T, int ldt, cplx* X, int n) {
  const double ulp = 2.0 * RCWA_DBL_EPS;
  const double smlnum = RCWA_DBL_MIN * ((double)n / ulp);
  for (size_t idx = threadIdx.x; idx < (size_t)n * n; idx += blockDim.x) {
    const int i = (int)(idx / n), k = (int)(idx % n);
    if (i >= k) X[idx] = mkc(i == k ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  // column k of X is owned by thread k % blockDim.x for the whole sweep, so
  // its earlier entries are always the thread's own writes
  for (int i = n - 2; i >= 0; --i) {
    const cplx tii = T[(size_t)i * ldt + i];
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      if (k <= i) continue;
      cplx acc = T[(size_t)i * ldt + k];
      for (int j = i + 1; j < k; ++j) acc = cfma(T[(size_t)i * ldt + j], X[(size_t)j * n + k], acc);
      const cplx tkk = T[(size_t)k * ldt + k];
      const double smin = fmax(ulp * cabs1(tkk), smlnum);
      cplx d = csub(tii, tkk);
      if (cabs1(d) < smin) d = mkc(smin, 0.0);
      X[(size_t)i * n + k] = cneg(cdiv(acc, d));
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kEigThreads) hessenberg_kernel(cplx* const* Aarr, int n, int lda, void* work) {
  __shared__ double red[kEigThreads / 32];
  const Scratch s = scratch_for(work, n, blockIdx.x);
  hessenberg(Aarr[blockIdx.x], n, lda, s, red);
}

__global__ void __launch_bounds__(kEigThreads) schur_kernel(cplx* const* Aarr, int n, int lda, cplx* w_all,
                                                           void* work, int* info_all) {
  __shared__ cplx Wt[kWin][kWin + 1];
  __shared__ int redi[kEigThreads / 32];
  __shared__ double rc[kWin];
  __shared__ cplx rs[kWin];
  cplx* A = Aarr[blockIdx.x];
  const Scratch s = scratch_for(work, n, blockIdx.x);
  const int status = schur(A, lda, s.Z, n, Wt, rc, rs, redi);
  cplx* w = w_all + (size_t)blockIdx.x * n;
  for (int k = threadIdx.x; k < n; k += blockDim.x) w[k] = A[(size_t)k * lda + k];
  if (threadIdx.x == 0) info_all[blockIdx.x] = status;
}

__global__ void __launch_bounds__(kEigThreads) trevc_kernel(cplx* const* Aarr, int n, int lda, void* work) {
  const Scratch s = scratch_for(work, n, blockIdx.x);
  trevc(Aarr[blockIdx.x], lda, s.X, n);
}

// unit 2-norm columns; non-finite eigenpairs flag the matrix
__global__ void normalize_kernel(cplx* const* VRarr, int n, int ldv, const cplx* w_all, int* info_all) {
  cplx* VR = VRarr[blockIdx.y];
  const cplx* w = w_all + (size_t)blockIdx.y * n;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double ss = 0.0;
  for (int i = 0; i < n; ++i) ss += cnorm2(VR[(size_t)i * ldv + j]);
  const double sc = ss > 0.0 ? 1.0 / sqrt(ss) : 1.0;
  for (int i = 0; i < n; ++i) VR[(size_t)i * ldv + j] = cscale(VR[(size_t)i * ldv + j], sc);
  if (!isfinite(sc) || !isfinite(ss) || !isfinite(w[j].x) || !isfinite(w[j].y))
    atomicCAS(&info_all[blockIdx.y], 0, RCWA_ERR_NONFINITE);
}


}  // namespace

size_t zgeev_workspace_bytes(int n) { return workspace_bytes(n); }

cudaError_t zgeev_batched(cplx* const* A, int n, int lda, cplx* w, cplx* const* VR, int ldv, void* work,
                          int* info, int batch, cudaStream_t st, StageProf* prof) {
  if (batch <= 0 || n <= 0) return cudaSuccess;
  StageProf none;
  StageProf& P = prof ? *prof : none;
  hessenberg_kernel<<<batch, kEigThreads, 0, st>>>(A, n, lda, work);
  P.mark(st, kStHessenberg);
  schur_kernel<<<batch, kEigThreads, 0, st>>>(A, n, lda, w, work, info);
  P.mark(st, kStSchur);
  trevc_kernel<<<batch, kEigThreads, 0, st>>>(A, n, lda, work);
  P.mark(st, kStTrevc);
  // VR = Z X for every matrix (Z column-major == transposed operand)
  GemmArgs g{};
  g.A = nullptr;
  g.A0 = (const cplx*)work;
  g.sA = workspace_bytes(n) / sizeof(cplx);
  g.B = nullptr;
  g.B0 = (const cplx*)work + (size_t)n * n;
  g.sB = g.sA;
  g.D = VR;
  g.M = n; g.N = n; g.K = n;
  g.lda = n; g.ldb = n; g.ldd = ldv; g.ldc = ldv;
  g.transA = 1; g.transB = 0;
  g.alpha = mkc(1.0, 0.0); g.beta = mkc(0.0, 0.0); g.gammaI = mkc(0.0, 0.0);
  g.batch = batch;
  cudaError_t err = zgemm_batched(g, st);
  if (err != cudaSuccess) return err;
  P.mark(st, kStBackTransform);
  dim3 grid((n + 127) / 128, batch);
  normalize_kernel<<<grid, 128, 0, st>>>(VR, n, ldv, w, info);
  P.mark(st, kStNormalize);
  return cudaGetLastError();
}
