// RCWA-specific element-wise kernels and the efficiency reduction.
#include "rcwa_kernels.cuh"

namespace {

__device__ __forceinline__ void set_status(int* status, int point, int code) {
  if (status) atomicCAS(&status[point], 0, code);
}

// M = (P*Q)/k0^2 of Layer::waveEqnCoeff + WaveEquationSolver::solve
// (rcwa/Layer.cpp:150-220, rcwa/WaveEquationSolver.cpp:45), expanded with the
// diagonal Kx = diag(a), Ky = diag(b) and E = fe33^-1:
//   M11 = k0^2 fe11 - Db^2 - Da X1     M12 = Da Db - Da X2
//   M21 = Da Db - Db X1                M22 = k0^2 fe22 - Da^2 - Db X2
// with X1 = E Da fe11, X2 = E Db fe22 (the only O(N^3) products).
__global__ void assemble_m_kernel(const LayerItem* items, int N) {
  const LayerItem it = items[blockIdx.y];
  const int n = 2 * N;
  const double k02 = it.k0 * it.k0;
  const size_t total = (size_t)n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / n), c = (int)(e % n);
    const int rr = r % N, cc = c % N;
    const bool diag = (rr == cc);
    const cplx a = it.ab[rr], b = it.ab[N + rr];
    const size_t o = (size_t)rr * N + cc;
    cplx v;
    if (r < N && c < N) {
      v = cscale(it.fe11[o], k02);
      if (diag) v = csub(v, cmul(b, b));
      v = csub(v, cmul(a, it.X1[o]));
    } else if (r < N) {
      v = diag ? cmul(a, b) : mkc(0.0, 0.0);
      v = csub(v, cmul(a, it.X2[o]));
    } else if (c < N) {
      v = diag ? cmul(a, b) : mkc(0.0, 0.0);
      v = csub(v, cmul(b, it.X1[o]));
    } else {
      v = cscale(it.fe22[o], k02);
      if (diag) v = csub(v, cmul(a, a));
      v = csub(v, cmul(b, it.X2[o]));
    }
    it.M[e] = v;
  }
}

// gamma = GammaSqrtOp(mu) (keff = k0*gamma, rcwa/WaveEquationSolver.cpp:49,
// rcwa/Layer.cpp:269) and V = Q W diag(1/keff) (WaveEquationSolver.cpp:51):
//   (QW)_top = -Da Db Wt + Da^2 Wb - k0^2 fe22 Wb
//   (QW)_bot = -Db^2 Wt + Da Db Wb + k0^2 fe11 Wt
// The products fe22*Wb (top rows) and fe11*Wt (bottom rows) arrive in V from
// the GEMMs.
__global__ void finish_modes_kernel(const LayerItem* items, int N, int* status) {
  const LayerItem it = items[blockIdx.y];
  const int n = 2 * N;
  const size_t total = (size_t)n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / n), c = (int)(e % n);
    const int rr = r % N;
    const cplx g = gamma_sqrt(it.mu[c]);
    const cplx keff = cscale(g, it.k0);
    const cplx a = it.ab[rr], b = it.ab[N + rr];
    const cplx wt = it.W[(size_t)rr * n + c], wb = it.W[(size_t)(N + rr) * n + c];
    cplx q;
    const double k02 = it.k0 * it.k0;
    if (r < N) q = cadd(csub(cscale(it.V[e], -k02), cmul(cmul(a, b), wt)), cmul(cmul(a, a), wb));
    else q = cadd(csub(cscale(it.V[e], k02), cmul(cmul(b, b), wt)), cmul(cmul(a, b), wb));
    if (keff.x == 0.0 && keff.y == 0.0) {
      set_status(status, it.point, RCWA_ERR_GRAZING);
      it.V[e] = mkc(0.0, 0.0);
    } else {
      it.V[e] = cdiv(q, keff);
    }
    if (r == 0) it.gamma[c] = g;
  }
}

// Magnetic layers: P / k0^2 and Q element by element (MagItem).  The
// diagonal matrices Da, Db scale rows and columns of E and H; the
// permeability and permittivity convolution matrices enter unscaled.
__global__ void assemble_pq_kernel(const MagItem* items, int N, int with_p) {
  const MagItem it = items[blockIdx.y];
  const int n = 2 * N;
  const double k02 = it.k0 * it.k0, ik02 = 1.0 / k02;
  const size_t total = (size_t)n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / n), c = (int)(e % n);
    const int rr = r % N, cc = c % N;
    const size_t o = (size_t)rr * N + cc;
    const bool top = r < N, left = c < N;
    // row factor of block row, column factor of block column
    const double fr_p = top ? it.ab[rr].x : it.ab[N + rr].x;
    const double fc_p = left ? it.ab[N + cc].x : it.ab[cc].x;
    cplx q = cscale(it.H[o], fr_p * fc_p);
    if (top && left) q = cneg(q);
    else if (top) q = csub(q, cscale(it.fe22[o], k02));
    else if (left) q = cadd(cneg(q), cscale(it.fe11[o], k02));
    it.Q[e] = q;
    if (with_p) {
      cplx p = cscale(it.E[o], fr_p * fc_p);
      if (top && !left) p = csub(cscale(it.fm22[o], k02), p);
      else if (!top && left) p = csub(p, cscale(it.fm11[o], k02));
      else if (!top) p = cneg(p);
      it.P[e] = cscale(p, ik02);
    }
  }
}

// C (n x 2, row-major) = [e_r0, e_r1] for every item.
__global__ void unit_columns_kernel(cplx* const* C, int n, int r0, int r1) {
  cplx* c = C[blockIdx.y];
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)2 * n; e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / 2), k = (int)(e % 2);
    c[e] = mkc(r == (k == 0 ? r0 : r1) ? 1.0 : 0.0, 0.0);
  }
}

// Modes of a magnetic layer: V = (Q W) diag(1/keff) (rcwa/WaveEquationSolver.cpp:36).
__global__ void finish_modes_scaled_kernel(const LayerItem* items, int N, int* status) {
  const LayerItem it = items[blockIdx.y];
  const int n = 2 * N;
  const size_t total = (size_t)n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / n), c = (int)(e % n);
    const cplx g = gamma_sqrt(it.mu[c]);
    const cplx keff = cscale(g, it.k0);
    if (keff.x == 0.0 && keff.y == 0.0) {
      set_status(status, it.point, RCWA_ERR_GRAZING);
      it.V[e] = mkc(0.0, 0.0);
    } else {
      it.V[e] = cdiv(it.V[e], keff);
    }
    if (r == 0) it.gamma[c] = g;
  }
}

// Uniform half-space: P*Q = k0^2 (k0^2 eps - a^2 - b^2) per harmonic for both
// field components, so W = I, keff = k0*GammaSqrtOp(k0^2 eps - a^2 - b^2) and
// V = Q / keff with Q's 2x2 block per harmonic
//   [[-a b, a^2 - k0^2 eps], [k0^2 eps - b^2, a b]].
// A magnetic half-space (uniform mu): P*Q = k0^2 (k0^2 eps mu - a^2 - b^2)
// and Q = [[-a b / mu, a^2 / mu - k0^2 eps], [k0^2 eps - b^2 / mu, a b / mu]]
// (the magnetic branch with Fmu = mu I, H = I / mu).
__global__ void halfspace_kernel(const HalfItem* items, int N, int* status) {
  const HalfItem it = items[blockIdx.y];
  const int n = 2 * N;
  const double k02 = it.k0 * it.k0;
  const cplx ke = cscale(it.eps, k02);
  const cplx kem = it.magnetic ? cscale(cmul(it.eps, it.mu), k02) : ke;
  const cplx minv = it.magnetic ? cdiv(mkc(1.0, 0.0), it.mu) : mkc(1.0, 0.0);
  const size_t total = (size_t)n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / n), c = (int)(e % n);
    it.W[e] = mkc(r == c ? 1.0 : 0.0, 0.0);
    const int h = c % N;
    cplx v = mkc(0.0, 0.0);
    const cplx a = it.ab[h], b = it.ab[N + h];
    const cplx mu = csub(csub(kem, cmul(a, a)), cmul(b, b));
    const cplx g = gamma_sqrt(mu);
    const cplx keff = cscale(g, it.k0);
    if (r % N == h) {
      cplx q;
      const bool top = r < N, left = c < N;
      if (!it.magnetic) {
        if (top && left) q = cneg(cmul(a, b));
        else if (top) q = csub(cmul(a, a), ke);
        else if (left) q = csub(ke, cmul(b, b));
        else q = cmul(a, b);
      } else {
        if (top && left) q = cneg(cmul(cmul(a, b), minv));
        else if (top) q = csub(cmul(cmul(a, a), minv), ke);
        else if (left) q = csub(ke, cmul(cmul(b, b), minv));
        else q = cmul(cmul(a, b), minv);
      }
      if (keff.x == 0.0 && keff.y == 0.0) set_status(status, it.point, RCWA_ERR_GRAZING);
      else v = cdiv(q, keff);
    }
    it.V[e] = v;
    if (r == 0) it.gamma[c] = g;
  }
}

// The interface matrices IH = Va^-1 Vb of rcwa/RCWASolver.cpp:537-543 when
// layer a is the uniform superstrate: Va couples only rows h and N+h, so its
// LU is N independent 2x2 eliminations (IE = Wa^-1 Wb = Wb since Wa = I).
__global__ void halfspace_solve_kernel(const HalfSolveItem* items, int N, int* status) {
  const HalfSolveItem it = items[blockIdx.y];
  const int n = 2 * N;
  const size_t total = (size_t)N * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int h = (int)(e / n), c = (int)(e % n);
    cplx p = it.V0[(size_t)h * n + h], q = it.V0[(size_t)h * n + N + h];
    cplx r = it.V0[(size_t)(N + h) * n + h], s = it.V0[(size_t)(N + h) * n + N + h];
    cplx x0 = it.X[(size_t)h * n + c], x1 = it.X[(size_t)(N + h) * n + c];
    if (cabs1(r) > cabs1(p)) {
      cplx t = p; p = r; r = t;
      t = q; q = s; s = t;
      t = x0; x0 = x1; x1 = t;
    }
    if (p.x == 0.0 && p.y == 0.0) { set_status(status, it.point, RCWA_ERR_SINGULAR); continue; }
    const cplx l = cdiv(r, p);
    const cplx u = csub(s, cmul(l, q));
    if (u.x == 0.0 && u.y == 0.0) { set_status(status, it.point, RCWA_ERR_SINGULAR); continue; }
    const cplx y1 = cdiv(csub(x1, cmul(l, x0)), u);
    const cplx y0 = cdiv(csub(x0, cmul(q, y1)), p);
    it.X[(size_t)h * n + c] = y0;
    it.X[(size_t)(N + h) * n + c] = y1;
  }
}

// waveRud = Phi Rud Phi, waveTdd = Tdd Phi, Phi = diag(exp(i gamma d))
// (rcwa/RCWASolver.cpp:421-434).
__global__ void phase_kernel(const PhaseItem* items, int n) {
  const PhaseItem it = items[blockIdx.y];
  const size_t total = (size_t)n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / n), c = (int)(e % n);
    const cplx gr = it.gamma[r], gc = it.gamma[c];
    const cplx pr = cexp_(mkc(-gr.y * it.thick, gr.x * it.thick));
    const cplx pc = cexp_(mkc(-gc.y * it.thick, gc.x * it.thick));
    it.Rud[e] = cmul(cmul(pr, it.Rud[e]), pc);
    it.Tdd[e] = cmul(it.Tdd[e], pc);
  }
}

__global__ void axpby_kernel(const cplx* const* X, const cplx* const* Y, cplx* const* D, cplx a, cplx b, int n) {
  const cplx* x = X[blockIdx.y];
  const cplx* y = Y[blockIdx.y];
  cplx* d = D[blockIdx.y];
  const size_t total = (size_t)n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x)
    d[e] = cfma(a, x[e], cmul(b, y[e]));
}

__global__ void cascade_init_kernel(cplx* const* Rud, cplx* const* Tdd, int n) {
  cplx* R = Rud[blockIdx.y];
  cplx* T = Tdd[blockIdx.y];
  const size_t total = (size_t)n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    R[e] = mkc(0.0, 0.0);
    T[e] = mkc((e / n) == (e % n) ? 1.0 : 0.0, 0.0);
  }
}

// generateHorizontalPlaneWave + scatterPlaneWave + sums
// (rcwa/RCWASolver.cpp:1778-1908, sol/rcwa_bridge.cpp:311-312).  With the
// analytic half-space modes W_ref = W_trn = I, c = [px delta; py delta], so
// cref = px Rud(:,inc) + py Rud(:,N+inc) and the harmonics are cref itself;
// with a patterned half-space c = W_ref^-1 [px delta; py delta] and the
// harmonics W_ref Rud c, W_trn Tdd c come from the precomputed responses
// Rc, Tc.
__global__ void scatter_kernel(const ScatterItem* items, int N, int nx, int ny, int* status) {
  const ScatterItem it = items[blockIdx.x];
  const int inc = ny * ((nx - 1) / 2) + (ny - 1) / 2;
  const int n = 2 * N;
  const double k02 = it.k0 * it.k0;
  const cplx kr2 = cscale(it.n2_ref, k02), kt2 = cscale(it.n2_trn, k02);
  __shared__ double red[2][256];
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  // incident kz
  const cplx ai = it.ab[inc], bi = it.ab[N + inc];
  const cplx kzinc_c = cneg(csqrt_principal(csub(csub(kr2, cmul(ai, ai)), cmul(bi, bi))));
  const double kzinc = fabs(kzinc_c.x);
  double sr = 0.0, st = 0.0;
  for (int h = threadIdx.x; h < N; h += blockDim.x) {
    cplx rx, ry, tx, ty;
    if (it.Rc) {
      const cplx* Rr = it.Rc;
      const cplx* Tt = it.Tc;
      rx = cfma(it.px, Rr[(size_t)h * 2], cmul(it.py, Rr[(size_t)h * 2 + 1]));
      ry = cfma(it.px, Rr[(size_t)(N + h) * 2], cmul(it.py, Rr[(size_t)(N + h) * 2 + 1]));
      tx = cfma(it.px, Tt[(size_t)h * 2], cmul(it.py, Tt[(size_t)h * 2 + 1]));
      ty = cfma(it.px, Tt[(size_t)(N + h) * 2], cmul(it.py, Tt[(size_t)(N + h) * 2 + 1]));
    } else {
      const cplx* Rr = it.Rud;
      const cplx* Tt = it.Tdd;
      rx = cfma(it.px, Rr[(size_t)h * n + inc], cmul(it.py, Rr[(size_t)h * n + N + inc]));
      ry = cfma(it.px, Rr[(size_t)(N + h) * n + inc], cmul(it.py, Rr[(size_t)(N + h) * n + N + inc]));
      tx = cfma(it.px, Tt[(size_t)h * n + inc], cmul(it.py, Tt[(size_t)h * n + N + inc]));
      ty = cfma(it.px, Tt[(size_t)(N + h) * n + inc], cmul(it.py, Tt[(size_t)(N + h) * n + N + inc]));
    }
    const cplx a = it.ab[h], b = it.ab[N + h];
    const cplx kt = cadd(cmul(a, a), cmul(b, b));
    const cplx kzr = cneg(csqrt_principal(csub(kr2, kt)));
    const cplx kzt = csqrt_principal(csub(kt2, kt));
    if ((kzr.x == 0.0 && kzr.y == 0.0) || (kzt.x == 0.0 && kzt.y == 0.0)) {
      atomicOr(&bad, 1);
      continue;
    }
    const cplx rz = cdiv(cfma(a, rx, cmul(b, ry)), kzr);
    const cplx tz = cdiv(cfma(a, tx, cmul(b, ty)), kzt);
    const double r3 = cnorm2(rx) + cnorm2(ry) + cnorm2(rz);
    const double t3 = cnorm2(tx) + cnorm2(ty) + cnorm2(tz);
    const double REF = fabs(kzr.x) * r3 / kzinc;
    const double TRN = it.trn_scale * fabs(kzt.x) * t3 / kzinc;
    if (it.ref) it.ref[h] = REF;
    if (it.trn) it.trn[h] = TRN;
    sr += REF;
    st += TRN;
  }
  red[0][threadIdx.x] = sr;
  red[1][threadIdx.x] = st;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      red[0][threadIdx.x] += red[0][threadIdx.x + s];
      red[1][threadIdx.x] += red[1][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *it.R = red[0][0];
    *it.T = red[1][0];
    if (bad || kzinc < 1e-12 * it.k0) set_status(status, it.point, RCWA_ERR_GRAZING);
    else if (!isfinite(red[0][0]) || !isfinite(red[1][0])) set_status(status, it.point, RCWA_ERR_NONFINITE);
  }
}

__global__ void fold_info_kernel(const int* info, const int* item_point, int count, int code, int* status) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < count; b += gridDim.x * blockDim.x) {
    const int v = info[b];
    if (v != 0) atomicCAS(&status[item_point[b]], 0, code > 0 ? code : v);
  }
}

inline dim3 ew_grid(size_t elems, int count) {
  size_t blocks = (elems + 255) / 256;
  if (blocks > 1024) blocks = 1024;
  return dim3((unsigned)blocks, (unsigned)count);
}

}  // namespace

cudaError_t assemble_m(const LayerItem* items, int count, int N, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  assemble_m_kernel<<<ew_grid((size_t)4 * N * N, count), 256, 0, st>>>(items, N);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t finish_modes(const LayerItem* items, int count, int N, int* status, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  finish_modes_kernel<<<ew_grid((size_t)4 * N * N, count), 256, 0, st>>>(items, N, status);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t unit_columns(cplx* const* C, int n, int r0, int r1, int count, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  unit_columns_kernel<<<ew_grid((size_t)2 * n, count), 256, 0, st>>>(C, n, r0, r1);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t assemble_pq(const MagItem* items, int count, int N, bool with_p, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  assemble_pq_kernel<<<ew_grid((size_t)4 * N * N, count), 256, 0, st>>>(items, N, with_p ? 1 : 0);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t finish_modes_scaled(const LayerItem* items, int count, int N, int* status, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  finish_modes_scaled_kernel<<<ew_grid((size_t)4 * N * N, count), 256, 0, st>>>(items, N, status);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t halfspace_modes(const HalfItem* items, int count, int N, int* status, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  halfspace_kernel<<<ew_grid((size_t)4 * N * N, count), 256, 0, st>>>(items, N, status);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t halfspace_solve(const HalfSolveItem* items, int count, int N, int* status, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  halfspace_solve_kernel<<<ew_grid((size_t)2 * N * N, count), 256, 0, st>>>(items, N, status);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t apply_phase(const PhaseItem* items, int count, int n, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  phase_kernel<<<ew_grid((size_t)n * n, count), 256, 0, st>>>(items, n);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t scatter_efficiencies(const ScatterItem* items, int count, int N, int nx, int ny, int* status,
                                 cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  scatter_kernel<<<count, 256, 0, st>>>(items, N, nx, ny, status);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t zaxpby_batched(const cplx* const* X, const cplx* const* Y, cplx* const* D, cplx a, cplx b, int n,
                           int count, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  axpby_kernel<<<ew_grid((size_t)n * n, count), 256, 0, st>>>(X, Y, D, a, b, n);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t cascade_init(cplx* const* Rud, cplx* const* Tdd, int n, int count, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  cascade_init_kernel<<<ew_grid((size_t)n * n, count), 256, 0, st>>>(Rud, Tdd, n);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t fold_info(const int* info, const int* item_point, int count, int code, int* status,
                      cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  fold_info_kernel<<<(count + 255) / 256, 256, 0, st>>>(info, item_point, count, code, status);
  ++launch_counter();
  return cudaGetLastError();
}
