// Kernel (a): Fourier coefficient tables and convolution matrices.
//
// FourierSolver1D::solve      rcwa/FourierSolver1D.cpp:11-41
// ToeplitzMatrixXcs           rcwa/ToeplitzMatrixXcs.cpp:8-44
// BlockToeplitzMatrixXcs      rcwa/BlockToeplitzMatrixXcs.cpp:5-53
// FourierSolver2D::solve      rcwa/FourierSolver2D.cpp:12-351
//
// Stage 1 (one CTA per layer) evaluates the closed-form sinc coefficients of
// the cell grid into small tables: the 2D Laurent table, the strip-indicator
// coefficients, and the Toeplitz matrices of the 1/eps coefficients of every
// strip.  Stage 2 inverts those Toeplitz matrices with the batched LU.  Stage 3
// is the HBM-bound gather that writes the three N x N matrices from tables
// staged in shared memory, whole rows at a time.
#include <algorithm>

#include "fourier.cuh"
#include "linalg.cuh"

namespace {

constexpr double kPi = 3.1415926535897932;  // the reference's Pi (rcwa/defns.h:25)

struct TabLayout {
  size_t f2d, fy, fx, tx, txinv, ty, tyinv, total;
};

__host__ __device__ inline TabLayout tab_layout(int nx, int ny, int ncx, int ncy) {
  const size_t nys = (size_t)max(ncy - 1, 1), nxs = (size_t)max(ncx - 1, 1);
  TabLayout t;
  t.f2d = 0;
  t.fy = t.f2d + (size_t)(2 * nx - 1) * (2 * ny - 1);
  t.fx = t.fy + nys * (2 * ny - 1);
  t.tx = t.fx + nxs * (2 * nx - 1);
  t.txinv = t.tx + nys * nx * nx;
  t.ty = t.txinv + nys * nx * nx;
  t.tyinv = t.ty + nxs * ny * ny;
  t.total = t.tyinv + nxs * ny * ny;
  return t;
}

__device__ __forceinline__ double sinc_ref(double x) {
  return x == 0.0 ? 1.0 : sin(kPi * x) / (kPi * x);
}

// One term of FourierSolver1D::solve for cell [x0, x1] of a period d and
// order m, value fj: fj/d * exp(-i m pi (x1+x0)/d) * sinc(m (x1-x0)/d) * (x1-x0).
__device__ __forceinline__ cplx fterm(cplx fj, double x0, double x1, double d, int m) {
  const double w = x1 - x0;
  if (m == 0) return cscale(fj, w / d);
  double s, c;
  sincos(m * kPi * (x1 + x0) / d, &s, &c);
  const cplx ph = mkc(c, -s);
  return cscale(cmul(cscale(fj, 1.0 / d), ph), sinc_ref(m * w / d) * w);
}

// Tables for each job; thread-strided loops, no cross-thread dependencies.
__global__ void conv_tables_kernel(ConvJob* jobs, int nx, int ny, int max_ncx, int max_ncy) {
  const ConvJob J = jobs[blockIdx.x];
  const TabLayout L = tab_layout(nx, ny, max_ncx, max_ncy);
  cplx* tab = J.tab;
  const int nxs = J.ncx - 1, nys = J.ncy - 1;
  const int mxs = max_ncx - 1, mys = max_ncy - 1;
  const double dx = J.cx[J.ncx - 1] - J.cx[0];
  const double dy = J.cy[J.ncy - 1] - J.cy[0];
  const int PX = 2 * nx - 1, PY = 2 * ny - 1;
  const int hx = (PX - 1) / 2, hy = (PY - 1) / 2;
  if (J.f2d) {
    // a given Laurent table: copied; the strip tables stay identity / zero
    for (int idx = threadIdx.x; idx < PX * PY; idx += blockDim.x) tab[L.f2d + idx] = J.f2d[idx];
    for (int idx = threadIdx.x; idx < mys * PY; idx += blockDim.x) tab[L.fy + idx] = mkc(0.0, 0.0);
    for (int idx = threadIdx.x; idx < mxs * PX; idx += blockDim.x) tab[L.fx + idx] = mkc(0.0, 0.0);
    for (int idx = threadIdx.x; idx < mys * nx * nx; idx += blockDim.x) {
      const int r = (idx / nx) % nx, c = idx % nx;
      tab[L.tx + idx] = tab[L.txinv + idx] = mkc(r == c ? 1.0 : 0.0, 0.0);
    }
    for (int idx = threadIdx.x; idx < mxs * ny * ny; idx += blockDim.x) {
      const int r = (idx / ny) % ny, c = idx % ny;
      tab[L.ty + idx] = tab[L.tyinv + idx] = mkc(r == c ? 1.0 : 0.0, 0.0);
    }
    return;
  }
  // strip indicators: fY[i][q] (y strip i), fX[i][p] (x strip i)
  for (int idx = threadIdx.x; idx < mys * PY; idx += blockDim.x) {
    const int i = idx / PY, q = idx % PY;
    tab[L.fy + idx] = (i < nys) ? fterm(mkc(1.0, 0.0), J.cy[i], J.cy[i + 1], dy, q - hy) : mkc(0.0, 0.0);
  }
  for (int idx = threadIdx.x; idx < mxs * PX; idx += blockDim.x) {
    const int i = idx / PX, p = idx % PX;
    tab[L.fx + idx] = (i < nxs) ? fterm(mkc(1.0, 0.0), J.cx[i], J.cx[i + 1], dx, p - hx) : mkc(0.0, 0.0);
  }
  // Laurent table F2D[p][q] = sum_i (x coefficients of eps row i)[p] * fY_i[q]
  for (int idx = threadIdx.x; idx < PX * PY; idx += blockDim.x) {
    const int p = idx / PY, q = idx % PY;
    cplx acc = mkc(0.0, 0.0);
    for (int i = 0; i < nys; ++i) {
      cplx fx = mkc(0.0, 0.0);
      for (int j = 0; j < nxs; ++j) fx = cadd(fx, fterm(J.eps[(size_t)i * nxs + j], J.cx[j], J.cx[j + 1], dx, p - hx));
      const cplx fy = fterm(mkc(1.0, 0.0), J.cy[i], J.cy[i + 1], dy, q - hy);
      acc = cfma(fx, fy, acc);
    }
    tab[L.f2d + idx] = acc;
  }
  // Toeplitz matrices of the 1/eps coefficients: TX_i (x, per y strip),
  // TY_i (y, per x strip); T(r, c) = F[(r - c) + n - 1]; unused strips = I.
  for (int idx = threadIdx.x; idx < mys * nx * nx; idx += blockDim.x) {
    const int i = idx / (nx * nx), r = (idx / nx) % nx, c = idx % nx;
    cplx v;
    if (i < nys) {
      v = mkc(0.0, 0.0);
      for (int j = 0; j < nxs; ++j)
        v = cadd(v, fterm(cdiv(mkc(1.0, 0.0), J.eps[(size_t)i * nxs + j]), J.cx[j], J.cx[j + 1], dx, r - c));
    } else {
      v = mkc(r == c ? 1.0 : 0.0, 0.0);
    }
    tab[L.tx + idx] = v;
    tab[L.txinv + idx] = mkc(r == c ? 1.0 : 0.0, 0.0);
  }
  for (int idx = threadIdx.x; idx < mxs * ny * ny; idx += blockDim.x) {
    const int i = idx / (ny * ny), r = (idx / ny) % ny, c = idx % ny;
    cplx v;
    if (i < nxs) {
      v = mkc(0.0, 0.0);
      for (int j = 0; j < nys; ++j)
        v = cadd(v, fterm(cdiv(mkc(1.0, 0.0), J.eps[(size_t)j * nxs + i]), J.cy[j], J.cy[j + 1], dy, r - c));
    } else {
      v = mkc(r == c ? 1.0 : 0.0, 0.0);
    }
    tab[L.ty + idx] = v;
    tab[L.tyinv + idx] = mkc(r == c ? 1.0 : 0.0, 0.0);
  }
}

// Gather: the three N x N convolution matrices, written row by row.
//   fe33(row,col) = F2D[(m-j)+nx-1][(n-l)+ny-1]
//   fe11(row,col) = sum_i fY_i[(n-l)+ny-1] * TXinv_i[m][j]
//   fe22(row,col) = sum_i fX_i[(m-j)+nx-1] * TYinv_i[n][l]
// with m = row/ny, n = row%ny, j = col/ny, l = col%ny.  A CTA owns rows n0..n1
// of block row m of one layer.  Everything its outputs depend on is staged in
// shared memory first: the F2D rows m..m+nx-1, the per-(j, q) sums
// C11[j][q] = sum_i fY_i[q] TXinv_i[m][j] (so fe11 becomes a table look-up),
// the weights fX_i[m-j+nx-1] and, when they fit, the TYinv blocks.  The output
// then streams to HBM as whole rows, 16-byte elements on consecutive threads.
constexpr int kGatherThreads = 256;
constexpr size_t kGatherSmemMax = 200 * 1024;

__host__ __device__ inline size_t gather_smem_base(int nx, int ny, int max_ncx) {
  const size_t PY = 2 * (size_t)ny - 1, mxs = (size_t)max(max_ncx - 1, 1);
  return sizeof(cplx) * (2 * (size_t)nx * PY + (size_t)nx * mxs);
}
__host__ __device__ inline size_t gather_smem_ty(int ny, int max_ncx) {
  return sizeof(cplx) * (size_t)max(max_ncx - 1, 1) * ny * ny;
}

__global__ void __launch_bounds__(kGatherThreads) conv_gather_kernel(const ConvJob* jobs, int nx, int ny,
                                                                    int max_ncx, int max_ncy, int rows_per_cta,
                                                                    int ty_in_smem) {
  extern __shared__ __align__(16) unsigned char gsm[];
  const ConvJob J = jobs[blockIdx.z];
  const TabLayout L = tab_layout(nx, ny, max_ncx, max_ncy);
  const cplx* __restrict__ tab = J.tab;
  const int N = nx * ny;
  const int nxs = J.ncx - 1, nys = J.ncy - 1, mxs = max(max_ncx - 1, 1);
  const int PY = 2 * ny - 1, PX = 2 * nx - 1;
  const int m = blockIdx.x;
  const int n0 = blockIdx.y * rows_per_cta, n1 = min(ny, n0 + rows_per_cta);
  if (n0 >= n1) return;
  cplx* F33 = reinterpret_cast<cplx*>(gsm);  // [nx][PY]
  cplx* C11 = F33 + (size_t)nx * PY;         // [nx][PY]
  cplx* W22 = C11 + (size_t)nx * PY;         // [nx][mxs]
  cplx* TYs = W22 + (size_t)nx * mxs;        // [mxs][ny][ny] when staged
  const cplx* TY = ty_in_smem ? TYs : tab + L.tyinv;
  const bool laurent = J.f2d != nullptr;  // all three matrices from the F2D table
  const int tid = threadIdx.x;
  for (int idx = tid; idx < nx * PY; idx += blockDim.x) {
    const int j = idx / PY, q = idx % PY;
    F33[idx] = __ldg(&tab[L.f2d + (size_t)(m - j + nx - 1) * PY + q]);
    cplx acc = mkc(0.0, 0.0);
    for (int i = 0; i < nys; ++i)
      acc = cfma(__ldg(&tab[L.fy + (size_t)i * PY + q]), __ldg(&tab[L.txinv + ((size_t)i * nx + m) * nx + j]), acc);
    C11[idx] = acc;
  }
  for (int idx = tid; idx < nx * mxs; idx += blockDim.x) {
    const int j = idx / mxs, i = idx % mxs;
    W22[idx] = i < nxs ? __ldg(&tab[L.fx + (size_t)i * PX + (m - j + nx - 1)]) : mkc(0.0, 0.0);
  }
  if (ty_in_smem)
    for (int idx = tid; idx < nxs * ny * ny; idx += blockDim.x) TYs[idx] = __ldg(&tab[L.tyinv + idx]);
  __syncthreads();
  for (int n = n0; n < n1; ++n) {
    const size_t row = (size_t)(m * ny + n) * N;
    for (int c = tid; c < N; c += blockDim.x) {
      const int j = c / ny, l = c - j * ny;
      const int t = j * PY + (n - l + ny - 1);
      if (J.fe33) J.fe33[row + c] = F33[t];
      if (laurent) {
        if (J.fe11) J.fe11[row + c] = F33[t];
        if (J.fe22) J.fe22[row + c] = F33[t];
        continue;
      }
      if (J.fe11) J.fe11[row + c] = C11[t];
      if (J.fe22) {
        cplx acc = mkc(0.0, 0.0);
        const cplx* w = W22 + (size_t)j * mxs;
        const cplx* ty = TY + (size_t)n * ny + l;
        for (int i = 0; i < nxs; ++i) acc = cfma(w[i], ty[(size_t)i * ny * ny], acc);
        J.fe22[row + c] = acc;
      }
    }
  }
}

__global__ void fourier1d_kernel(const double* x, int nxe, double d, const cplx* f, int M, cplx* Ff) {
  for (int i = threadIdx.x; i < M; i += blockDim.x) {
    const int m = i - (M - 1) / 2;
    cplx acc = mkc(0.0, 0.0);
    for (int j = 1; j < nxe; ++j) acc = cadd(acc, fterm(f[j - 1], x[j - 1], x[j], d, m));
    Ff[i] = acc;
  }
}

__global__ void fill_table_ptrs(const ConvJob* jobs, int njobs, int nx, int ny, int max_ncx, int max_ncy,
                                cplx** tx, cplx** txinv, cplx** ty, cplx** tyinv) {
  const TabLayout L = tab_layout(nx, ny, max_ncx, max_ncy);
  const int mys = max_ncy - 1, mxs = max_ncx - 1;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < njobs * max(mys, mxs);
       idx += gridDim.x * blockDim.x) {
    const int b = idx / max(mys, mxs), i = idx % max(mys, mxs);
    cplx* tab = jobs[b].tab;
    if (i < mys) {
      tx[b * mys + i] = tab + L.tx + (size_t)i * nx * nx;
      txinv[b * mys + i] = tab + L.txinv + (size_t)i * nx * nx;
    }
    if (i < mxs) {
      ty[b * mxs + i] = tab + L.ty + (size_t)i * ny * ny;
      tyinv[b * mxs + i] = tab + L.tyinv + (size_t)i * ny * ny;
    }
  }
}

}  // namespace

size_t conv_table_elems(int nx, int ny, int ncx, int ncy) { return tab_layout(nx, ny, ncx, ncy).total; }

cudaError_t conv_matrices(const ConvLaunch& P, cudaStream_t st, StageProf* prof) {
  if (P.njobs <= 0) return cudaSuccess;
  const int mys = P.max_ncy - 1, mxs = P.max_ncx - 1;
  conv_tables_kernel<<<P.njobs, 256, 0, st>>>(P.jobs, P.nx, P.ny, P.max_ncx, P.max_ncy);
  ++launch_counter();
  fill_table_ptrs<<<(P.njobs * max(mys, mxs) + 255) / 256, 256, 0, st>>>(
      P.jobs, P.njobs, P.nx, P.ny, P.max_ncx, P.max_ncy, P.tx_ptrs, P.txinv_ptrs, P.ty_ptrs, P.tyinv_ptrs);
  ++launch_counter();
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  if ((err = zgetrf_batched(P.tx_ptrs, P.nx, P.nx, P.ipiv, P.info, P.njobs * mys, st)) != cudaSuccess) return err;
  if ((err = zgetrs_batched(P.tx_ptrs, P.nx, P.nx, P.ipiv, P.txinv_ptrs, P.nx, P.nx, P.njobs * mys, st)) !=
      cudaSuccess)
    return err;
  if ((err = zgetrf_batched(P.ty_ptrs, P.ny, P.ny, P.ipiv, P.info, P.njobs * mxs, st)) != cudaSuccess) return err;
  if ((err = zgetrs_batched(P.ty_ptrs, P.ny, P.ny, P.ipiv, P.tyinv_ptrs, P.ny, P.ny, P.njobs * mxs, st)) !=
      cudaSuccess)
    return err;
  if (prof) prof->mark(st, kStConvTables);
  // rows of a block row split so that the grid covers the SMs about twice
  int sms = 148;
  {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  const long long per_split = (long long)P.nx * P.njobs;
  int nsplit = (int)std::min<long long>(P.ny, std::max<long long>(1, (2LL * sms + per_split - 1) / per_split));
  const int rows = (P.ny + nsplit - 1) / nsplit;
  nsplit = (P.ny + rows - 1) / rows;
  size_t smem = gather_smem_base(P.nx, P.ny, P.max_ncx);
  const int ty_in_smem = smem + gather_smem_ty(P.ny, P.max_ncx) <= kGatherSmemMax ? 1 : 0;
  if (ty_in_smem) smem += gather_smem_ty(P.ny, P.max_ncx);
  if (smem > kGatherSmemMax) return cudaErrorInvalidValue;  // harmonic grid beyond the staged tables
  static SmemAttrOnce attr;
  if ((err = attr.ensure(conv_gather_kernel, (int)kGatherSmemMax)) != cudaSuccess) return err;
  dim3 grid(P.nx, nsplit, P.njobs);
  conv_gather_kernel<<<grid, kGatherThreads, smem, st>>>(P.jobs, P.nx, P.ny, P.max_ncx, P.max_ncy, rows, ty_in_smem);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t fourier1d_device(const double* x, int nxe, double d, const cplx* f, int M, cplx* Ff, cudaStream_t st) {
  fourier1d_kernel<<<1, 256, 0, st>>>(x, nxe, d, f, M, Ff);
  ++launch_counter();
  return cudaGetLastError();
}
