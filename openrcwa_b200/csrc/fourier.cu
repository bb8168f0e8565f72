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
// is the HBM-bound gather that writes the three N x N matrices, each output
// element a short sum over strips read from the L1/L2-resident tables.
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

// Gather: one thread per output element of each N x N matrix.
//   fe33(row,col) = F2D[(m-j)+nx-1][(n-l)+ny-1]
//   fe11(row,col) = sum_i fY_i[(n-l)+ny-1] * TXinv_i[m][j]
//   fe22(row,col) = sum_i fX_i[(m-j)+nx-1] * TYinv_i[n][l]
// with m = row/ny, n = row%ny, j = col/ny, l = col%ny.
__global__ void __launch_bounds__(256) conv_gather_kernel(const ConvJob* jobs, int nx, int ny, int max_ncx,
                                                         int max_ncy) {
  const ConvJob J = jobs[blockIdx.y];
  const TabLayout L = tab_layout(nx, ny, max_ncx, max_ncy);
  const cplx* __restrict__ tab = J.tab;
  const int N = nx * ny;
  const int nxs = J.ncx - 1, nys = J.ncy - 1;
  const int PY = 2 * ny - 1, PX = 2 * nx - 1;
  const size_t total = (size_t)N * N;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int row = (int)(e / N), col = (int)(e % N);
    const int m = row / ny, n = row % ny, j = col / ny, l = col % ny;
    const int dm = m - j + nx - 1, dn = n - l + ny - 1;
    if (J.fe33) J.fe33[e] = __ldg(&tab[L.f2d + (size_t)dm * PY + dn]);
    if (J.fe11) {
      cplx acc = mkc(0.0, 0.0);
      for (int i = 0; i < nys; ++i)
        acc = cfma(__ldg(&tab[L.fy + (size_t)i * PY + dn]), __ldg(&tab[L.txinv + ((size_t)i * nx + m) * nx + j]), acc);
      J.fe11[e] = acc;
    }
    if (J.fe22) {
      cplx acc = mkc(0.0, 0.0);
      for (int i = 0; i < nxs; ++i)
        acc = cfma(__ldg(&tab[L.fx + (size_t)i * PX + dm]), __ldg(&tab[L.tyinv + ((size_t)i * ny + n) * ny + l]), acc);
      J.fe22[e] = acc;
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

cudaError_t conv_matrices(const ConvLaunch& P, cudaStream_t st) {
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
  const size_t NN = (size_t)P.nx * P.ny * P.nx * P.ny;
  const size_t nblk = (NN + 255) / 256;
  dim3 grid((unsigned)(nblk < 2048 ? nblk : 2048), P.njobs);
  conv_gather_kernel<<<grid, 256, 0, st>>>(P.jobs, P.nx, P.ny, P.max_ncx, P.max_ncy);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t fourier1d_device(const double* x, int nxe, double d, const cplx* f, int M, cplx* Ff, cudaStream_t st) {
  fourier1d_kernel<<<1, 256, 0, st>>>(x, nxe, d, f, M, Ff);
  ++launch_counter();
  return cudaGetLastError();
}
