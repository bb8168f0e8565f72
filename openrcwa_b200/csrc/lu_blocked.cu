// Blocked LU factorisation and solves with 128-wide blocks.
//
// The factorisation factors each 128-column block with the panel-by-panel LU
// of linalg.cu confined to the block (zgetrf_columns: 32-column panels, row
// interchanges across whole rows), solves the block row right of it against
// the block's unit lower triangle, and updates the trailing matrix with one
// batched product of K = 128.
//
// The solves are right-looking blocked forward and back substitution over
// 128-row blocks: each block's triangle is solved in FP64 (one thread per
// right-hand side, 32-row quarters of the triangle staged in shared memory),
// and the rows below (forward) or above (backward) take the block's
// contribution through one batched product per block with FP64 accumulation
// into B.  The inverse variant solves on the identity without the row
// interchanges and interchanges the columns afterwards (the getri order), its
// forward updates cut to the columns the lower-triangular L^-1 fills.
//
// The batched products are the FP64 tensor-path GEMM (linalg.cu), or for
// mixed plans the 3xTF32 tcgen05 product (gemm_tc.cu).
#include "gemm_tc.cuh"
#include "linalg.cuh"
#include "lu_blocked.cuh"

namespace {

constexpr int kNb = 128;  // rows per block
// right-hand sides per CTA of the diagonal-block solves (one per thread): the
// tiles of the triangle staged in shared memory serve all of them; a build
// parameter (measured on B200, cfg2 mixed step, interface solves + tau
// inverse: 447 / 427 / 416 ms with 64 / 128 / 256; the results are the same,
// each column is solved alone)
#ifndef RCWA_DIAG_THREADS
#define RCWA_DIAG_THREADS 256
#endif
constexpr int kDiagThreads = RCWA_DIAG_THREADS;

// B <- P B: the interchanges of getrf, one thread per column
__global__ void laswp_kernel(cplx* const* Barr, int n, int ldb, int nrhs, const int* ipiv_all) {
  const int b = blockIdx.y, c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nrhs) return;
  cplx* B = Barr[b];
  const int* ipiv = ipiv_all + (size_t)b * n;
  for (int j = 0; j < n; ++j) {
    const int p = ipiv[j];
    if (p != j) {
      const cplx t = B[(size_t)j * ldb + c];
      B[(size_t)j * ldb + c] = B[(size_t)p * ldb + c];
      B[(size_t)p * ldb + c] = t;
    }
  }
}

__device__ __forceinline__ void load_tile32(cplx (*Tsm)[33], const cplx* LU, int lda, int r0, int c0, int h, int w) {
  for (int idx = threadIdx.x; idx < 32 * 32; idx += blockDim.x) {
    const int r = idx / 32, q = idx % 32;
    Tsm[r][q] = (r < h && q < w) ? LU[(size_t)(r0 + r) * lda + c0 + q] : mkc(0.0, 0.0);
  }
}

// Rows [r0, r0 + rows) of B (rows <= 128) <- T^-1 B for the diagonal block
// T of LU at (r0, r0): unit lower (forward) or upper (backward); columns
// [c_lo, nrhs) only (the inverse's forward pass skips columns whose rows
// here are still zero).
template <bool kUpper>
__global__ void __launch_bounds__(kDiagThreads) trsm_diag_kernel(const cplx* const* LUarr, int lda,
                                                                 cplx* const* Barr, int ldb, int nrhs, int r0,
                                                                 int rows, int c_lo) {
  __shared__ cplx Tsm[32][33];
  __shared__ cplx dinv[32];  // backward: reciprocals of the quarter's diagonal
  const int b = blockIdx.y;
  const int c = c_lo + blockIdx.x * kDiagThreads + threadIdx.x;
  const bool col = c < nrhs;
  const cplx* LU = LUarr[b];
  cplx* B = Barr[b];
  const int nq = (rows + 31) / 32;
  for (int step = 0; step < nq; ++step) {
    const int qi = kUpper ? nq - 1 - step : step;
    const int h0 = r0 + 32 * qi, hw = min(32, r0 + rows - h0);
    cplx x[32];
#pragma unroll
    for (int r = 0; r < 32; ++r) x[r] = (col && r < hw) ? B[(size_t)(h0 + r) * ldb + c] : mkc(0.0, 0.0);
    // the quarters already solved: above (forward) or below (backward); their
    // values come back four at a time so the loads overlap
    for (int s2 = 0; s2 < step; ++s2) {
      const int pj = kUpper ? nq - 1 - s2 : s2;
      const int p0 = r0 + 32 * pj, pw = min(32, r0 + rows - p0);
      __syncthreads();
      load_tile32(Tsm, LU, lda, h0, p0, hw, pw);
      __syncthreads();
      if (col) {
#pragma unroll
        for (int q0 = 0; q0 < 32; q0 += 4) {
          cplx y[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) y[u] = q0 + u < pw ? B[(size_t)(p0 + q0 + u) * ldb + c] : mkc(0.0, 0.0);
#pragma unroll
          for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int r = 0; r < 32; ++r) x[r] = cfma(cneg(Tsm[r][q0 + u]), y[u], x[r]);
        }
      }
    }
    __syncthreads();
    load_tile32(Tsm, LU, lda, h0, h0, hw, hw);
    if (kUpper) {
      __syncthreads();
      if (threadIdx.x < 32) {
        const int q = threadIdx.x;
        dinv[q] = q < hw ? cdiv(mkc(1.0, 0.0), Tsm[q][q]) : mkc(0.0, 0.0);
      }
    }
    __syncthreads();
    // the quarter's own triangle, column by column: each finished entry
    // updates the rows still open, all independent of one another
    if (col) {
      if (!kUpper) {
#pragma unroll
        for (int q = 0; q < 31; ++q)
#pragma unroll
          for (int r = q + 1; r < 32; ++r) x[r] = cfma(cneg(Tsm[r][q]), x[q], x[r]);
      } else {
#pragma unroll
        for (int q = 31; q >= 0; --q) {
          x[q] = cmul(x[q], dinv[q]);
#pragma unroll
          for (int r = 0; r < q; ++r) x[r] = cfma(cneg(Tsm[r][q]), x[q], x[r]);
        }
      }
#pragma unroll
      for (int r = 0; r < 32; ++r)
        if (r < hw) B[(size_t)(h0 + r) * ldb + c] = x[r];
    }
  }
}

}  // namespace

namespace {
cudaError_t blocked_update(const GemmArgs& g, const TcProducts* tc, cudaStream_t st) {
  return tc ? zgemm_tf32x3_batched(g, tc->scale_ws, tc->err, st, 128, tc->planes, tc->planes_bytes)
            : zgemm_batched(g, st);
}
}  // namespace

cudaError_t zgetrf_blocked_batched(cplx* const* A, int n, int lda, int* ipiv, int* info, int batch,
                                   const TcProducts* tc, cudaStream_t st) {
  if (batch <= 0 || n <= 0) return cudaSuccess;
  cudaError_t e;
  for (int kb = 0; kb < n; kb += kNb) {
    const int ke = min(n, kb + kNb);
    if ((e = zgetrf_columns(A, n, lda, kb, ke, ipiv, info, batch, st)) != cudaSuccess) return e;
    if (ke == n) break;
    // U12 = L11^-1 A12: the block's rows, columns ke .. n-1
    trsm_diag_kernel<false><<<dim3((n - ke + kDiagThreads - 1) / kDiagThreads, batch), kDiagThreads, 0, st>>>(
        (const cplx* const*)A, lda, A, lda, n, kb, ke - kb, ke);
    ++launch_counter();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // A22 -= L21 U12
    GemmArgs g{};
    g.A = (const cplx* const*)A; g.offA = (size_t)ke * lda + kb;
    g.B = (const cplx* const*)A; g.offB = (size_t)kb * lda + ke;
    g.C = (const cplx* const*)A; g.offC = (size_t)ke * lda + ke;
    g.D = A; g.offD = (size_t)ke * lda + ke;
    g.M = n - ke; g.N = n - ke; g.K = ke - kb;
    g.lda = lda; g.ldb = lda; g.ldc = lda; g.ldd = lda;
    g.alpha = mkc(-1.0, 0.0); g.beta = mkc(1.0, 0.0); g.gammaI = mkc(0.0, 0.0);
    g.batch = batch;
    if ((e = blocked_update(g, tc, st)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t zgetrs_blocked_batched(const cplx* const* LU, int n, int lda, const int* ipiv, cplx* const* B,
                                   int nrhs, int ldb, int batch, bool inverse, const TcProducts* tc, cudaStream_t st) {
  if (batch <= 0 || n <= 0 || nrhs <= 0) return cudaSuccess;
  if (inverse && nrhs != n) return cudaErrorInvalidValue;
  auto update = [&](const GemmArgs& g) { return blocked_update(g, tc, st); };
  cudaError_t e;
  if (inverse) {
    if ((e = zset_identity_batched(B, n, ldb, batch, st)) != cudaSuccess) return e;
  } else {
    laswp_kernel<<<dim3((nrhs + 127) / 128, batch), 128, 0, st>>>(B, n, ldb, nrhs, ipiv);
    ++launch_counter();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  // forward: L (unit lower)
  for (int kb = 0; kb < n; kb += kNb) {
    const int rw = min(kNb, n - kb);
    // the inverse's rows kb.. are zero in the columns past the block (L^-1 is lower triangular)
    const int c_lo = 0, c_hi = inverse ? kb + rw : nrhs;
    trsm_diag_kernel<false><<<dim3((c_hi - c_lo + kDiagThreads - 1) / kDiagThreads, batch), kDiagThreads, 0, st>>>(
        LU, lda, B, ldb, c_hi, kb, rw, c_lo);
    ++launch_counter();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int m2 = n - kb - rw;
    if (m2 > 0) {
      GemmArgs g{};
      g.A = LU; g.offA = (size_t)(kb + rw) * lda + kb;
      g.B = (const cplx* const*)B; g.offB = (size_t)kb * ldb;
      g.C = (const cplx* const*)B; g.offC = (size_t)(kb + rw) * ldb;
      g.D = B; g.offD = (size_t)(kb + rw) * ldb;
      g.M = m2; g.N = c_hi; g.K = rw;
      g.lda = lda; g.ldb = ldb; g.ldc = ldb; g.ldd = ldb;
      g.alpha = mkc(-1.0, 0.0); g.beta = mkc(1.0, 0.0); g.gammaI = mkc(0.0, 0.0);
      g.batch = batch;
      if ((e = update(g)) != cudaSuccess) return e;
    }
  }
  // backward: U
  for (int kb = ((n - 1) / kNb) * kNb; kb >= 0; kb -= kNb) {
    const int rw = min(kNb, n - kb);
    trsm_diag_kernel<true><<<dim3((nrhs + kDiagThreads - 1) / kDiagThreads, batch), kDiagThreads, 0, st>>>(
        LU, lda, B, ldb, nrhs, kb, rw, 0);
    ++launch_counter();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (kb > 0) {
      GemmArgs g{};
      g.A = LU; g.offA = (size_t)kb;
      g.B = (const cplx* const*)B; g.offB = (size_t)kb * ldb;
      g.C = (const cplx* const*)B; g.offC = 0;
      g.D = B; g.offD = 0;
      g.M = kb; g.N = nrhs; g.K = rw;
      g.lda = lda; g.ldb = ldb; g.ldc = ldb; g.ldd = ldb;
      g.alpha = mkc(-1.0, 0.0); g.beta = mkc(1.0, 0.0); g.gammaI = mkc(0.0, 0.0);
      g.batch = batch;
      if ((e = update(g)) != cudaSuccess) return e;
    }
  }
  if (inverse) return zcolperm_batched(B, n, ldb, ipiv, batch, st);
  return cudaSuccess;
}
