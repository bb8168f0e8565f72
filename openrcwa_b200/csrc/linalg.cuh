// Batched complex-FP64 dense linear algebra used by the RCWA engine.
// Matrices are row-major double2 with a leading dimension; a batch is given
// as a device array of per-item pointers so that items may live anywhere.
#pragma once
#include "common.cuh"

struct GemmArgs {
  const cplx* const* A;   // op(A) is M x K
  const cplx* const* B;   // op(B) is K x N
  const cplx* const* C;   // may be null when beta == 0
  cplx* const* D;         // D = alpha*op(A)*diag(s)*op(B) + beta*C + gammaI*I
  const cplx* const* s;   // optional diagonal between op(A) and op(B) (length K)
  int M, N, K;
  int lda, ldb, ldc, ldd;
  int transA, transB;     // 0: as stored, 1: transposed
  cplx alpha, beta, gammaI;
  int batch;
  // strided batches: used for an operand whose pointer array above is null
  const cplx* A0 = nullptr;
  const cplx* B0 = nullptr;
  cplx* D0 = nullptr;
  size_t sA = 0, sB = 0, sD = 0;
  // element offsets added to every item's A, B, C and D (sub-blocks)
  size_t offA = 0, offB = 0, offC = 0, offD = 0;
  // op(B) is upper triangular: output column tile [n0, n0+64) only needs
  // k < n0 + 64
  int triB = 0;
};

// D = alpha*op(A)*diag(s)*op(B) + beta*C + gammaI*I for every batch item.
cudaError_t zgemm_batched(const GemmArgs& g, cudaStream_t st);

// In-place LU with partial pivoting (row interchanges, LAPACK getrf
// convention, 0-based pivots) of square n x n matrices.  info[b] = 0, or k+1
// when U(k,k) is exactly zero.  schedule 0: one CTA factors each matrix;
// schedule 1: panel by panel, the panel factorisation one CTA per matrix and
// the triangular solve and trailing update spread over all SMs; -1: the
// default rule (zgetrf_default_schedule: schedule 0 for n <= 128 or batches of
// at least four waves of CTAs, else 2 from n = 256 on, else 1); schedule 2: 128-column blocks, each
// factorised as in schedule 1 and followed by one K = 128 trailing update
// (zgetrf_blocked_batched in lu_blocked.cuh).  All pivot by the same rule;
// their rounding differs in the trailing updates.
int zgetrf_default_schedule(int n, int batch, int sms = 0);  // sms <= 0: this device's SM count
cudaError_t zgetrf_batched(cplx* const* A, int n, int lda, int* ipiv, int* info, int batch,
                           cudaStream_t st, int schedule = -1);
// Columns k0 .. ce-1 of the panel-by-panel LU, whose columns before k0 are
// factorised and whose columns from k0 on have taken every update of them:
// 32-column panels (row interchanges across whole rows) with the U12 solves
// and FP64 trailing updates confined to columns < ce.  The columns from ce on
// are left to the caller (a blocked LU's trailing update).  k0 = 0 clears info.
cudaError_t zgetrf_columns(cplx* const* A, int n, int lda, int k0, int ce, int* ipiv, int* info, int batch,
                           cudaStream_t st);

// Solve A X = B in place of B (n x nrhs) from the factors of zgetrf_batched.
cudaError_t zgetrs_batched(const cplx* const* LU, int n, int lda, const int* ipiv,
                           cplx* const* B, int nrhs, int ldb, int batch, cudaStream_t st);

// X = A^-1 (n x n, into X, not in place) from the factors of zgetrf_batched:
// the LAPACK getri order (L^-1 and U^-1 on the identity without the row
// interchanges, then the column interchanges), a third fewer flops than
// zgetrs_batched on the identity.
cudaError_t zgetri_batched(const cplx* const* LU, int n, int lda, const int* ipiv, cplx* const* X, int ldx,
                           int batch, cudaStream_t st);

// X <- X P for the column interchanges of zgetrf_batched (LAPACK getri's
// last step), every batch item.
cudaError_t zcolperm_batched(cplx* const* X, int n, int ldx, const int* ipiv, int batch, cudaStream_t st);

// B = I (n x n) for every batch item.
cudaError_t zset_identity_batched(cplx* const* B, int n, int ldb, int batch, cudaStream_t st);

// Copy src -> dst (rows x cols) for every batch item.
cudaError_t zcopy_batched(const cplx* const* src, int lds, cplx* const* dst, int ldd, int rows,
                          int cols, int batch, cudaStream_t st);
