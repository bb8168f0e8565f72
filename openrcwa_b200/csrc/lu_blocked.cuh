// Blocked LU factorisation and solves with 128-wide blocks.
#pragma once
#include "common.cuh"

// The tensor-core context of a mixed plan's products: scale workspace (two
// ints per batch entry), error flag and plane scratch of zgemm_tf32x3_batched.
struct TcProducts {
  int* scale_ws;
  int* err;
  float* planes;
  size_t planes_bytes;
};

// LU with partial pivoting in place, like zgetrf_batched (same pivots rule,
// ipiv and info), in 128-column blocks whose trailing updates are batched
// products: FP64 (tc = nullptr), or 3xTF32 tcgen05 products with FP64
// accumulation for mixed plans (about 21 significant bits in the updates;
// the pivot choices then follow the perturbed values).
cudaError_t zgetrf_blocked_batched(cplx* const* A, int n, int lda, int* ipiv, int* info, int batch,
                                   const TcProducts* tc, cudaStream_t st);

// Solve A X = B in place of B (n x nrhs) from the factors of zgetrf_batched,
// or (inverse, nrhs = n) X = A^-1 into B in the getri order.  The updates
// between 128-row blocks are batched products: FP64 (tc = nullptr), or 3xTF32
// tcgen05 products with FP64 accumulation (about 21 significant bits in the
// updates, like a mixed plan's cascade products).  The blocks' triangles are
// solved in FP64 either way.
cudaError_t zgetrs_blocked_batched(const cplx* const* LU, int n, int lda, const int* ipiv, cplx* const* B, int nrhs,
                                   int ldb, int batch, bool inverse, const TcProducts* tc, cudaStream_t st);
