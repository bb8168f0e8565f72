// Batched eigen-decomposition of general complex matrices (right eigenvectors).
#pragma once
#include "common.cuh"

// Workspace bytes per matrix for zgeev_batched at order n.
size_t zgeev_workspace_bytes(int n);

// For every batch item: A (n x n row-major, destroyed: holds the Schur form on
// return) -> w (n eigenvalues), VR (n x n row-major, column k the unit-norm
// right eigenvector of w[k]).  work: batch * zgeev_workspace_bytes(n) bytes.
// info[b] = 0, or RCWA_ERR_NOCONV / RCWA_ERR_NONFINITE.
cudaError_t zgeev_batched(cplx* const* A, int n, int lda, cplx* w, cplx* const* VR, int ldv,
                          void* work, int* info, int batch, cudaStream_t st, StageProf* prof = nullptr);
