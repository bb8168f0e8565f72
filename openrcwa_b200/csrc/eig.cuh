// Batched eigen-decomposition of general complex matrices (right eigenvectors).
#pragma once
#include "common.cuh"

constexpr int kEigPanel = 64;  // Hessenberg panel width
// Default active-block size below which the Schur iteration switches from
// multishift sweeps with early deflation to single-shift sweeps (also its
// smallest allowed value).
constexpr int kSchurCrossover = 64;

// Workspace bytes per matrix for zgeev_batched at order n: Schur vectors and
// eigenvector matrix (2 n^2), work vectors (4 n), panel buffers (4 n x 64 and
// max(n, 64) x 64), the triangular factors of all panels, and the reflector
// scalars.
__host__ __device__ constexpr size_t zgeev_workspace_bytes(int n) {
  return ((2 * (size_t)n * n + 4 * (size_t)n + 4 * (size_t)n * kEigPanel +
           (size_t)(n > kEigPanel ? n : kEigPanel) * kEigPanel +
           ((size_t)(n + kEigPanel - 1) / kEigPanel + 1) * kEigPanel * kEigPanel) * 16 +
          (size_t)n * 8 + 255) & ~(size_t)255;
}

// For every batch item: A (n x n row-major, destroyed: holds the Schur form on
// return) -> w (n eigenvalues), VR (n x n row-major, column k the unit-norm
// right eigenvector of w[k]).  work: batch * zgeev_workspace_bytes(n) bytes.
// info[b] = 0, or RCWA_ERR_NOCONV / RCWA_ERR_NONFINITE.  ms_min: the Schur
// crossover (active blocks below it use single-shift sweeps; matrices below
// it run the single-shift kernel); values below kSchurCrossover are raised
// to it.
cudaError_t zgeev_batched(cplx* const* A, int n, int lda, cplx* w, cplx* const* VR, int ldv,
                          void* work, int* info, int batch, cudaStream_t st, StageProf* prof = nullptr,
                          int ms_min = kSchurCrossover);
