// Convolution-matrix assembly (Laurent and inverse rules) for layers given as
// piecewise-constant permittivity on a rectangular cell grid.
#pragma once
#include "common.cuh"

// Geometry/material of one patterned layer as the device sees it.
struct ConvJob {
  const double* cx;    // ncx edges
  const double* cy;    // ncy edges
  const cplx* eps;     // (ncy-1) x (ncx-1), row = y strip
  int ncx, ncy;
  // outputs (row-major N x N, N = nx*ny); any may be null
  cplx* fe11;          // DiscontinuousX rule
  cplx* fe22;          // DiscontinuousY rule
  cplx* fe33;          // ContinuousXY rule
  // per-job table scratch (see conv_table_elems)
  cplx* tab;
  // a caller-given 2D Laurent table ((2nx-1) x (2ny-1), row p = x order
  // p-nx+1) instead of the cells: all three matrices are its block-Toeplitz
  // matrix (the Laurent rule for every tensor); nullptr for cell layers
  const cplx* f2d = nullptr;
};

// complex elements of table scratch needed by one job
size_t conv_table_elems(int nx, int ny, int ncx, int ncy);

// Fills fe11/fe22/fe33 for every job (same nx, ny for all jobs).  lu_* are
// scratch pointer arrays sized for the small Toeplitz inversions:
// the engine passes device buffers that hold max_strips*jobs pointers.
struct ConvLaunch {
  ConvJob* jobs;       // device array [njobs]
  int njobs, nx, ny;
  int max_ncx, max_ncy;
  // Toeplitz inverse scratch: one matrix per (job, strip)
  cplx** tx_ptrs;      // device [njobs*(max_ncy-1)] -> nx x nx matrices inside tab
  cplx** txinv_ptrs;
  cplx** ty_ptrs;      // device [njobs*(max_ncx-1)] -> ny x ny
  cplx** tyinv_ptrs;
  int* ipiv;           // device [njobs*max(max_ncy-1, max_ncx-1)*max(nx,ny)]
  int* info;           // device [njobs*max(...)]
};

// With prof, the time up to the gather is charged to the conv_tables stage
// (tables and Toeplitz inverses); the caller marks the gather's end.
cudaError_t conv_matrices(const ConvLaunch& L, cudaStream_t st, StageProf* prof = nullptr);

// FourierSolver1D::solve on the device: Ff[M] from edges x[nxe], f[nxe-1].
cudaError_t fourier1d_device(const double* x, int nxe, double d, const cplx* f, int M, cplx* Ff,
                             cudaStream_t st);
