// Element-wise and reduction kernels specific to the RCWA solve.
#pragma once
#include "common.cuh"

// One patterned-layer job: the wave-equation matrix of one layer at one point.
struct LayerItem {
  const cplx* fe11;   // N x N  DiscontinuousX
  const cplx* fe22;   // N x N  DiscontinuousY
  const cplx* X1;     // N x N  E * diag(alpha) * fe11, E = fe33^-1
  const cplx* X2;     // N x N  E * diag(beta)  * fe22
  const cplx* ab;     // alpha[N] then beta[N] (complex, imaginary part 0)
  cplx* M;            // n x n  (P*Q)/k0^2
  cplx* W;            // n x n  eigenvectors (row-major)
  cplx* V;            // n x n  on input rows [0,N) = fe22 Wb, rows [N,2N) = fe11 Wt
  const cplx* mu;     // n eigenvalues of M
  cplx* gamma;        // n  Layer::gamma()
  double k0;
  int point;
};

// One magnetic patterned layer (relative permeability != 1 in some cell):
// the dense P and Q of the magnetic branch of Layer::waveEqnCoeff
// (rcwa/Layer.cpp:128-164, 205-213), E = fe33^-1, H = fmu33^-1:
//   P = [[Da E Db, k0^2 Fmu22 - Da E Da], [Db E Db - k0^2 Fmu11, -Db E Da]]
//   Q = [[-Da H Db, Da H Da - k0^2 Fe22], [-Db H Db + k0^2 Fe11, Db H Da]]
struct MagItem {
  const cplx* E;      // N x N  permittivity ContinuousXY inverse
  const cplx* H;      // N x N  permeability ContinuousXY inverse
  const cplx* fe11;   // N x N  permittivity DiscontinuousX
  const cplx* fe22;   // N x N  permittivity DiscontinuousY
  const cplx* fm11;   // N x N  permeability DiscontinuousX
  const cplx* fm22;   // N x N  permeability DiscontinuousY
  const cplx* ab;     // alpha[N] then beta[N]
  cplx* P;            // n x n  P / k0^2 (written when requested)
  cplx* Q;            // n x n  Q
  double k0;
};

// Uniform half-space of one point.
struct HalfItem {
  const cplx* ab;
  cplx eps;
  cplx mu;            // relative permeability (1: the non-magnetic formulas)
  int magnetic;       // mu != 1
  double k0;
  cplx* W;            // n x n  (identity)
  cplx* V;            // n x n  Q*W/keff, 2x2 blocks per harmonic
  cplx* gamma;        // n
  int point;
};

// Interface whose upper layer is a uniform half-space: X <- V0^-1 X.
struct HalfSolveItem {
  cplx* X;            // n x n right-hand sides, overwritten
  const cplx* V0;     // n x n half-space V (2x2 blocks of diagonal N x N blocks)
  int point;
};

struct PhaseItem {
  cplx* Rud;
  cplx* Tdd;
  const cplx* gamma;
  double thick;
};

struct ScatterItem {
  const cplx* Rud;
  const cplx* Tdd;
  // a point with a patterned half-space: the responses to the two unit
  // plane-wave inputs, n x 2 row-major, W_ref Rud W_ref^-1 [e_inc, e_N+inc]
  // and W_trn Tdd W_ref^-1 [e_inc, e_N+inc] (nullptr: W_ref = W_trn = I and
  // the Rud, Tdd columns inc and N+inc are these responses)
  const cplx* Rc = nullptr;
  const cplx* Tc = nullptr;
  const cplx* ab;
  cplx n2_ref, n2_trn;  // eps * mu of the half-spaces: k^2 = k0^2 eps mu
  double trn_scale;     // |mu_ref / mu_trn|, the flux ratio of the transmitted orders
  double k0;
  cplx px, py;
  double* ref;        // N (device)
  double* trn;        // N (device)
  double* R;          // scalar (device)
  double* T;
  int point;
};

cudaError_t assemble_m(const LayerItem* items, int count, int N, cudaStream_t st);
cudaError_t finish_modes(const LayerItem* items, int count, int N, int* status, cudaStream_t st);
cudaError_t halfspace_modes(const HalfItem* items, int count, int N, int* status, cudaStream_t st);
// C (n x 2, row-major) = [e_r0, e_r1] for every item
cudaError_t unit_columns(cplx* const* C, int n, int r0, int r1, int count, cudaStream_t st);
// P / k0^2 (with_p) and Q of magnetic layers, n x n each
cudaError_t assemble_pq(const MagItem* items, int count, int N, bool with_p, cudaStream_t st);
// V <- V diag(1/keff), gamma = GammaSqrtOp(mu): the modes of a layer whose
// V arrives as the full product Q W
cudaError_t finish_modes_scaled(const LayerItem* items, int count, int N, int* status, cudaStream_t st);
cudaError_t apply_phase(const PhaseItem* items, int count, int n, cudaStream_t st);
// X <- V0^-1 X per item: for each order h, rows h and N+h of X against the 2x2
// block [V0(h,h) V0(h,N+h); V0(N+h,h) V0(N+h,N+h)] by Gaussian elimination
// with partial pivoting (the steps the dense LU takes on this structure);
// an exactly singular block sets RCWA_ERR_SINGULAR for the item's point.
cudaError_t halfspace_solve(const HalfSolveItem* items, int count, int N, int* status, cudaStream_t st);
cudaError_t scatter_efficiencies(const ScatterItem* items, int count, int N, int nx, int ny, int* status,
                                 cudaStream_t st);
// D = a*X + b*Y (n x n) for every item
cudaError_t zaxpby_batched(const cplx* const* X, const cplx* const* Y, cplx* const* D, cplx a, cplx b, int n,
                           int count, cudaStream_t st);
// zero (n x n) the Rud and set Tdd = I
cudaError_t cascade_init(cplx* const* Rud, cplx* const* Tdd, int n, int count, cudaStream_t st);
// status[item_point[b]] <- code when info[b] != 0 (first error wins)
cudaError_t fold_info(const int* info, const int* item_point, int count, int code_if_nonzero, int* status,
                      cudaStream_t st);
