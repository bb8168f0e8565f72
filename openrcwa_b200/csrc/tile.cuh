// Register-blocked complex-FP64 tile GEMM shared by the GEMM, LU, triangular
// solve and eigensolver kernels.  A CTA of kTileThreads (256) threads computes
// one 64x64 output tile; thread (tx, ty) owns rows ty+16i and columns tx+16j,
// i, j in [0, 4).  Operand slabs of 16 along K are staged in shared memory
// (one padding column avoids bank conflicts on the transposed stores).
#pragma once
#include "common.cuh"

constexpr int kTBM = 64;
constexpr int kTBN = 64;
constexpr int kTBK = 16;
constexpr int kTileThreads = 256;

struct TileSmem {
  cplx As[kTBK][kTBM + 1];
  cplx Bs[kTBK][kTBN + 1];
};

__device__ __forceinline__ void tile_zero(cplx acc[4][4]) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = mkc(0.0, 0.0);
}

// acc += op(A)[m0:m0+64, :K] * diag(s) * op(B)[:K, n0:n0+64], where op(A) is
// M x K and op(B) is K x N; TA/TB select the transposed reading of a
// row-major operand.  Out-of-range elements read as zero.  Every thread of
// the CTA must call this (it contains __syncthreads).
template <bool TA, bool TB>
__device__ __forceinline__ void tile_mma(TileSmem& sm, cplx acc[4][4], const cplx* __restrict__ A, int lda,
                                         const cplx* __restrict__ B, int ldb, const cplx* __restrict__ s,
                                         int M, int N, int K, int m0, int n0) {
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  for (int k0 = 0; k0 < K; k0 += kTBK) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int idx = tid + r * kTileThreads;
      int mm, kk;
      if (!TA) { kk = idx & 15; mm = idx >> 4; }
      else { mm = idx & 63; kk = idx >> 6; }
      const int gm = m0 + mm, gk = k0 + kk;
      cplx v = mkc(0.0, 0.0);
      if (gm < M && gk < K) v = TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
      sm.As[kk][mm] = v;
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int idx = tid + r * kTileThreads;
      int nn, kk;
      if (!TB) { nn = idx & 63; kk = idx >> 6; }
      else { kk = idx & 15; nn = idx >> 4; }
      const int gn = n0 + nn, gk = k0 + kk;
      cplx v = mkc(0.0, 0.0);
      if (gn < N && gk < K) {
        v = TB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn];
        if (s) v = cmul(s[gk], v);
      }
      sm.Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kTBK; ++kk) {
      cplx a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = sm.As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = sm.Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = cfma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
}

// D[m0.., n0..] = alpha*acc + beta*C + gammaI*(m == n)  (C may be null when
// beta is zero; C may alias D).
__device__ __forceinline__ void tile_store(const cplx acc[4][4], cplx* D, int ldd, const cplx* C, int ldc,
                                           cplx alpha, cplx beta, cplx gammaI, int M, int N, int m0, int n0) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty + 16 * i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx + 16 * j;
      if (n >= N) continue;
      cplx v = cmul(alpha, acc[i][j]);
      if (C) v = cfma(beta, C[(size_t)m * ldc + n], v);
      if (m == n) v = cadd(v, gammaI);
      D[(size_t)m * ldd + n] = v;
    }
  }
}

static_assert(sizeof(cplx) * 32 * 33 <= sizeof(TileSmem), "32x32 triangular block must fit the tile buffer");
