// Complex-FP64 tile GEMM on the FP64 tensor path, shared by the GEMM, LU,
// triangular solve and eigensolver kernels.  A CTA of kTileThreads (256)
// threads computes one 64x64 output tile with mma.sync m8n8k4 f64 (DMMA):
// warp w owns rows 16*(w%4) .. +16 and columns 32*(w/4) .. +32, i.e. 2 x 4
// blocks of 8 x 8, each a real and an imaginary accumulator fragment; a
// complex product takes four real MMAs.  Operand slabs of 16 along K are
// staged in shared memory as separate real and imaginary planes (row pitch
// 68 doubles makes the fragment loads conflict free), and the next slab is
// fetched into registers while the current one is multiplied.
#pragma once
#include "common.cuh"

constexpr int kTBM = 64;
constexpr int kTBN = 64;
constexpr int kTBK = 16;
constexpr int kTileThreads = 256;
constexpr int kTilePitch = 68;

struct TileSmem {
  double Ar[kTBK][kTilePitch], Ai[kTBK][kTilePitch];  // op(A)(m, k) at [k][m]
  double Br[kTBK][kTilePitch], Bi[kTBK][kTilePitch];  // op(B)(k, n) at [k][n]
};

// Accumulator layout: acc[i][j] with i = 2*rt + e, j = ct holds element
// (16*(w%4) + 8*rt + lane/4, 32*(w/4) + 8*ct + 2*(lane%4) + e) of the tile.
__device__ __forceinline__ void tile_zero(cplx acc[4][4]) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = mkc(0.0, 0.0);
}

// Barrier over the kTileThreads threads that run the tile routines (named
// barrier 1), so that a larger CTA can leave its other warps out of a tile
// product; with a CTA of exactly kTileThreads it is a full barrier.
__device__ __forceinline__ void tile_barrier() { asm volatile("bar.sync 1, %0;" ::"n"(kTileThreads) : "memory"); }

// d(8x8 fragment, two doubles per lane) += a(8x4) * b(4x8)
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// kL2: every operand load goes to L2 (ld.global.cg), for operands written by
// other CTAs of a cluster earlier in the same kernel.
template <bool TA, bool TB, bool kL2 = false>
__device__ __forceinline__ void tile_fetch(const cplx* __restrict__ A, int lda, const cplx* __restrict__ B, int ldb,
                                           const cplx* __restrict__ s, int M, int N, int K, int m0, int n0, int k0,
                                           cplx pa[4], cplx pb[4]) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int idx = tid + r * kTileThreads;
    int mm, kk;
    if (!TA) { kk = idx & 15; mm = idx >> 4; }
    else { mm = idx & 63; kk = idx >> 6; }
    const int gm = m0 + mm, gk = k0 + kk;
    cplx v = mkc(0.0, 0.0);
    if (gm < M && gk < K) {
      const cplx* pa_ = TA ? A + (size_t)gk * lda + gm : A + (size_t)gm * lda + gk;
      v = kL2 ? __ldcg(pa_) : *pa_;
    }
    pa[r] = v;
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
      const cplx* pb_ = TB ? B + (size_t)gn * ldb + gk : B + (size_t)gk * ldb + gn;
      v = kL2 ? __ldcg(pb_) : *pb_;
      if (s) v = cmul(kL2 ? __ldcg(s + gk) : s[gk], v);
    }
    pb[r] = v;
  }
}

template <bool TA, bool TB>
__device__ __forceinline__ void tile_stage(TileSmem& sm, const cplx pa[4], const cplx pb[4]) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int idx = tid + r * kTileThreads;
    int mm, kk;
    if (!TA) { kk = idx & 15; mm = idx >> 4; }
    else { mm = idx & 63; kk = idx >> 6; }
    sm.Ar[kk][mm] = pa[r].x;
    sm.Ai[kk][mm] = pa[r].y;
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int idx = tid + r * kTileThreads;
    int nn, kk;
    if (!TB) { nn = idx & 63; kk = idx >> 6; }
    else { kk = idx & 15; nn = idx >> 4; }
    sm.Br[kk][nn] = pb[r].x;
    sm.Bi[kk][nn] = pb[r].y;
  }
}

// acc += op(A)[m0:m0+64, :K] * diag(s) * op(B)[:K, n0:n0+64], where op(A) is
// M x K and op(B) is K x N; TA/TB select the transposed reading of a
// row-major operand.  Out-of-range elements read as zero.  The first
// kTileThreads threads of the CTA must all call this (it contains
// tile_barrier).
template <bool TA, bool TB, bool kL2 = false>
__device__ __forceinline__ void tile_mma(TileSmem& sm, cplx acc[4][4], const cplx* __restrict__ A, int lda,
                                         const cplx* __restrict__ B, int ldb, const cplx* __restrict__ s,
                                         int M, int N, int K, int m0, int n0) {
  if (K <= 0) return;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = 16 * (w & 3), wn = 32 * (w >> 2);
  cplx pa[4], pb[4];
  tile_fetch<TA, TB, kL2>(A, lda, B, ldb, s, M, N, K, m0, n0, 0, pa, pb);
  tile_stage<TA, TB>(sm, pa, pb);
  tile_barrier();
  for (int k0 = 0; k0 < K; k0 += kTBK) {
    const bool more = k0 + kTBK < K;
    if (more) tile_fetch<TA, TB, kL2>(A, lda, B, ldb, s, M, N, K, m0, n0, k0 + kTBK, pa, pb);
#pragma unroll
    for (int k4 = 0; k4 < kTBK; k4 += 4) {
      double ar[2], ai[2], an[2], br[4], bi[4];
#pragma unroll
      for (int rt = 0; rt < 2; ++rt) {
        ar[rt] = sm.Ar[k4 + t][wm + 8 * rt + g];
        ai[rt] = sm.Ai[k4 + t][wm + 8 * rt + g];
        an[rt] = -ai[rt];
      }
#pragma unroll
      for (int ct = 0; ct < 4; ++ct) {
        br[ct] = sm.Br[k4 + t][wn + 8 * ct + g];
        bi[ct] = sm.Bi[k4 + t][wn + 8 * ct + g];
      }
#pragma unroll
      for (int rt = 0; rt < 2; ++rt)
#pragma unroll
        for (int ct = 0; ct < 4; ++ct) {
          cplx& c0 = acc[2 * rt][ct];
          cplx& c1 = acc[2 * rt + 1][ct];
          dmma_8x8x4(c0.x, c1.x, ar[rt], br[ct]);
          dmma_8x8x4(c0.x, c1.x, an[rt], bi[ct]);
          dmma_8x8x4(c0.y, c1.y, ar[rt], bi[ct]);
          dmma_8x8x4(c0.y, c1.y, ai[rt], br[ct]);
        }
    }
    tile_barrier();
    if (more) {
      tile_stage<TA, TB>(sm, pa, pb);
      tile_barrier();
    }
  }
}

// D[m0.., n0..] = alpha*acc + beta*C + gammaI*(m == n)  (C may be null when
// beta is zero; C may alias D).
__device__ __forceinline__ void tile_store(const cplx acc[4][4], cplx* D, int ldd, const cplx* C, int ldc,
                                           cplx alpha, cplx beta, cplx gammaI, int M, int N, int m0, int n0) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = 16 * (w & 3), wn = 32 * (w >> 2);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + wm + 8 * (i >> 1) + g;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + wn + 8 * j + 2 * t + (i & 1);
      if (n >= N) continue;
      cplx v = cmul(alpha, acc[i][j]);
      if (C) v = cfma(beta, C[(size_t)m * ldc + n], v);
      if (m == n) v = cadd(v, gammaI);
      D[(size_t)m * ldd + n] = v;
    }
  }
}

static_assert(sizeof(cplx) * 32 * 33 <= sizeof(TileSmem), "32x32 triangular block must fit the tile buffer");
