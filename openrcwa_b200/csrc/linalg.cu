// Batched complex-FP64 GEMM, LU (getrf) and LU solve (getrs).
//
// GEMM: 64x64 output tiles, 256 threads, every thread owns a 4x4 block of
// complex accumulators in registers; operand tiles are staged in shared memory
// (K-slab of 16).  The same tile routine drives the trailing updates of the
// one-CTA-per-matrix blocked LU and of the blocked triangular solves, so the
// O(n^3) part of every factorisation runs as register-blocked FP64 FMAs.
#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>

#include <cooperative_groups.h>

#include "linalg.cuh"
#include "lu_blocked.cuh"
#include "tile.cuh"

namespace {

__global__ void __launch_bounds__(kTileThreads) zgemm_kernel(GemmArgs g) {
  __shared__ TileSmem sm;
  const int b = blockIdx.z;
  const cplx* A = (g.A ? g.A[b] : g.A0 + b * g.sA) + g.offA;
  const cplx* B = (g.B ? g.B[b] : g.B0 + b * g.sB) + g.offB;
  const cplx* s = g.s ? g.s[b] : nullptr;
  const int m0 = blockIdx.y * kTBM, n0 = blockIdx.x * kTBN;
  const int K = g.triB ? min(g.K, n0 + kTBN) : g.K;
  cplx acc[4][4];
  tile_zero(acc);
  if (g.transA) {
    if (g.transB) tile_mma<true, true>(sm, acc, A, g.lda, B, g.ldb, s, g.M, g.N, K, m0, n0);
    else tile_mma<true, false>(sm, acc, A, g.lda, B, g.ldb, s, g.M, g.N, K, m0, n0);
  } else {
    if (g.transB) tile_mma<false, true>(sm, acc, A, g.lda, B, g.ldb, s, g.M, g.N, K, m0, n0);
    else tile_mma<false, false>(sm, acc, A, g.lda, B, g.ldb, s, g.M, g.N, K, m0, n0);
  }
  const cplx* C = (g.beta.x != 0.0 || g.beta.y != 0.0) ? g.C[b] + g.offC : nullptr;
  tile_store(acc, (g.D ? g.D[b] : g.D0 + b * g.sD) + g.offD, g.ldd, C, g.ldc, g.alpha, g.beta, g.gammaI, g.M, g.N,
             m0, n0);
}

// Factorise panel columns kb .. kb+jb-1 of the n x n matrix A in place (rows
// kb .. n-1), LAPACK getf2 order: pivot = largest |re|+|im| in the column
// (first index on ties), the pivot rows are interchanged across all n columns,
// the column is scaled by the reciprocal pivot and the rest of the panel gets
// the rank-1 update.  The update reads the pivot row from shared memory and
// issues the loads of eight elements before their stores, so a thread keeps
// eight L2 requests in flight instead of one; it also tracks the largest
// entry of the next column, which is that column's pivot search.  Whole CTA;
// info keeps the first exactly-zero pivot.
__device__ void lu_panel(cplx* A, int n, int lda, int kb, int jb, int* ipiv, int& info, double* red_v, int* red_i,
                         int* s_piv, cplx* prow) {
  const int tid = threadIdx.x, nthr = blockDim.x;
  constexpr int kU = 8;
  double best = -1.0;
  int bi = kb;
  for (int i0 = kb + tid; i0 < n; i0 += kU * nthr) {
    double v[kU];
#pragma unroll
    for (int q = 0; q < kU; ++q) {
      const int i = i0 + q * nthr;
      v[q] = i < n ? cabs1(A[(size_t)i * lda + kb]) : -1.0;
    }
#pragma unroll
    for (int q = 0; q < kU; ++q)
      if (v[q] > best) { best = v[q]; bi = i0 + q * nthr; }
  }
  const int ce = kb + jb;  // panel end (exclusive)
  for (int j = kb; j < ce; ++j) {
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_down_sync(0xffffffffu, best, off);
      const int oi = __shfl_down_sync(0xffffffffu, bi, off);
      if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
    }
    if ((tid & 31) == 0) { red_v[tid >> 5] = best; red_i[tid >> 5] = bi; }
    __syncthreads();
    if (tid == 0) {
      double bv = red_v[0];
      int bix = red_i[0];
      for (int w = 1; w < nthr / 32; ++w)
        if (red_v[w] > bv || (red_v[w] == bv && red_i[w] < bix)) { bv = red_v[w]; bix = red_i[w]; }
      *s_piv = bix;
      ipiv[j] = bix;
    }
    __syncthreads();
    const int p = *s_piv;
    if (p != j) {
      for (int c = tid; c < n; c += nthr) {
        cplx t = A[(size_t)j * lda + c];
        A[(size_t)j * lda + c] = A[(size_t)p * lda + c];
        A[(size_t)p * lda + c] = t;
      }
    }
    __syncthreads();
    for (int c = j + tid; c < ce; c += nthr) prow[c - kb] = A[(size_t)j * lda + c];
    __syncthreads();
    const cplx piv = prow[j - kb];
    if (piv.x == 0.0 && piv.y == 0.0) {
      if (info == 0) info = j + 1;
    } else {
      const cplx inv = cdiv(mkc(1.0, 0.0), piv);
      for (int i0 = j + 1 + tid; i0 < n; i0 += kU * nthr) {
        cplx v[kU];
#pragma unroll
        for (int q = 0; q < kU; ++q) {
          const int i = i0 + q * nthr;
          if (i < n) v[q] = A[(size_t)i * lda + j];
        }
#pragma unroll
        for (int q = 0; q < kU; ++q) {
          const int i = i0 + q * nthr;
          if (i < n) A[(size_t)i * lda + j] = cmul(v[q], inv);
        }
      }
    }
    __syncthreads();
    best = -1.0;
    bi = j + 1;
    const int w = ce - j - 1;
    if (w > 0) {
      const int total = (n - j - 1) * w;
      for (int base = tid; base < total; base += kU * nthr) {
        cplx l[kU], a[kU];
#pragma unroll
        for (int q = 0; q < kU; ++q) {
          const int idx = base + q * nthr;
          if (idx < total) {
            const int i = j + 1 + idx / w, c = j + 1 + idx % w;
            l[q] = A[(size_t)i * lda + j];
            a[q] = A[(size_t)i * lda + c];
          }
        }
#pragma unroll
        for (int q = 0; q < kU; ++q) {
          const int idx = base + q * nthr;
          if (idx < total) {
            const int i = j + 1 + idx / w, c = j + 1 + idx % w;
            const cplx v = cfma(cneg(l[q]), prow[c - kb], a[q]);
            A[(size_t)i * lda + c] = v;
            if (c == j + 1) {
              const double av = cabs1(v);
              if (av > best) { best = av; bi = i; }
            }
          }
        }
      }
    }
    __syncthreads();
  }
}

// U12(:, c) = L11^-1 A12(:, c) for columns c = c0 + tid (L11 unit lower,
// jb x jb at (kb, kb), staged in Lsm); threads with c >= n idle.
__device__ void lu_trsm_cols(cplx* A, int n, int lda, int kb, int jb, int c, cplx (*Lsm)[33]) {
  if (c >= n) return;
  for (int r = 1; r < jb; ++r) {
    cplx x = A[(size_t)(kb + r) * lda + c];
    for (int q = 0; q < r; ++q) x = cfma(cneg(Lsm[r][q]), A[(size_t)(kb + q) * lda + c], x);
    A[(size_t)(kb + r) * lda + c] = x;
  }
}

// One CTA per matrix: right-looking blocked LU, panel width 32; the U12 block
// row by a shared-memory triangular solve and the trailing matrix by the
// register-blocked tile GEMM.
__global__ void __launch_bounds__(kTileThreads) zgetrf_kernel(cplx* const* Aarr, int n, int lda,
                                                             int* ipiv_all, int* info_all) {
  // the triangular block and the GEMM slabs are used in separate phases
  __shared__ __align__(16) unsigned char smem_raw[sizeof(TileSmem)];
  TileSmem& sm = *reinterpret_cast<TileSmem*>(smem_raw);
  cplx (*Lsm)[33] = reinterpret_cast<cplx (*)[33]>(smem_raw);
  __shared__ double red_v[kTileThreads / 32];
  __shared__ int red_i[kTileThreads / 32];
  __shared__ int s_piv;
  __shared__ cplx prow[32];
  const int tid = threadIdx.x;
  const int b = blockIdx.x;
  cplx* A = Aarr[b];
  int* ipiv = ipiv_all + (size_t)b * n;
  int info = 0;
  for (int kb = 0; kb < n; kb += 32) {
    const int jb = min(32, n - kb);
    lu_panel(A, n, lda, kb, jb, ipiv, info, red_v, red_i, &s_piv, prow);
    if (kb + jb < n) {
      for (int idx = tid; idx < jb * jb; idx += kTileThreads) {
        const int r = idx / jb, q = idx % jb;
        Lsm[r][q] = A[(size_t)(kb + r) * lda + kb + q];
      }
      __syncthreads();
      for (int c = kb + jb + tid; c < n; c += kTileThreads) lu_trsm_cols(A, n, lda, kb, jb, c, Lsm);
      __syncthreads();
      const int m2 = n - kb - jb;
      const int tiles_m = (m2 + kTBM - 1) / kTBM, tiles_n = (m2 + kTBN - 1) / kTBN;
      const cplx* L21 = A + (size_t)(kb + jb) * lda + kb;
      const cplx* U12 = A + (size_t)kb * lda + kb + jb;
      cplx* A22 = A + (size_t)(kb + jb) * lda + kb + jb;
      for (int t = 0; t < tiles_m * tiles_n; ++t) {
        const int tm = (t / tiles_n) * kTBM, tn = (t % tiles_n) * kTBN;
        cplx acc[4][4];
        tile_zero(acc);
        tile_mma<false, false>(sm, acc, L21, lda, U12, lda, nullptr, m2, m2, jb, tm, tn);
        tile_store(acc, A22, lda, A22, lda, mkc(-1.0, 0.0), mkc(1.0, 0.0), mkc(0.0, 0.0), m2, m2, tm, tn);
      }
      __syncthreads();
    }
  }
  if (tid == 0) info_all[b] = info;
}

// Panel width of the multi-launch LU, and the panel kernel's block size: a
// whole SM per panel keeps enough loads in flight for the rank-1 updates,
// whose rows come from L2.
constexpr int kLuPanel = 32;
constexpr int kLuPanelThreads = 512;

// Panel step of the multi-launch LU: one CTA per matrix factorises columns
// kb .. kb+jb-1 (the first panel also clears info).
__global__ void __launch_bounds__(kLuPanelThreads) getrf_panel_kernel(cplx* const* Aarr, int n, int lda, int kb,
                                                                     int jb, int* ipiv_all, int* info_all) {
  __shared__ double red_v[kLuPanelThreads / 32];
  __shared__ int red_i[kLuPanelThreads / 32];
  __shared__ int s_piv;
  __shared__ cplx prow[kLuPanel];
  const int b = blockIdx.x;
  int info = kb == 0 ? 0 : info_all[b];
  lu_panel(Aarr[b], n, lda, kb, jb, ipiv_all + (size_t)b * n, info, red_v, red_i, &s_piv, prow);
  if (threadIdx.x == 0) info_all[b] = info;
}

// Panel step of the multi-launch LU for few large matrices: a thread-block
// cluster of C CTAs per matrix shares the panel.  Rows kb..n-1 are split into
// C slices; per column every CTA finds the largest |re|+|im| of its slice
// (smallest row on ties), the CTAs read each other's candidates from shared
// memory (distributed shared memory of the cluster) and take the same pivot,
// swap their share of the columns of the two rows, and after a cluster
// barrier scale and update their own rows.  Every element gets the same
// operations as in lu_panel, so the factors are identical.
__global__ void __launch_bounds__(kLuPanelThreads) getrf_panel_team_kernel(cplx* const* Aarr, int n, int lda,
                                                                          int kb, int jb, int* ipiv_all,
                                                                          int* info_all) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  __shared__ double red_v[kLuPanelThreads / 32];
  __shared__ int red_i[kLuPanelThreads / 32];
  __shared__ double s_bv;  // this CTA's pivot candidate
  __shared__ int s_bi;
  __shared__ int s_piv;
  __shared__ cplx prow[kLuPanel];
  const int C = (int)cl.num_blocks(), rank = (int)cl.block_rank();
  const int b = blockIdx.x / C;
  const int tid = threadIdx.x, nthr = blockDim.x;
  constexpr int kU = 8;
  cplx* A = Aarr[b];
  int* ipiv = ipiv_all + (size_t)b * n;
  int info = kb == 0 ? 0 : __ldcg(info_all + b);
  const int per = (n - kb + C - 1) / C;
  const int lo = kb + rank * per, hi = min(n, lo + per);
  const int cper = (n + C - 1) / C;
  const int clo = rank * cper, chi = min(n, clo + cper);
  double best = -1.0;
  int bi = n;
  for (int i0 = max(lo, kb) + tid; i0 < hi; i0 += kU * nthr) {
    double v[kU];
#pragma unroll
    for (int q = 0; q < kU; ++q) {
      const int i = i0 + q * nthr;
      v[q] = i < hi ? cabs1(A[(size_t)i * lda + kb]) : -1.0;
    }
#pragma unroll
    for (int q = 0; q < kU; ++q)
      if (v[q] > best) { best = v[q]; bi = i0 + q * nthr; }
  }
  const int ce = kb + jb;
  for (int j = kb; j < ce; ++j) {
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_down_sync(0xffffffffu, best, off);
      const int oi = __shfl_down_sync(0xffffffffu, bi, off);
      if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
    }
    if ((tid & 31) == 0) { red_v[tid >> 5] = best; red_i[tid >> 5] = bi; }
    __syncthreads();
    if (tid == 0) {
      double bv = red_v[0];
      int bix = red_i[0];
      for (int w = 1; w < nthr / 32; ++w)
        if (red_v[w] > bv || (red_v[w] == bv && red_i[w] < bix)) { bv = red_v[w]; bix = red_i[w]; }
      s_bv = bv;
      s_bi = bix;
    }
    cl.sync();
    if (tid == 0) {
      double bv = -1.0;
      int bix = n;
      for (int r = 0; r < C; ++r) {
        const double v = *cl.map_shared_rank(&s_bv, r);
        const int ix = *cl.map_shared_rank(&s_bi, r);
        if (v > bv || (v == bv && ix < bix)) { bv = v; bix = ix; }
      }
      // a column of zeros below the diagonal keeps its row (lu_panel's
      // candidate is row j then)
      s_piv = bix < n ? bix : j;
      if (rank == 0) ipiv[j] = s_piv;
    }
    __syncthreads();
    const int p = s_piv;
    if (p != j) {
      for (int c = clo + tid; c < chi; c += nthr) {
        cplx t = A[(size_t)j * lda + c];
        A[(size_t)j * lda + c] = A[(size_t)p * lda + c];
        A[(size_t)p * lda + c] = t;
      }
    }
    // the swap is complete everywhere, and every CTA has read the candidates
    cl.sync();
    for (int c = j + tid; c < ce; c += nthr) prow[c - kb] = __ldcg(A + (size_t)j * lda + c);
    __syncthreads();
    const cplx piv = prow[j - kb];
    const int r0 = max(lo, j + 1);
    if (piv.x == 0.0 && piv.y == 0.0) {
      if (info == 0) info = j + 1;
    } else {
      const cplx inv = cdiv(mkc(1.0, 0.0), piv);
      for (int i0 = r0 + tid; i0 < hi; i0 += kU * nthr) {
        cplx v[kU];
#pragma unroll
        for (int q = 0; q < kU; ++q) {
          const int i = i0 + q * nthr;
          if (i < hi) v[q] = A[(size_t)i * lda + j];
        }
#pragma unroll
        for (int q = 0; q < kU; ++q) {
          const int i = i0 + q * nthr;
          if (i < hi) A[(size_t)i * lda + j] = cmul(v[q], inv);
        }
      }
    }
    __syncthreads();
    best = -1.0;
    bi = n;
    const int w = ce - j - 1;
    if (w > 0 && r0 < hi) {
      const int total = (hi - r0) * w;
      for (int base = tid; base < total; base += kU * nthr) {
        cplx l[kU], a[kU];
#pragma unroll
        for (int q = 0; q < kU; ++q) {
          const int idx = base + q * nthr;
          if (idx < total) {
            const int i = r0 + idx / w, c = j + 1 + idx % w;
            l[q] = A[(size_t)i * lda + j];
            a[q] = A[(size_t)i * lda + c];
          }
        }
#pragma unroll
        for (int q = 0; q < kU; ++q) {
          const int idx = base + q * nthr;
          if (idx < total) {
            const int i = r0 + idx / w, c = j + 1 + idx % w;
            const cplx v = cfma(cneg(l[q]), prow[c - kb], a[q]);
            A[(size_t)i * lda + c] = v;
            if (c == j + 1) {
              const double av = cabs1(v);
              if (av > best || (av == best && i < bi)) { best = av; bi = i; }
            }
          }
        }
      }
    }
    __syncthreads();
  }
  if (rank == 0 && tid == 0) info_all[b] = info;
  // no CTA leaves while another may still read its candidate
  cl.sync();
}

// U12 of the multi-launch LU: one CTA per (matrix, 64 columns right of the
// panel, up to column ce), a thread per column; the unit lower L11 (jb <=
// kLuPanel) is read through the read-only path (every thread reads the same
// entry).
__global__ void __launch_bounds__(64) getrf_trsm_kernel(cplx* const* Aarr, int lda, int kb, int jb, int ce) {
  cplx* A = Aarr[blockIdx.y];
  const int c = kb + jb + blockIdx.x * 64 + threadIdx.x;
  if (c >= ce) return;
  for (int r = 1; r < jb; ++r) {
    cplx x = A[(size_t)(kb + r) * lda + c];
    const cplx* Lr = A + (size_t)(kb + r) * lda + kb;
    for (int q = 0; q < r; ++q) x = cfma(cneg(__ldg(&Lr[q])), A[(size_t)(kb + q) * lda + c], x);
    A[(size_t)(kb + r) * lda + c] = x;
  }
}

// Blocked LU solve, left-looking: one CTA per (matrix, 64-column slab of B).
// Each 64-row block of the slab first takes the contribution of all rows
// already solved as one long-K tile GEMM (L(rb:, :rb) X(:rb) forward,
// U(rb:, re:) X(re:) backward), then its diagonal block is solved in two
// 32-row halves, one thread per column with the column in registers.
__device__ __forceinline__ void load_block32(cplx (*Tsm)[33], const cplx* LU, int lda, int r0, int c0, int h, int w) {
  for (int idx = threadIdx.x; idx < h * w; idx += blockDim.x) {
    const int r = idx / w, q = idx % w;
    Tsm[r][q] = LU[(size_t)(r0 + r) * lda + c0 + q];
  }
}

// kInv (the inverse, LAPACK getri order): B starts as the identity without
// the row interchanges, so column c of L^-1 is zero above row c and the
// forward pass of the slab starting at column c0 begins at row c0 with its
// long-K products cut to K = c0 .. rb; the column interchanges follow in
// zcolperm_kernel.  This saves a third of the flops of solving against P.
template <bool kInv>
__global__ void __launch_bounds__(kTileThreads) zgetrs_kernel(const cplx* const* LUarr, int n, int lda,
                                                             const int* ipiv_all, cplx* const* Barr,
                                                             int nrhs, int ldb) {
  __shared__ __align__(16) unsigned char smem_raw[sizeof(TileSmem)];
  TileSmem& sm = *reinterpret_cast<TileSmem*>(smem_raw);
  cplx (*Tsm)[33] = reinterpret_cast<cplx (*)[33]>(smem_raw);
  const int tid = threadIdx.x;
  const int b = blockIdx.y;
  const int c0 = blockIdx.x * 64;
  const int cw = min(64, nrhs - c0);
  const cplx* LU = LUarr[b];
  const int* ipiv = ipiv_all + (size_t)b * n;
  cplx* B = Barr[b] + c0;
  if (kInv) {
    for (int idx = tid; idx < n * cw; idx += blockDim.x) {
      const int r = idx / cw, c = idx % cw;
      B[(size_t)r * ldb + c] = mkc(r == c0 + c ? 1.0 : 0.0, 0.0);
    }
  } else if (tid < cw) {
    for (int j = 0; j < n; ++j) {
      const int p = ipiv[j];
      if (p != j) {
        cplx t = B[(size_t)j * ldb + tid];
        B[(size_t)j * ldb + tid] = B[(size_t)p * ldb + tid];
        B[(size_t)p * ldb + tid] = t;
      }
    }
  }
  __syncthreads();
  // forward substitution with the unit lower factor (rows below k0 of the
  // slab are zero for the inverse)
  const int k0 = kInv ? c0 : 0;
  for (int rb = k0; rb < n; rb += 64) {
    const int rw = min(64, n - rb);
    if (rb > k0) {
      cplx acc[4][4];
      tile_zero(acc);
      tile_mma<false, false>(sm, acc, LU + (size_t)rb * lda + k0, lda, B + (size_t)k0 * ldb, ldb, nullptr, rw, cw,
                             rb - k0, 0, 0);
      tile_store(acc, B + (size_t)rb * ldb, ldb, B + (size_t)rb * ldb, ldb, mkc(-1.0, 0.0), mkc(1.0, 0.0),
                 mkc(0.0, 0.0), rw, cw, 0, 0);
      __syncthreads();
    }
    for (int h0 = rb; h0 < rb + rw; h0 += 32) {
      const int hw = min(32, rb + rw - h0);
      if (h0 > rb) {
        // the first half of the block feeds the second
        load_block32(Tsm, LU, lda, h0, rb, hw, 32);
        __syncthreads();
        if (tid < cw) {
          cplx x[32];
#pragma unroll
          for (int q = 0; q < 32; ++q) x[q] = B[(size_t)(rb + q) * ldb + tid];
          for (int r = 0; r < hw; ++r) {
            cplx acc = B[(size_t)(h0 + r) * ldb + tid];
#pragma unroll
            for (int q = 0; q < 32; ++q) acc = cfma(cneg(Tsm[r][q]), x[q], acc);
            B[(size_t)(h0 + r) * ldb + tid] = acc;
          }
        }
        __syncthreads();
      }
      load_block32(Tsm, LU, lda, h0, h0, hw, hw);
      __syncthreads();
      if (tid < cw) {
        // the column's solved entries are re-read from L1
        for (int r = 1; r < hw; ++r) {
          cplx acc = B[(size_t)(h0 + r) * ldb + tid];
          for (int q = 0; q < r; ++q) acc = cfma(cneg(Tsm[r][q]), B[(size_t)(h0 + q) * ldb + tid], acc);
          B[(size_t)(h0 + r) * ldb + tid] = acc;
        }
      }
      __syncthreads();
    }
  }
  // back substitution with the upper factor
  for (int rb = ((n - 1) / 64) * 64; rb >= 0; rb -= 64) {
    const int re = min(n, rb + 64), rw = re - rb;
    if (re < n) {
      cplx acc[4][4];
      tile_zero(acc);
      tile_mma<false, false>(sm, acc, LU + (size_t)rb * lda + re, lda, B + (size_t)re * ldb, ldb, nullptr, rw, cw,
                             n - re, 0, 0);
      tile_store(acc, B + (size_t)rb * ldb, ldb, B + (size_t)rb * ldb, ldb, mkc(-1.0, 0.0), mkc(1.0, 0.0),
                 mkc(0.0, 0.0), rw, cw, 0, 0);
      __syncthreads();
    }
    for (int h0 = (rw > 32) ? rb + 32 : rb; h0 >= rb; h0 -= 32) {
      const int hw = min(32, re - h0);
      const int tail = re - h0 - hw;  // rows of this block below the half, already solved
      if (tail > 0) {
        load_block32(Tsm, LU, lda, h0, h0 + hw, hw, tail);
        __syncthreads();
        if (tid < cw) {
          cplx x[32];
#pragma unroll
          for (int q = 0; q < 32; ++q) x[q] = q < tail ? B[(size_t)(h0 + hw + q) * ldb + tid] : mkc(0.0, 0.0);
          for (int r = 0; r < hw; ++r) {
            cplx acc = B[(size_t)(h0 + r) * ldb + tid];
#pragma unroll
            for (int q = 0; q < 32; ++q)
              if (q < tail) acc = cfma(cneg(Tsm[r][q]), x[q], acc);
            B[(size_t)(h0 + r) * ldb + tid] = acc;
          }
        }
        __syncthreads();
      }
      load_block32(Tsm, LU, lda, h0, h0, hw, hw);
      __syncthreads();
      if (tid < cw) {
        for (int r = hw - 1; r >= 0; --r) {
          cplx acc = B[(size_t)(h0 + r) * ldb + tid];
          for (int q = r + 1; q < hw; ++q) acc = cfma(cneg(Tsm[r][q]), B[(size_t)(h0 + q) * ldb + tid], acc);
          B[(size_t)(h0 + r) * ldb + tid] = cdiv(acc, Tsm[r][r]);
        }
      }
      __syncthreads();
    }
  }
}

// X <- X P for the column interchanges of getrf (ipiv, applied from the
// last to the first as LAPACK getri does): rows of X pass through shared
// memory, `rows` per CTA; the permutation is rebuilt per CTA from ipiv.
__global__ void zcolperm_kernel(cplx* const* Xarr, int n, int ldx, const int* ipiv_all, int rows) {
  extern __shared__ __align__(16) unsigned char dsm[];
  int* perm = reinterpret_cast<int*>(dsm);
  cplx* buf = reinterpret_cast<cplx*>(dsm + (((size_t)n * sizeof(int) + 15) & ~(size_t)15));
  const int b = blockIdx.y, r0 = blockIdx.x * rows;
  const int* ipiv = ipiv_all + (size_t)b * n;
  cplx* X = Xarr[b];
  const int rw = min(rows, n - r0);
  for (int c = threadIdx.x; c < n; c += blockDim.x) perm[c] = c;
  for (int idx = threadIdx.x; idx < rw * n; idx += blockDim.x)
    buf[idx] = X[(size_t)(r0 + idx / n) * ldx + idx % n];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int j = n - 1; j >= 0; --j) {
      const int p = ipiv[j];
      if (p != j) { const int t = perm[j]; perm[j] = perm[p]; perm[p] = t; }
    }
  __syncthreads();
  for (int idx = threadIdx.x; idx < rw * n; idx += blockDim.x) {
    const int r = idx / n, c = idx % n;
    X[(size_t)(r0 + r) * ldx + c] = buf[(size_t)r * n + perm[c]];
  }
}

__global__ void identity_kernel(cplx* const* Barr, int n, int ldb) {
  cplx* B = Barr[blockIdx.y];
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < (size_t)n * n;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx / n), c = (int)(idx % n);
    B[(size_t)r * ldb + c] = mkc(r == c ? 1.0 : 0.0, 0.0);
  }
}

__global__ void copy_kernel(const cplx* const* S, int lds, cplx* const* Dd, int ldd, int rows, int cols) {
  const cplx* s = S[blockIdx.y];
  cplx* d = Dd[blockIdx.y];
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < (size_t)rows * cols;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx / cols), c = (int)(idx % cols);
    d[(size_t)r * ldd + c] = s[(size_t)r * lds + c];
  }
}

}  // namespace

cudaError_t zgemm_batched(const GemmArgs& g, cudaStream_t st) {
  if (g.batch <= 0 || g.M <= 0 || g.N <= 0) return cudaSuccess;
  dim3 grid((g.N + kTBN - 1) / kTBN, (g.M + kTBM - 1) / kTBM, g.batch);
  zgemm_kernel<<<grid, kTileThreads, 0, st>>>(g);
  ++launch_counter();
  return cudaGetLastError();
}

namespace {
int sm_count() {
  static int count = 0;
  if (!count) {
    int dev = 0, c = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) ==
                                                  cudaSuccess && c > 0)
      count = c;
    else
      return 148;
  }
  return count;
}
}  // namespace

namespace {
// CTAs per matrix of the multi-launch LU's panel step (0: automatic), set by
// rcwa_set_lu_cluster.
std::atomic<int> g_lu_team{0};
constexpr int kLuTeamMinN = 1024;

int lu_team_size(int n, int batch) {
  const int forced = g_lu_team.load();
  if (forced > 0) return forced;
  const int sms = sm_count();
  if (n < kLuTeamMinN || 2 * batch > sms) return 1;
  static std::mutex mu;
  static std::map<int, int> cache;  // batch -> size
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(batch);
  if (it != cache.end()) return it->second;
  int pick = 1;
  for (int c = std::min(8, sms / batch); c >= 2; --c) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c);
    cfg.blockDim = dim3(kLuPanelThreads);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = c;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nc = 0;
    if (cudaOccupancyMaxActiveClusters(&nc, (void*)getrf_panel_team_kernel, &cfg) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (nc >= batch) {
      pick = c;
      break;
    }
  }
  cache[batch] = pick;
  return pick;
}

cudaError_t launch_panel(cplx* const* A, int n, int lda, int kb, int jb, int* ipiv, int* info, int batch, int team,
                         cudaStream_t st) {
  if (team <= 1) {
    getrf_panel_kernel<<<batch, kLuPanelThreads, 0, st>>>(A, n, lda, kb, jb, ipiv, info);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(batch * team);
  cfg.blockDim = dim3(kLuPanelThreads);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = team;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, getrf_panel_team_kernel, A, n, lda, kb, jb, ipiv, info);
}
}  // namespace

extern "C" int rcwa_set_lu_cluster(int ctas) {
  if (ctas < 0 || ctas > 8) return RCWA_ERR_INVALID;
  g_lu_team.store(ctas);
  return RCWA_OK;
}

extern "C" int rcwa_lu_cluster_size(int n, int batch) {
  if (batch <= 0 || n <= 0) return 1;
  return lu_team_size(n, batch);
}

int zgetrf_default_schedule(int n, int batch, int sms) {
  if (sms <= 0) sms = sm_count();
  // 128-column blocks from n = 256 on (measured on B200 at n = 882: 148
  // matrices 41.9 -> 32.4 ms, 296 matrices 74.0 -> 57.5 ms against panel by panel)
  if (n <= 128 || batch >= 4 * sms) return 0;
  return n >= 256 ? 2 : 1;
}

cudaError_t zgetrf_batched(cplx* const* A, int n, int lda, int* ipiv, int* info, int batch,
                           cudaStream_t st, int schedule) {
  if (batch <= 0 || n <= 0) return cudaSuccess;
  if (schedule < 0) schedule = zgetrf_default_schedule(n, batch);
  if (schedule == 0) {
    zgetrf_kernel<<<batch, kTileThreads, 0, st>>>(A, n, lda, ipiv, info);
    ++launch_counter();
    return cudaGetLastError();
  }
  if (schedule == 2) return zgetrf_blocked_batched(A, n, lda, ipiv, info, batch, nullptr, st);
  return zgetrf_columns(A, n, lda, 0, n, ipiv, info, batch, st);
}

cudaError_t zgetrf_columns(cplx* const* A, int n, int lda, int k0, int ce, int* ipiv, int* info, int batch,
                           cudaStream_t st) {
  if (batch <= 0 || k0 < 0 || ce > n || k0 >= ce) return cudaErrorInvalidValue;
  // a cluster of CTAs per matrix shares each panel when the batch leaves SMs idle
  const int team = lu_team_size(n, batch);
  for (int kb = k0; kb < ce; kb += kLuPanel) {
    const int jb = min(kLuPanel, ce - kb);
    cudaError_t pe = launch_panel(A, n, lda, kb, jb, ipiv, info, batch, team, st);
    if (pe != cudaSuccess) return pe;
    ++launch_counter();
    const int m2 = n - kb - jb, w = ce - kb - jb;
    if (m2 <= 0 || w <= 0) break;
    getrf_trsm_kernel<<<dim3((w + 63) / 64, batch), 64, 0, st>>>(A, lda, kb, jb, ce);
    ++launch_counter();
    // A22 -= L21 U12 (the block's columns)
    GemmArgs g{};
    g.A = A; g.B = A; g.C = A; g.D = A;
    g.offA = (size_t)(kb + jb) * lda + kb;
    g.offB = (size_t)kb * lda + kb + jb;
    g.offC = g.offD = (size_t)(kb + jb) * lda + kb + jb;
    g.M = m2; g.N = w; g.K = jb;
    g.lda = g.ldb = g.ldc = g.ldd = lda;
    g.alpha = mkc(-1.0, 0.0); g.beta = mkc(1.0, 0.0); g.gammaI = mkc(0.0, 0.0);
    g.batch = batch;
    cudaError_t err = zgemm_batched(g, st);
    if (err != cudaSuccess) return err;
  }
  return cudaGetLastError();
}

// From this order on, solves with at least 64 right-hand sides run blocked
// (lu_blocked.cu: 128-row triangles plus batched GEMM updates over the whole
// grid) instead of one CTA per 64-column slab; a build parameter.
#ifndef RCWA_BLOCKED_SOLVE_MIN_N
#define RCWA_BLOCKED_SOLVE_MIN_N 256
#endif
constexpr int kBlockedSolveMinN = RCWA_BLOCKED_SOLVE_MIN_N;

cudaError_t zgetrs_batched(const cplx* const* LU, int n, int lda, const int* ipiv, cplx* const* B,
                           int nrhs, int ldb, int batch, cudaStream_t st) {
  if (batch <= 0 || n <= 0 || nrhs <= 0) return cudaSuccess;
  if (n >= kBlockedSolveMinN && nrhs >= 64)
    return zgetrs_blocked_batched(LU, n, lda, ipiv, B, nrhs, ldb, batch, false, nullptr, st);
  dim3 grid((nrhs + 63) / 64, batch);
  zgetrs_kernel<false><<<grid, kTileThreads, 0, st>>>(LU, n, lda, ipiv, B, nrhs, ldb);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t zgetri_batched(const cplx* const* LU, int n, int lda, const int* ipiv, cplx* const* X, int ldx,
                           int batch, cudaStream_t st) {
  if (batch <= 0 || n <= 0) return cudaSuccess;
  if (n >= kBlockedSolveMinN) return zgetrs_blocked_batched(LU, n, lda, ipiv, X, n, ldx, batch, true, nullptr, st);
  dim3 grid((n + 63) / 64, batch);
  zgetrs_kernel<true><<<grid, kTileThreads, 0, st>>>(LU, n, lda, ipiv, X, n, ldx);
  ++launch_counter();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return zcolperm_batched(X, n, ldx, ipiv, batch, st);
}

cudaError_t zcolperm_batched(cplx* const* X, int n, int ldx, const int* ipiv, int batch, cudaStream_t st) {
  cudaError_t e;
  // rows per CTA: as many as fit in 64 KB next to the permutation
  const size_t perm_bytes = ((size_t)n * sizeof(int) + 15) & ~(size_t)15;
  const int rows = (int)std::max<size_t>(1, std::min<size_t>(8, (64u << 10) / ((size_t)n * sizeof(cplx))));
  const size_t smem = perm_bytes + (size_t)rows * n * sizeof(cplx);
  if (smem > (size_t)(227u << 10)) return cudaErrorInvalidValue;
  static SmemAttrOnce attr;
  if ((e = attr.ensure(zcolperm_kernel, (int)(227u << 10))) != cudaSuccess) return e;
  zcolperm_kernel<<<dim3((n + rows - 1) / rows, batch), 256, smem, st>>>(X, n, ldx, ipiv, rows);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t zset_identity_batched(cplx* const* B, int n, int ldb, int batch, cudaStream_t st) {
  if (batch <= 0 || n <= 0) return cudaSuccess;
  dim3 grid(min(1024, (n * n + 255) / 256), batch);
  identity_kernel<<<grid, 256, 0, st>>>(B, n, ldb);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t zcopy_batched(const cplx* const* src, int lds, cplx* const* dst, int ldd, int rows, int cols,
                          int batch, cudaStream_t st) {
  if (batch <= 0 || rows <= 0 || cols <= 0) return cudaSuccess;
  dim3 grid(min(1024, (rows * cols + 255) / 256), batch);
  copy_kernel<<<grid, 256, 0, st>>>(src, lds, dst, ldd, rows, cols);
  ++launch_counter();
  return cudaGetLastError();
}
