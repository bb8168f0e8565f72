// Batched complex eigensolver, one CTA per matrix, FP64 throughout:
//   1. Householder reduction to upper Hessenberg form, Q accumulated backwards;
//   2. single-shift complex QR iteration (Wilkinson shifts, exceptional shifts
//      every 10 sweeps, Ahues-Tisseur deflation test) producing the Schur form
//      T with Schur vectors Z.  The bulge is chased by one warp inside a
//      32 x 32 window held in shared memory; the window's rotations are then
//      applied to the rest of T and to Z by the whole CTA, each thread
//      streaming one row or column through the whole rotation sequence;
//   3. eigenvectors of T by back-substitution (protected small divisors),
//      back-transformed with Z by the tile GEMM and normalised to unit 2-norm.
// This replaces LAPACK zgeev('N','V') behind MKLEigenSolver
// (rcwa/MKLEigenSolver.hpp:102-179).  Balancing is not applied.
#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>

#include "eig.cuh"
#include "linalg.cuh"
#include "tile.cuh"

namespace {

constexpr int kEigThreads = kTileThreads;  // 256
constexpr int kWin = 32;
constexpr int kItsPerEig = 300;

constexpr int kHb = kEigPanel;

__host__ __device__ inline size_t workspace_bytes(int n) { return zgeev_workspace_bytes(n); }

struct Scratch {
  cplx* Z;     // n*n, column-major: Z(r, c) = Z[c*n + r]
  cplx* X;     // n*n, row-major upper-triangular eigenvector matrix of T
  cplx* v;     // n: current Householder vector / work column
  cplx* wv;    // n
  cplx* uv;    // n
  cplx* v0;    // n: leading element of each stored reflector
  cplx* Vb;    // n x kHb  panel reflectors, explicit (row-major)
  cplx* VH;    // kHb x n  their conjugate transposes (or n x kHb conj(V))
  cplx* Yb;    // n x kHb  A V T  (also kHb x n work)
  cplx* Wb;    // kHb x n  (also n x kHb work)
  cplx* Vt;    // kHb x n  V^T (first kHb x kHb: T^H / T^T)
  cplx* Tall;  // (ceil(n/kHb)+1) x kHb x kHb  triangular factors of all panels
  double* tau; // n
};

#ifdef RCWA_EIG_STATS
// counters: 0 ms sweeps, 1 ss sweeps, 2 passes, 3 chase cycles, 4 replay cycles, 5 window-Schur cycles,
// 6 reordering and re-Hessenberg cycles, 7 early-deflation update cycles, 8 early-deflation cycles,
// 9 single-shift cycles, 10 Schur cycles, 11 early deflations, 12 deflated by them
__device__ unsigned long long g_eig_stats[32];
#define STAT_ADD(i, v) do { if (threadIdx.x == 0) atomicAdd(&g_eig_stats[i], (unsigned long long)(v)); } while (0)
#else
#define STAT_ADD(i, v) do { } while (0)
#endif

__device__ Scratch scratch_for(void* work, int n, int b) {
  const size_t nn = (size_t)n * n;
  const size_t nk = (size_t)n * kHb;
  char* base = (char*)work + (size_t)b * workspace_bytes(n);
  Scratch s;
  s.Z = (cplx*)base;
  s.X = s.Z + nn;
  s.v = s.X + nn;
  s.wv = s.v + n;
  s.uv = s.wv + n;
  s.v0 = s.uv + n;
  s.Vb = s.v0 + n;
  s.VH = s.Vb + nk;
  s.Yb = s.VH + nk;
  s.Wb = s.Yb + nk;
  s.Vt = s.Wb + nk;
  s.Tall = s.Vt + (size_t)(n > kHb ? n : kHb) * kHb;
  s.tau = (double*)(s.Tall + ((size_t)(n + kHb - 1) / kHb + 1) * kHb * kHb);
  return s;
}

// The CTAs that work on one matrix: a thread-block cluster of `size` CTAs
// (size 1: the CTA alone).  sync() is the cluster barrier, whose release and
// acquire make every CTA's global writes before it visible to all CTAs of the
// cluster after it; a lone CTA uses __syncthreads.  Every thread of every
// CTA of the team must reach each sync().
struct Team {
  int rank, size;
  __device__ void sync() const {
    if (size > 1) {
      asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
      asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
    } else {
      __syncthreads();
    }
  }
};

__device__ __forceinline__ Team cluster_team() {
  unsigned r, s;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  asm volatile("mov.u32 %0, %%cluster_nctarank;\n" : "=r"(s));
  return Team{(int)r, (int)s};
}

__device__ double block_sum(double v, double* red) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  return t;
}


__device__ int block_max_int(int v, int* red) {
  for (int off = 16; off > 0; off >>= 1) v = max(v, __shfl_down_sync(0xffffffffu, v, off));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  int t = red[0];
  for (int w = 1; w < (int)(blockDim.x >> 5); ++w) t = max(t, red[w]);
  return t;
}


// In-CTA GEMM over 64x64 tiles: D = alpha*op(A)*op(B) + beta*C (C may alias D).
// A CTA of a team takes the tiles t = rank, rank + size, ...; kL2 loads the
// operands from L2 (they may come from other CTAs of the team).
template <bool TA, bool TB, bool kL2 = false>
__device__ void cta_gemm(TileSmem& sm, int M, int N, int K, const cplx* A, int lda, const cplx* B, int ldb,
                         cplx* D, int ldd, const cplx* C, int ldc, cplx alpha, cplx beta, int rank = 0,
                         int size = 1) {
  if (M <= 0 || N <= 0) return;
  const int tm = (M + kTBM - 1) / kTBM, tn = (N + kTBN - 1) / kTBN;
  for (int t = rank; t < tm * tn; t += size) {
    const int m0 = (t / tn) * kTBM, n0 = (t % tn) * kTBN;
    cplx acc[4][4];
    tile_zero(acc);
    if (K > 0) tile_mma<TA, TB, kL2>(sm, acc, A, lda, B, ldb, nullptr, M, N, K, m0, n0);
    tile_store(acc, D, ldd, C, ldc, alpha, beta, mkc(0.0, 0.0), M, N, m0, n0);
  }
  tile_barrier();
}

// cta_gemm by the first kTileThreads threads of every CTA of a team (the
// Hessenberg kernel runs more warps than the tile routines use), the tiles
// split over the team, then a barrier over the team.
template <bool TA, bool TB, bool kTeam>
__device__ void cta_gemm_part(const Team& tm, TileSmem& sm, int M, int N, int K, const cplx* A, int lda,
                              const cplx* B, int ldb, cplx* D, int ldd, const cplx* C, int ldc, cplx alpha,
                              cplx beta) {
  if (threadIdx.x < kTileThreads) {
    if (kTeam)
      cta_gemm<TA, TB, true>(sm, M, N, K, A, lda, B, ldb, D, ldd, C, ldc, alpha, beta, tm.rank, tm.size);
    else
      cta_gemm<TA, TB>(sm, M, N, K, A, lda, B, ldb, D, ldd, C, ldc, alpha, beta);
  }
  tm.sync();
}

// Blocked Householder reduction to Hessenberg form in compact WY form, the
// scheme of LAPACK's gehrd/lahr2 (Quintana-Orti and van de Geijn, ACM TOMS
// 32(2), 2006).  For panel columns k..k+jb-1 the reflectors are generated one
// column at a time from A0 (the matrix at the panel start) corrected by
// Y = A0 V T; each column needs one product A0(:, j+1:) v_j, the only O(n^2)
// memory traffic per column.  The trailing matrix is then updated by
// A <- (I - V T^H V^H)(A - Y V^H) with tile GEMMs, and Q = prod(I - V T V^H)
// is formed backwards with tile GEMMs.  Reflectors H = I - tau v v^H are
// Hermitian with real tau; column j stores beta at (j+1, j) and the tail of
// v_j below it, v_j(j+1) = v0[j].
// A team of several CTAs (a cluster) shares the work of one matrix: the
// first CTA forms each reflector, every CTA then takes a slice of the rows of
// A0 v_j and Y, and the tiles of every GEMM are split over the team.  Each
// element is computed by the same operations as with one CTA, so the result
// does not depend on the team size.  kTeam: compiled for teams of more than
// one CTA (operands of the tile GEMMs then come from L2).
template <bool kTeam>
__device__ void hessenberg_blocked(cplx* A, int n, int lda, const Scratch& s, double* red, TileSmem& tsm,
                                   const Team& tm) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  const int nb = kHb;
  const bool lead = tm.rank == 0;
  // this CTA's rows of the matrix-vector products (an even split point)
  const int per = ((n + tm.size - 1) / tm.size + 1) & ~1;
  const int r0 = min(n, tm.rank * per), r1 = min(n, r0 + per);
  cplx* a = s.v;    // work column, then v_j
  __shared__ cplx z[2 * kHb];
  cplx* u = s.uv;   // n
  // the panel's reflectors V and Y = A0 V T column-major (column q at q*n),
  // so that every sweep over the rows is coalesced
  cplx* Vc = s.Vb;
  cplx* Yc = s.Yb;
  // v_j in shared memory during the panel (aliases the tile buffer)
  cplx* vs = reinterpret_cast<cplx*>(&tsm);
  const bool vs_ok = (size_t)n * sizeof(cplx) <= sizeof(TileSmem);
  for (int k = 0; k + 2 < n; k += nb) {
#ifdef RCWA_EIG_STATS
    const long long c_p0 = clock64();
#endif
    const int jb = min(nb, n - 2 - k);
    cplx* T = s.Tall + (size_t)(k / nb) * nb * nb;
    if (lead)
      for (int idx = tid; idx < nb * nb; idx += blockDim.x) T[idx] = mkc(0.0, 0.0);
    for (int jj = 0; jj < jb; ++jj) {
      const int j = k + jj;
#ifdef RCWA_EIG_STATS
      long long h_t = clock64();
#define HMARK(i) do { if (tid == 0 && lead) { const long long t_ = clock64(); atomicAdd(&g_eig_stats[i], (unsigned long long)(t_ - h_t)); h_t = t_; } } while (0)
#else
#define HMARK(i) do {} while (0)
#endif
      double tau = 0.0;
      if (lead) {
        // a = A0(:, j) - Y(:, :jj) conj(V(j, :jj))
        for (int i = tid; i < n; i += blockDim.x) {
          cplx acc = A[(size_t)i * lda + j];
          for (int q = 0; q < jj; ++q) acc = cfma(cneg(Yc[(size_t)q * n + i]), cconj(Vc[(size_t)q * n + j]), acc);
          a[i] = acc;
        }
        __syncthreads();
        HMARK(16);
        if (jj > 0) {
          // a(k+1:) <- (I - V T^H V^H) a(k+1:):  z = V^H a, z = T^H z, a -= V z
          for (int q = wid; q < jj; q += nw) {
            cplx acc = mkc(0.0, 0.0);
            for (int i = k + 1 + q + lane; i < n; i += 32) acc = cfmaconj(Vc[(size_t)q * n + i], a[i], acc);
            for (int off = 16; off > 0; off >>= 1) {
              acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
              acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
            }
            if (lane == 0) z[q] = acc;
          }
          __syncthreads();
          if (tid < jj) {
            cplx acc = mkc(0.0, 0.0);
            for (int q = 0; q <= tid; ++q) acc = cfmaconj(T[q * nb + tid], z[q], acc);  // (T^H z)_tid
            z[nb + tid] = acc;
          }
          __syncthreads();
          for (int i = k + 1 + tid; i < n; i += blockDim.x) {
            cplx acc = a[i];
            for (int q = 0; q < jj; ++q) acc = cfma(cneg(Vc[(size_t)q * n + i]), z[nb + q], acc);
            a[i] = acc;
          }
          __syncthreads();
        }
        HMARK(17);
        // reflector from a(j+1:)
        double sig = 0.0;
        for (int i = j + 2 + tid; i < n; i += blockDim.x) sig += cnorm2(a[i]);
        sig = block_sum(sig, red);
        const cplx alpha = a[j + 1];
        cplx beta = alpha, v0 = mkc(1.0, 0.0);
        if (sig != 0.0) {
          const double aa = cabs(alpha);
          const double xnorm = sqrt(aa * aa + sig);
          const cplx ph = aa > 0.0 ? cscale(alpha, 1.0 / aa) : mkc(1.0, 0.0);
          beta = cscale(ph, -xnorm);
          v0 = cscale(ph, aa + xnorm);
          tau = 2.0 / (cnorm2(v0) + sig);
        }
        // column j of the result; explicit v_j in V(:, jj) and V^H(jj, :),
        // and in shared memory for the matrix-vector product (the tile
        // buffer is free during the panel)
        for (int i = tid; i < n; i += blockDim.x) {
          cplx vi = mkc(0.0, 0.0);
          if (i <= j) A[(size_t)i * lda + j] = a[i];
          else if (i == j + 1) { A[(size_t)i * lda + j] = beta; vi = v0; }
          else { A[(size_t)i * lda + j] = a[i]; vi = a[i]; }
          if (tau == 0.0) vi = mkc(0.0, 0.0);
          Vc[(size_t)jj * n + i] = vi;
          s.VH[(size_t)jj * n + i] = cconj(vi);
          a[i] = vi;
          if (vs_ok) vs[i] = vi;
        }
        if (tid == 0) { s.tau[j] = tau; s.v0[j] = v0; }
      }
      tm.sync();
      if (!lead) {
        // the other CTAs of the team take v_j and tau from the first
        tau = __ldcg(s.tau + j);
        if (vs_ok) {
          for (int i = tid; i < n; i += blockDim.x) vs[i] = __ldcg(a + i);
          __syncthreads();
        }
      }
      HMARK(18);
      // u = A0(:, j+1:) v_j (one pass over the trailing columns), z = V(:, :jj)^H v_j.
      // The pass is bound by the loads in flight (the trailing matrix mostly
      // comes from L2): a warp takes two rows at a time and issues all eight
      // loads of a 128-column step at once, predicated at the row end rather
      // than finished by a serial tail loop; v_j comes from shared memory.
      const cplx* vj = vs_ok ? vs : a;
      for (int i0 = r0 + 2 * wid; i0 < r1; i0 += 2 * nw) {
        const bool two = i0 + 1 < r1;
        const cplx* row0 = A + (size_t)i0 * lda;
        const cplx* row1 = two ? row0 + lda : row0;
        cplx acc0 = mkc(0.0, 0.0), acc1 = mkc(0.0, 0.0);
        for (int c = j + 1 + lane; c < n; c += 128) {
          cplx r0v[4], r1v[4], w[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int cc = c + 32 * q;
            const bool in = cc < n;
            r0v[q] = in ? row0[cc] : mkc(0.0, 0.0);
            r1v[q] = in ? row1[cc] : mkc(0.0, 0.0);
            w[q] = in ? vj[cc] : mkc(0.0, 0.0);
          }
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            acc0 = cfma(r0v[q], w[q], acc0);
            acc1 = cfma(r1v[q], w[q], acc1);
          }
        }
        for (int off = 16; off > 0; off >>= 1) {
          acc0.x += __shfl_xor_sync(0xffffffffu, acc0.x, off);
          acc0.y += __shfl_xor_sync(0xffffffffu, acc0.y, off);
          acc1.x += __shfl_xor_sync(0xffffffffu, acc1.x, off);
          acc1.y += __shfl_xor_sync(0xffffffffu, acc1.y, off);
        }
        if (lane == 0) {
          u[i0] = acc0;
          if (two) u[i0 + 1] = acc1;
        }
      }
      HMARK(19);
      for (int q = wid; q < jj; q += nw) {
        cplx acc = mkc(0.0, 0.0);
        for (int i = j + 1 + lane; i < n; i += 32) acc = cfmaconj(Vc[(size_t)q * n + i], Vc[(size_t)jj * n + i], acc);
        for (int off = 16; off > 0; off >>= 1) {
          acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
          acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
        }
        if (lane == 0) z[q] = acc;
      }
      __syncthreads();
      HMARK(20);
      // Y(:, jj) = tau (u - Y(:, :jj) z); T(:jj, jj) = -tau T(:jj, :jj) z; T(jj, jj) = tau
      for (int i = r0 + tid; i < r1; i += blockDim.x) {
        cplx acc = u[i];
        for (int q = 0; q < jj; ++q) acc = cfma(cneg(Yc[(size_t)q * n + i]), z[q], acc);
        Yc[(size_t)jj * n + i] = cscale(acc, tau);
      }
      if (lead) {
        if (tid < jj) {
          cplx acc = mkc(0.0, 0.0);
          for (int q = tid; q < jj; ++q) acc = cfma(T[tid * nb + q], z[q], acc);
          T[tid * nb + jj] = cscale(acc, -tau);
        }
        if (tid == 0) T[jj * nb + jj] = mkc(tau, 0.0);
      }
      tm.sync();
      HMARK(21);
#undef HMARK
    }
#ifdef RCWA_EIG_STATS
    const long long c_p1 = clock64();
    if (lead) STAT_ADD(13, c_p1 - c_p0);
#endif
    // trailing columns c0..n-1
    const int c0 = k + jb;
    const int m2 = n - c0;
    if (m2 > 0) {
      // A(:, c0:) -= Y V(c0:, :)^H
      cta_gemm_part<true, false, kTeam>(tm, tsm, n, m2, jb, Yc, n, s.VH + c0, n, A + c0, lda, A + c0, lda,
                                        mkc(-1.0, 0.0), mkc(1.0, 0.0));
      // W = V(k+1:, :)^H A(k+1:, c0:)  (jb x m2), W2 = T^H W, A(k+1:, c0:) -= V(k+1:, :) W2
      cta_gemm_part<false, false, kTeam>(tm, tsm, jb, m2, n - k - 1, s.VH + k + 1, n,
                                         A + (size_t)(k + 1) * lda + c0, lda, s.Wb + c0, n, nullptr, 0,
                                         mkc(1.0, 0.0), mkc(0.0, 0.0));
      if (lead)
        for (int idx = tid; idx < nb * nb; idx += blockDim.x) {
          const int r = idx / nb, c = idx % nb;
          s.Vt[idx] = (r < jb && c < jb) ? cconj(T[c * nb + r]) : mkc(0.0, 0.0);  // T^H in Vt
        }
      tm.sync();
      cta_gemm_part<false, false, kTeam>(tm, tsm, jb, m2, jb, s.Vt, nb, s.Wb + c0, n, s.Yb + c0, n, nullptr, 0,
                                         mkc(1.0, 0.0), mkc(0.0, 0.0));
      cta_gemm_part<true, false, kTeam>(tm, tsm, n - k - 1, m2, jb, Vc + k + 1, n, s.Yb + c0, n,
                                        A + (size_t)(k + 1) * lda + c0, lda, A + (size_t)(k + 1) * lda + c0, lda,
                                        mkc(-1.0, 0.0), mkc(1.0, 0.0));
    }
#ifdef RCWA_EIG_STATS
    if (lead) STAT_ADD(14, clock64() - c_p1);
#endif
  }
#ifdef RCWA_EIG_STATS
  const long long c_q0 = clock64();
#endif
  // Z (column-major, i.e. Zt = Z^T row-major) = Q, accumulated backwards:
  // Zt(k+1:, k+1:) -= (Zt conj(V)) T^T V^T
  for (size_t idx = (size_t)r0 * n + tid; idx < (size_t)r1 * n; idx += blockDim.x)
    s.Z[idx] = mkc((idx / n) == (idx % n) ? 1.0 : 0.0, 0.0);
  tm.sync();
  const int npan = (n >= 3) ? (n - 3) / nb + 1 : 0;
  for (int pnl = npan - 1; pnl >= 0; --pnl) {
    const int k = pnl * nb;
    const int jb = min(nb, n - 2 - k);
    const cplx* T = s.Tall + (size_t)pnl * nb * nb;
    // conj(V) (n x nb, in Wb) and V^T (nb x n, in VH) from the stored reflectors
    for (int i = r0 + tid; i < r1; i += blockDim.x) {
      for (int q = 0; q < nb; ++q) {
        const int j = k + q;
        cplx vi = mkc(0.0, 0.0);
        if (q < jb && s.tau[j] != 0.0) {
          if (i == j + 1) vi = s.v0[j];
          else if (i > j + 1) vi = A[(size_t)i * lda + j];
        }
        s.Wb[(size_t)i * nb + q] = cconj(vi);
        s.VH[(size_t)q * n + i] = vi;
      }
    }
    if (lead)
      for (int idx = tid; idx < nb * nb; idx += blockDim.x) {
        const int r = idx / nb, c = idx % nb;
        s.Vt[idx] = T[c * nb + r];  // T^T
      }
    tm.sync();
    const int m = n - k - 1;
    cplx* Zs = s.Z + (size_t)(k + 1) * n + (k + 1);
    cta_gemm_part<false, false, kTeam>(tm, tsm, m, jb, m, Zs, n, s.Wb + (size_t)(k + 1) * nb, nb, s.Yb, nb,
                                       nullptr, 0, mkc(1.0, 0.0), mkc(0.0, 0.0));
    cta_gemm_part<false, false, kTeam>(tm, tsm, m, jb, jb, s.Yb, nb, s.Vt, nb, s.Vb, nb, nullptr, 0,
                                       mkc(1.0, 0.0), mkc(0.0, 0.0));
    cta_gemm_part<false, false, kTeam>(tm, tsm, m, m, jb, s.Vb, nb, s.VH + k + 1, n, Zs, n, Zs, n,
                                       mkc(-1.0, 0.0), mkc(1.0, 0.0));
  }
  for (size_t idx = (size_t)r0 * n + tid; idx < (size_t)r1 * n; idx += blockDim.x) {
    const int i = (int)(idx / n), j = (int)(idx % n);
    if (i > j + 1) A[(size_t)i * lda + j] = mkc(0.0, 0.0);
  }
  tm.sync();
#ifdef RCWA_EIG_STATS
  if (lead) STAT_ADD(15, clock64() - c_q0);
#endif
}

// ---------------------------------------------------------------- QR
// Rotation [c s; -conj(s) c] (c real) with G [x; y] = [r; 0], evaluated
// with two reciprocal square roots after scaling both inputs by a power of
// two: c = |x| / |(x, y)|, s = x conj(y) / (|x| |(x, y)|).
__device__ __forceinline__ void givens_fast(cplx x, cplx y, double& c, cplx& s) {
  const double m = fmax(fmax(fabs(x.x), fabs(x.y)), fmax(fabs(y.x), fabs(y.y)));
  if (m == 0.0 || (y.x == 0.0 && y.y == 0.0)) { c = 1.0; s = mkc(0.0, 0.0); return; }
  int e;
  frexp(m, &e);
  const double sc = ldexp(1.0, -e);
  x = cscale(x, sc);
  y = cscale(y, sc);
  const double ax2 = cnorm2(x), ay2 = cnorm2(y);
  if (ax2 == 0.0) { c = 0.0; s = mkc(1.0, 0.0); return; }
  const double ra = rsqrt(ax2), rr = rsqrt(ax2 + ay2);
  c = ax2 * ra * rr;
  s = cscale(cmul(x, cconj(y)), ra * rr);
}

// Negligible subdiagonal T(k,k-1) inside the active block [l, i]:
// the standard relative test refined by the criterion of Ahues and Tisseur
// (LAPACK Working Note 122, 1997).
__device__ bool negligible(const cplx* T, int ldt, int k, int l, int i, double ulp, double smlnum) {
  const cplx h = T[(size_t)k * ldt + k - 1];
  const double ah = cabs1(h);
  if (ah <= smlnum) return true;
  const cplx hkk = T[(size_t)k * ldt + k], hk1 = T[(size_t)(k - 1) * ldt + k - 1];
  double tst = cabs1(hk1) + cabs1(hkk);
  if (tst == 0.0) {
    if (k - 2 >= l) tst += cabs1(T[(size_t)(k - 1) * ldt + k - 2]);
    if (k + 1 <= i) tst += cabs1(T[(size_t)(k + 1) * ldt + k]);
  }
  if (ah <= ulp * tst) {
    const double up = cabs1(T[(size_t)(k - 1) * ldt + k]);
    const double ab = fmax(ah, up), ba = fmin(ah, up);
    const double d1 = cabs1(hkk), d2 = cabs1(csub(hk1, hkk));
    const double aa = fmax(d1, d2), bb = fmin(d1, d2);
    const double sc = aa + ab;
    if (ba * (ab / sc) <= fmax(smlnum, ulp * (bb * (aa / sc)))) return true;
  }
  return false;
}

// Eigenvalue of the trailing 2x2 [[a, b], [c, d]] closest to d:
// d - b*c / (delta + r), delta = (a - d)/2, r = sqrt(delta^2 + b*c) taken on
// the side of delta so that the denominator does not cancel.
__device__ cplx wilkinson_shift(cplx a, cplx b, cplx c, cplx d) {
  const cplx bc = cmul(b, c);
  const double sbc = cabs1(bc);
  if (sbc == 0.0) return d;
  const cplx delta = cscale(csub(a, d), 0.5);
  const double sc = fmax(cabs1(delta), sqrt(sbc));
  const cplx ds = cscale(delta, 1.0 / sc);
  cplx r = csqrt_principal(cadd(cmul(ds, ds), cscale(bc, 1.0 / (sc * sc))));
  r = cscale(r, sc);
  if (delta.x * r.x + delta.y * r.y < 0.0) r = cneg(r);
  const cplx den = cadd(delta, r);
  if (den.x == 0.0 && den.y == 0.0) return d;
  return csub(d, cdiv(bc, den));
}

__device__ void qr_sweep(cplx* T, int ldt, cplx* Z, int n, int l, int i, cplx shift,
                         cplx (*Wt)[kWin + 1], double* rc, cplx* rs) {
  const int tid = threadIdx.x;
  int k = l, ws = l;
  while (k <= i - 1) {
    const int we = min(ws + kWin - 1, i);
    const int ke = (we == i) ? i - 1 : we - 2;
    const int w = we - ws + 1;
    for (int idx = tid; idx < w * w; idx += blockDim.x)
      Wt[idx / w][idx % w] = T[(size_t)(ws + idx / w) * ldt + ws + idx % w];
    __syncthreads();
    if (tid < 32) {
      const int lane = tid;
      for (int r = k; r <= ke; ++r) {
        cplx x, y;
        if (r == l) {
          x = csub(Wt[r - ws][r - ws], shift);
          y = Wt[r + 1 - ws][r - ws];
        } else {
          x = Wt[r - ws][r - 1 - ws];
          y = Wt[r + 1 - ws][r - 1 - ws];
        }
        double c;
        cplx sn;
        givens_fast(x, y, c, sn);
        const int j0 = (r == l) ? r : r - 1;
        const int jj = j0 - ws + lane;
        if (jj < w) {
          const cplx a = Wt[r - ws][jj], b = Wt[r + 1 - ws][jj];
          Wt[r - ws][jj] = cfma(sn, b, cscale(a, c));
          Wt[r + 1 - ws][jj] = cfma(cneg(cconj(sn)), a, cscale(b, c));
        }
        __syncwarp();
        if (lane == 0 && r > l) Wt[r + 1 - ws][r - 1 - ws] = mkc(0.0, 0.0);
        const int iend = min(r + 2, i) - ws;
        if (lane <= iend) {
          const cplx a = Wt[lane][r - ws], b = Wt[lane][r + 1 - ws];
          Wt[lane][r - ws] = cfma(cconj(sn), b, cscale(a, c));
          Wt[lane][r + 1 - ws] = cfma(cneg(sn), a, cscale(b, c));
        }
        __syncwarp();
        if (lane == 0) { rc[r - k] = c; rs[r - k] = sn; }
      }
    }
    __syncthreads();
    for (int idx = tid; idx < w * w; idx += blockDim.x)
      T[(size_t)(ws + idx / w) * ldt + ws + idx % w] = Wt[idx / w][idx % w];
    // deferred application of rotations k..ke outside the window
    const int nrot = ke - k + 1;
    const int nright = n - 1 - we;
    const int nup = ws;
    const int ntask = nright + nup + n;
    for (int t = tid; t < ntask; t += blockDim.x) {
      if (t < nright) {
        const int j = we + 1 + t;
        cplx x = T[(size_t)k * ldt + j];
        for (int q = 0; q < nrot; ++q) {
          const cplx y = T[(size_t)(k + q + 1) * ldt + j];
          const double c = rc[q];
          const cplx sn = rs[q];
          T[(size_t)(k + q) * ldt + j] = cfma(sn, y, cscale(x, c));
          x = cfma(cneg(cconj(sn)), x, cscale(y, c));
        }
        T[(size_t)(k + nrot) * ldt + j] = x;
      } else if (t < nright + nup) {
        const int ii = t - nright;
        cplx* row = T + (size_t)ii * ldt;
        cplx x = row[k];
        for (int q = 0; q < nrot; ++q) {
          const cplx y = row[k + q + 1];
          const double c = rc[q];
          const cplx sn = rs[q];
          row[k + q] = cfma(cconj(sn), y, cscale(x, c));
          x = cfma(cneg(sn), x, cscale(y, c));
        }
        row[k + nrot] = x;
      } else {
        const int ii = t - nright - nup;
        cplx x = Z[(size_t)k * n + ii];
        for (int q = 0; q < nrot; ++q) {
          const cplx y = Z[(size_t)(k + q + 1) * n + ii];
          const double c = rc[q];
          const cplx sn = rs[q];
          Z[(size_t)(k + q) * n + ii] = cfma(cconj(sn), y, cscale(x, c));
          x = cfma(cneg(sn), x, cscale(y, c));
        }
        Z[(size_t)(k + nrot) * n + ii] = x;
      }
    }
    __syncthreads();
    ws = ke;
    k = ke + 1;
  }
}

// Returns 0 or RCWA_ERR_NOCONV.
__device__ int schur(cplx* T, int ldt, cplx* Z, int n, cplx (*Wt)[kWin + 1], double* rc, cplx* rs,
                     int* redi, int sweep_cap) {
  const double ulp = 2.0 * RCWA_DBL_EPS;
  const double smlnum = RCWA_DBL_MIN * ((double)n / ulp);
  int i = n - 1;
  long long total = 0;
  const long long itmax_total = sweep_cap > 0 ? min(30LL * max(10, n), (long long)sweep_cap) : 30LL * max(10, n);
  while (i >= 0) {
    int l = 0;
    bool conv = false;
    for (int its = 0; its <= kItsPerEig; ++its) {
      int best = l;
      for (int k = l + 1 + threadIdx.x; k <= i; k += blockDim.x)
        if (negligible(T, ldt, k, l, i, ulp, smlnum)) best = max(best, k);
      l = block_max_int(best, redi);
      if (l > 0 && threadIdx.x == 0) T[(size_t)l * ldt + l - 1] = mkc(0.0, 0.0);
      __syncthreads();
      if (l >= i) { conv = true; break; }
      cplx shift;
      if (its == 10 || its == 30) {
        shift = cadd(T[(size_t)l * ldt + l], mkc(0.75 * cabs1(T[(size_t)(l + 1) * ldt + l]), 0.0));
      } else if (its == 20 || its == 40) {
        shift = cadd(T[(size_t)i * ldt + i], mkc(0.75 * cabs1(T[(size_t)i * ldt + i - 1]), 0.0));
      } else {
        shift = wilkinson_shift(T[(size_t)(i - 1) * ldt + i - 1], T[(size_t)(i - 1) * ldt + i],
                                T[(size_t)i * ldt + i - 1], T[(size_t)i * ldt + i]);
      }
      __syncthreads();
      qr_sweep(T, ldt, Z, n, l, i, shift, Wt, rc, rs);
      if (++total > itmax_total) break;
    }
    if (!conv) return RCWA_ERR_NOCONV;
    i = l - 1;
  }
  return 0;
}


// ---------------------------------------------------------------- multishift QR
// Small-bulge multishift QR (the scheme of Braman, Byers and Mathias, SIAM J.
// Matrix Anal. Appl. 23(4), 2002) for complex Hessenberg matrices.  A sweep
// chases a chain of s single-shift bulges, three rows apart, from the top to
// the bottom of the active block.  The chain advances inside a 64 x 64 window
// held in shared memory, all bulges of one chain step in parallel (their row
// pairs and column pairs are disjoint).  Every rotation is logged; after a
// window pass the log is applied to the rest of T (the rows right of the
// window, the columns above it) and to Z, one line of 32 per warp task, with
// the part of each line the chain spans held in registers (replay_frame), so
// an element of T or Z crosses memory once per pass instead of once per
// rotation.
#ifndef RCWA_MS_WINDOW
#define RCWA_MS_WINDOW 64
#endif
constexpr int kMsW = RCWA_MS_WINDOW;  // window order (a build-time parameter)
#ifndef RCWA_MS_SHIFTS
#define RCWA_MS_SHIFTS 10
#endif
constexpr int kMsShifts = RCWA_MS_SHIFTS;  // bulges per sweep (a build-time parameter)
constexpr int kMsMin = kSchurCrossover;  // smallest crossover: the chase window needs 64 rows
constexpr int kMsThreads = 256;    // eight warps
constexpr int kMsLog = kMsW + 1;         // rotation log per bulge; slot kMsW holds the identity
constexpr int kMsMaxSteps = kMsW + 3 * kMsShifts;  // chain steps of one window pass

struct MsSmem {
  cplx* Wt;      // [kMsW][kMsW + 1]  the chase window
  cplx* work;    // early deflation's window, vectors and reflector; the small shift problem
  double* lc;    // [kMsShifts][kMsLog]  rotation cosines, bulge-major
  cplx* ls;      // [kMsShifts][kMsLog]  rotation sines
  int* ix;       // [kMsMaxSteps][kMsShifts]  log slot per chain step and bulge
  int* firstp;   // [kMsShifts] first rotation position of each bulge in the pass
  int* cnt;      // [kMsShifts] rotations of each bulge in the pass
  int* tfirst;   // [kMsShifts] pass step of each bulge's first rotation
  cplx* shifts;  // [kMsShifts]
  int* redi;     // [kMsThreads / 32]
  int* aed;      // [4] early-deflation results: converged flag, undeflated count, shift count
};

// the window is only used by the chase, the work area only by the early
// deflation and the shift computation between sweeps: they share one region
constexpr size_t kMsRegion = sizeof(cplx) * kMsW * (kMsW + 1);
constexpr size_t kMsSmemBytes = kMsRegion +
                                sizeof(double) * kMsShifts * kMsLog + sizeof(cplx) * kMsShifts * kMsLog +
                                sizeof(int) * kMsMaxSteps * kMsShifts + sizeof(int) * 3 * kMsShifts +
                                sizeof(cplx) * kMsShifts + sizeof(int) * (kMsThreads / 32 + 4);
static_assert(kMsSmemBytes <= 232448, "multishift shared memory exceeds the per-block limit");

__device__ MsSmem carve_ms_smem(unsigned char* base) {
  MsSmem sm;
  sm.Wt = (cplx*)base;
  sm.work = (cplx*)base;
  sm.ls = (cplx*)(base + kMsRegion);
  sm.shifts = sm.ls + kMsShifts * kMsLog;
  sm.lc = (double*)(sm.shifts + kMsShifts);
  sm.ix = (int*)(sm.lc + kMsShifts * kMsLog);
  sm.firstp = sm.ix + kMsMaxSteps * kMsShifts;
  sm.cnt = sm.firstp + kMsShifts;
  sm.tfirst = sm.cnt + kMsShifts;
  sm.redi = sm.tfirst + kMsShifts;
  sm.aed = sm.redi + kMsThreads / 32;
  return sm;
}

#define MSW(r, c) sm.Wt[(r) * (kMsW + 1) + (c)]

// Eigenvalues of the s x s upper Hessenberg matrix B (row stride ldb) by
// single-shift QR without vectors; one warp.  Unconverged remainders after
// the iteration budget are returned as their diagonal entries.
__device__ void small_eigs_warp(cplx* B, int ldb, int s, cplx* out) {
  const int lane = threadIdx.x & 31;
  const double ulp = 2.0 * RCWA_DBL_EPS;
  int hi = s - 1, its = 0;
  while (hi >= 0) {
    int lo = 0;
    for (int k = hi; k >= 1; --k) {
      const double h = cabs1(B[k * ldb + k - 1]);
      if (h <= ulp * (cabs1(B[(k - 1) * ldb + k - 1]) + cabs1(B[k * ldb + k])) || h < RCWA_DBL_MIN) {
        lo = k;
        break;
      }
    }
    if (lo == hi || its > 60) {
      for (int k = lo + lane; k <= hi; k += 32) out[k] = B[k * ldb + k];
      __syncwarp();
      hi = lo - 1;
      its = 0;
      continue;
    }
    cplx sh;
    if (its == 10 || its == 20) sh = cadd(B[hi * ldb + hi], mkc(0.75 * cabs1(B[hi * ldb + hi - 1]), 0.0));
    else sh = wilkinson_shift(B[(hi - 1) * ldb + hi - 1], B[(hi - 1) * ldb + hi], B[hi * ldb + hi - 1], B[hi * ldb + hi]);
    for (int r = lo; r < hi; ++r) {
      cplx x, y;
      if (r == lo) { x = csub(B[lo * ldb + lo], sh); y = B[(lo + 1) * ldb + lo]; }
      else { x = B[r * ldb + r - 1]; y = B[(r + 1) * ldb + r - 1]; }
      double c;
      cplx sn;
      givens_fast(x, y, c, sn);
      __syncwarp();
      const int j = ((r == lo) ? r : r - 1) + lane;
      if (j <= hi) {
        const cplx a = B[r * ldb + j], b = B[(r + 1) * ldb + j];
        B[r * ldb + j] = cfma(sn, b, cscale(a, c));
        B[(r + 1) * ldb + j] = cfma(cneg(cconj(sn)), a, cscale(b, c));
      }
      __syncwarp();
      if (r > lo && lane == 0) B[(r + 1) * ldb + r - 1] = mkc(0.0, 0.0);
      const int row = lo + lane;
      if (row <= min(r + 2, hi)) {
        const cplx a = B[row * ldb + r], b = B[row * ldb + r + 1];
        B[row * ldb + r] = cfma(cconj(sn), b, cscale(a, c));
        B[row * ldb + r + 1] = cfma(cneg(sn), a, cscale(b, c));
      }
      __syncwarp();
    }
    ++its;
  }
}

// ---------------------------------------------------------------- aggressive early deflation
// Aggressive early deflation (Braman, Byers and Mathias, SIAM J. Matrix Anal.
// Appl. 23(4), 2002; the complex variant of LAPACK's zlaqr3): the trailing
// kAedW x kAedW window of the active block is brought to Schur form with its
// unitary V; the spike s*conj(V(0,:)) that couples it to the rest tells which
// window eigenvalues have converged.  Converged ones at the bottom are
// deflated, the others are moved to the top by adjacent swaps and serve as
// shifts; the spike of the undeflated part is reflected onto its first entry
// and that part is returned to Hessenberg form by Householder reflectors.
// Measured on the cfg2 FP64 step (740 matrices of 882): Schur 2488 / 2286 /
// 2251 / 2228 / 2260 / 2251 ms with windows of 32 / 20 / 18 / 16 / 14 / 12
// (a smaller window's cheaper one-warp Schur against its fewer deflations);
// with 16, 8 and 12 shifts per sweep gave 2271 and 2231 ms against 2228.
#ifndef RCWA_AED_WINDOW
#define RCWA_AED_WINDOW 16
#endif
constexpr int kAedW = RCWA_AED_WINDOW;  // window order (one lane per column; a build-time parameter)
static_assert(kAedW <= 32 && kAedW >= kMsShifts + 2, "the early-deflation window is one warp wide");
constexpr int kAedLd = kAedW + 1;
constexpr int kAedNibble = 14;   // percent of the window deflated that skips the sweep
static_assert(sizeof(cplx) * (2 * kAedW * kAedLd + kAedW) <= kMsRegion &&
                  sizeof(cplx) * kMsShifts * (kMsShifts + 1) <= kMsRegion,
              "the early-deflation work area must fit in the chase window's region");

#define AW(r, c) W[(r) * kAedLd + (c)]
#define AV(r, c) V[(r) * kAedLd + (c)]

// Schur form of the Hessenberg window W (nw x nw) with V <- V G^H for every
// rotation G; single-shift QR by one warp.  Returns false when the iteration
// budget runs out.
__device__ bool aed_window_schur(cplx* W, cplx* V, int nw) {
  const int lane = threadIdx.x & 31;
  const double ulp = 2.0 * RCWA_DBL_EPS;
  int hi = nw - 1, its = 0, total = 0;
  while (hi >= 0) {
    __syncwarp();
    bool defl = false;
    if (lane >= 1 && lane <= hi) {
      const double h = cabs1(AW(lane, lane - 1));
      defl = h <= ulp * (cabs1(AW(lane - 1, lane - 1)) + cabs1(AW(lane, lane))) || h < RCWA_DBL_MIN;
    }
    const unsigned mask = __ballot_sync(0xffffffffu, defl);
    const int lo = mask ? 31 - __clz(mask) : 0;
    __syncwarp();
    if (lo == hi) {
      if (hi > 0 && lane == 0) AW(hi, hi - 1) = mkc(0.0, 0.0);
      --hi;
      its = 0;
      continue;
    }
    if (lo > 0 && lane == 0) AW(lo, lo - 1) = mkc(0.0, 0.0);
    if (++total > 30 * nw) return false;
    cplx sh;
    if (its == 10) sh = cadd(AW(lo, lo), mkc(0.75 * cabs1(AW(lo + 1, lo)), 0.0));
    else if (its == 20) sh = cadd(AW(hi, hi), mkc(0.75 * cabs1(AW(hi, hi - 1)), 0.0));
    else sh = wilkinson_shift(AW(hi - 1, hi - 1), AW(hi - 1, hi), AW(hi, hi - 1), AW(hi, hi));
    __syncwarp();
    for (int p = lo; p < hi; ++p) {
      cplx x, y;
      if (p == lo) { x = csub(AW(lo, lo), sh); y = AW(lo + 1, lo); }
      else { x = AW(p, p - 1); y = AW(p + 1, p - 1); }
      double c;
      cplx sn;
      givens_fast(x, y, c, sn);
      __syncwarp();
      if (lane >= (p == lo ? p : p - 1) && lane < nw) {
        const cplx a = AW(p, lane), b = AW(p + 1, lane);
        AW(p, lane) = cfma(sn, b, cscale(a, c));
        AW(p + 1, lane) = cfma(cneg(cconj(sn)), a, cscale(b, c));
      }
      __syncwarp();
      if (p > lo && lane == 0) AW(p + 1, p - 1) = mkc(0.0, 0.0);
      if (lane <= min(p + 2, hi)) {
        const cplx a = AW(lane, p), b = AW(lane, p + 1);
        AW(lane, p) = cfma(cconj(sn), b, cscale(a, c));
        AW(lane, p + 1) = cfma(cneg(sn), a, cscale(b, c));
      }
      if (lane < nw) {
        const cplx a = AV(lane, p), b = AV(lane, p + 1);
        AV(lane, p) = cfma(cconj(sn), b, cscale(a, c));
        AV(lane, p + 1) = cfma(cneg(sn), a, cscale(b, c));
      }
      __syncwarp();
    }
    ++its;
  }
  __syncwarp();
  return true;
}

// Swap the adjacent eigenvalues k, k+1 of the upper triangular W (LAPACK
// ztrexc step): G from (W(k,k+1), W(k+1,k+1) - W(k,k)) applied to rows
// k, k+1 right of the pair, to columns k, k+1 above it and to V; the
// diagonal entries trade places and W(k,k+1) keeps its value.  One warp.
__device__ void aed_swap(cplx* W, cplx* V, int nw, int k) {
  const int lane = threadIdx.x & 31;
  const cplx t11 = AW(k, k), t22 = AW(k + 1, k + 1);
  double c;
  cplx sn;
  givens_fast(AW(k, k + 1), csub(t22, t11), c, sn);
  __syncwarp();
  if (lane >= k + 2 && lane < nw) {
    const cplx a = AW(k, lane), b = AW(k + 1, lane);
    AW(k, lane) = cfma(sn, b, cscale(a, c));
    AW(k + 1, lane) = cfma(cneg(cconj(sn)), a, cscale(b, c));
  }
  if (lane < k) {
    const cplx a = AW(lane, k), b = AW(lane, k + 1);
    AW(lane, k) = cfma(cconj(sn), b, cscale(a, c));
    AW(lane, k + 1) = cfma(cneg(sn), a, cscale(b, c));
  }
  if (lane < nw) {
    const cplx a = AV(lane, k), b = AV(lane, k + 1);
    AV(lane, k) = cfma(cconj(sn), b, cscale(a, c));
    AV(lane, k + 1) = cfma(cneg(sn), a, cscale(b, c));
  }
  if (lane == 0) { AW(k, k) = t22; AW(k + 1, k + 1) = t11; }
  __syncwarp();
}

// Householder reflector H = I - tau v v^H with H^H x = beta e1 for the
// vector x[0..len) in shared memory (LAPACK zlarfg convention: v[0] = 1,
// tau = (beta - alpha)/beta, beta = -sign(Re alpha) ||x||); v overwrites x.
// One warp; returns tau (zero when x is already beta e1).
__device__ cplx aed_house(cplx* x, int len) {
  const int lane = threadIdx.x & 31;
  double part = (lane >= 1 && lane < len) ? cnorm2(x[lane]) : 0.0;
  for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(0xffffffffu, part, off);
  const cplx alpha = x[0];
  __syncwarp();
  if (part == 0.0 && alpha.y == 0.0) return mkc(0.0, 0.0);
  const double beta = -copysign(sqrt(cnorm2(alpha) + part), alpha.x);
  const cplx tau = mkc((beta - alpha.x) / beta, -alpha.y / beta);
  const cplx scal = cdiv(mkc(1.0, 0.0), csub(alpha, mkc(beta, 0.0)));
  if (lane >= 1 && lane < len) x[lane] = cmul(x[lane], scal);
  if (lane == 0) x[0] = mkc(beta, 0.0);  // beta kept in x[0]; v[0] = 1 implied
  __syncwarp();
  return tau;
}

// M(r0 + r, c) -= conj(tau) v[r] (v^H M(r0.., c)) for columns c in [c0, nw):
// the left product H^H M on rows r0 .. r0+len-1; v[0] = 1.  One warp.
__device__ void aed_left(cplx* M, const cplx* v, int len, cplx tau, int r0, int c0, int nw) {
  const int lane = threadIdx.x & 31;
  if (lane >= c0 && lane < nw) {
    cplx w = M[r0 * kAedLd + lane];
    for (int r = 1; r < len; ++r) w = cfmaconj(v[r], M[(r0 + r) * kAedLd + lane], w);
    const cplx f = cmul(cconj(tau), w);
    M[r0 * kAedLd + lane] = csub(M[r0 * kAedLd + lane], f);
    for (int r = 1; r < len; ++r) M[(r0 + r) * kAedLd + lane] = csub(M[(r0 + r) * kAedLd + lane], cmul(v[r], f));
  }
  __syncwarp();
}

// M(r, c0 + c) -= tau (M(r, c0..) v) conj(v[c]) for rows r < rows: the right
// product M H on columns c0 .. c0+len-1; v[0] = 1.  One warp.
__device__ void aed_right(cplx* M, const cplx* v, int len, cplx tau, int rows, int c0) {
  const int lane = threadIdx.x & 31;
  if (lane < rows) {
    cplx w = M[lane * kAedLd + c0];
    for (int c = 1; c < len; ++c) w = cfma(M[lane * kAedLd + c0 + c], v[c], w);
    const cplx f = cmul(tau, w);
    M[lane * kAedLd + c0] = csub(M[lane * kAedLd + c0], f);
    for (int c = 1; c < len; ++c)
      M[lane * kAedLd + c0 + c] = csub(M[lane * kAedLd + c0 + c], cmul(f, cconj(v[c])));
  }
  __syncwarp();
}

// Aggressive early deflation on the active block [l, i] (i - l + 1 > kAedW + 1).
// Returns the number of deflated eigenvalues (0 when none, -1 when the window
// did not converge and nothing was changed).  On return sm.shifts[0..cnt)
// hold the bottom undeflated window eigenvalues, cnt <= kMsShifts, in
// sm.aed[2].  Whole CTA.
// With a team of several CTAs every CTA computes the window's Schur form
// (the same operations on the same data), the first CTA's outcome is taken
// by all (ctrl[2..4]), the first CTA writes the window back and the
// off-window updates are split over the team.  *shift_count receives the
// number of shifts left in sm.shifts.
__device__ int aed(cplx* T, int ldt, cplx* Z, int n, int l, int i, const MsSmem& sm, const Team& tm, int* ctrl,
                   int* shift_count) {
  const int tid = threadIdx.x, nthr = blockDim.x;
  const bool lead = tm.rank == 0;
  const int stride = nthr * tm.size, off0 = tid + nthr * tm.rank;
  const int nw = kAedW;
  const int kw = i - nw + 1;
  cplx* W = sm.work;
  cplx* V = W + kAedW * kAedLd;
  cplx* hv = V + kAedW * kAedLd;
  const double ulp = 2.0 * RCWA_DBL_EPS;
  const double smlnum = RCWA_DBL_MIN * ((double)n / ulp);
  for (int idx = tid; idx < nw * nw; idx += nthr) {
    const int r = idx / nw, c = idx % nw;
    AW(r, c) = T[(size_t)(kw + r) * ldt + kw + c];
    AV(r, c) = mkc(r == c ? 1.0 : 0.0, 0.0);
  }
  const cplx s = T[(size_t)kw * ldt + kw - 1];
  __syncthreads();
  // every CTA holds the window before the first one writes it back
  if (tm.size > 1) tm.sync();
  if (tid < 32) {
    const int lane = tid;
#ifdef RCWA_EIG_STATS
    long long c_w0 = clock64();
#endif
    const bool ok = aed_window_schur(W, V, nw);
#ifdef RCWA_EIG_STATS
    if (lane == 0) { const long long c_w1 = clock64(); atomicAdd(&g_eig_stats[5], (unsigned long long)(c_w1 - c_w0)); c_w0 = c_w1; }
#endif
    int ns = nw;
    if (ok) {
      // deflation test from the bottom, undeflatable eigenvalues moved up
      int ilst = 0;
      const double as = cabs1(s);
      for (int knt = 0; knt < nw && ns > ilst; ++knt) {
        double foo = cabs1(AW(ns - 1, ns - 1));
        if (foo == 0.0) foo = as;
        if (as * cabs1(AV(0, ns - 1)) <= fmax(smlnum, ulp * foo)) {
          --ns;
        } else {
          for (int k = ns - 2; k >= ilst; --k) aed_swap(W, V, nw, k);
          ++ilst;
        }
      }
      // shifts: the bottom undeflated eigenvalues, before the reflection
      const int cnt = min(ns, kMsShifts);
      if (lane < cnt) sm.shifts[lane] = AW(ns - cnt + lane, ns - cnt + lane);
      if (lane == 0) sm.aed[2] = cnt;
      __syncwarp();
      if (ns < nw && ns > 1 && (s.x != 0.0 || s.y != 0.0)) {
        // reflect the spike onto its first entry
        if (lane < ns) hv[lane] = cmul(s, cconj(AV(0, lane)));
        __syncwarp();
        const cplx tau = aed_house(hv, ns);
        if (tau.x != 0.0 || tau.y != 0.0) {
          aed_left(W, hv, ns, tau, 0, 0, nw);
          aed_right(W, hv, ns, tau, ns, 0);
          aed_right(V, hv, ns, tau, nw, 0);
        }
        // back to Hessenberg form
        for (int j = 0; j + 2 < ns; ++j) {
          const int len = ns - j - 1;
          if (lane < len) hv[lane] = AW(j + 1 + lane, j);
          __syncwarp();
          const cplx tj = aed_house(hv, len);
          if (tj.x != 0.0 || tj.y != 0.0) {
            if (lane < len) AW(j + 1 + lane, j) = lane == 0 ? hv[0] : mkc(0.0, 0.0);
            __syncwarp();
            aed_left(W, hv, len, tj, j + 1, j + 1, nw);
            aed_right(W, hv, len, tj, ns, j + 1);
            aed_right(V, hv, len, tj, nw, j + 1);
          }
        }
      }
    }
    if (lane == 0) { sm.aed[0] = ok ? 1 : 0; sm.aed[1] = ns; }
#ifdef RCWA_EIG_STATS
    if (lane == 0) atomicAdd(&g_eig_stats[6], (unsigned long long)(clock64() - c_w0));
#endif
  }
  __syncthreads();
  bool ok = sm.aed[0] != 0;
  int ns = sm.aed[1];
  bool spike = s.x != 0.0 || s.y != 0.0;
  *shift_count = sm.aed[2];
  if (tm.size > 1) {
    if (lead && tid == 0) {
      ctrl[2] = ok ? ns : -1;
      ctrl[3] = sm.aed[2];
      ctrl[4] = spike ? 1 : 0;
    }
    tm.sync();
    const int c2 = __ldcg(ctrl + 2);
    ok = c2 >= 0;
    ns = ok ? c2 : ns;
    *shift_count = __ldcg(ctrl + 3);
    spike = __ldcg(ctrl + 4) != 0;
  }
  if (!ok) return -1;
  if (ns == nw && spike) return 0;
#ifdef RCWA_EIG_STATS
  const long long c_off = clock64();
#endif
  // window, spike and the off-window blocks
  if (lead) {
    for (int idx = tid; idx < nw * nw; idx += nthr) {
      const int r = idx / nw, c = idx % nw;
      T[(size_t)(kw + r) * ldt + kw + c] = AW(r, c);
    }
    if (tid == 0) T[(size_t)kw * ldt + kw - 1] = cmul(s, cconj(AV(0, 0)));
  }
  // rows kw..i right of the window: Vh * T
  for (int j = i + 1 + off0; j < n; j += stride) {
    cplx x[kAedW];
#pragma unroll
    for (int r = 0; r < kAedW; ++r) x[r] = T[(size_t)(kw + r) * ldt + j];
#pragma unroll 4
    for (int r = 0; r < kAedW; ++r) {
      cplx acc = mkc(0.0, 0.0);
#pragma unroll
      for (int c = 0; c < kAedW; ++c) acc = cfmaconj(AV(c, r), x[c], acc);
      T[(size_t)(kw + r) * ldt + j] = acc;
    }
  }
  // columns kw..i above the window: T * V
  for (int r = off0; r < kw; r += stride) {
    cplx x[kAedW];
#pragma unroll
    for (int c = 0; c < kAedW; ++c) x[c] = T[(size_t)r * ldt + kw + c];
#pragma unroll 4
    for (int c = 0; c < kAedW; ++c) {
      cplx acc = mkc(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < kAedW; ++k) acc = cfma(x[k], AV(k, c), acc);
      T[(size_t)r * ldt + kw + c] = acc;
    }
  }
  // Schur vectors (column-major): Z(:, kw..i) * V
  for (int r = off0; r < n; r += stride) {
    cplx x[kAedW];
#pragma unroll
    for (int c = 0; c < kAedW; ++c) x[c] = Z[(size_t)(kw + c) * n + r];
#pragma unroll 4
    for (int c = 0; c < kAedW; ++c) {
      cplx acc = mkc(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < kAedW; ++k) acc = cfma(x[k], AV(k, c), acc);
      Z[(size_t)(kw + c) * n + r] = acc;
    }
  }
  tm.sync();
#ifdef RCWA_EIG_STATS
  STAT_ADD(7, clock64() - c_off);
#endif
  return nw - ns;
}

#undef AW
#undef AV

// Off-window update of one window pass for one lane: the rotations of every
// bulge, in chain order, on one line of T or Z (a column of T right of the
// window, a row of T above it, a row of Z), read and written through
// base + r * stride for index r in [rlo, rhi].  At pass step sg bulge b acts
// on the pair (p, p+1), p = top0 + sg + 3 (kMsShifts - 1 - b), so the chain
// spans kMsFrame consecutive indices that slide by one per step.  That span
// is held in registers: each step loads the index entering at the bottom
// (kMsPre steps ahead), applies the kMsShifts rotations in registers and
// stores the index leaving at the top, so every element crosses memory once
// per pass and the rotations run from registers, not shared memory.
// Rows: [x; y] <- [c x + s y; -conj(s) x + c y]; columns: the conjugate
// transpose [c x + conj(s) y; -s x + c y].
constexpr int kMsFrame = 3 * (kMsShifts - 1) + 2;
constexpr int kMsPre = 4;

template <bool kRows>
__device__ __forceinline__ void replay_frame(cplx* base, size_t stride, int top0, int nsteps, int rlo, int rhi,
                                             const MsSmem& sm) {
  cplx f[kMsFrame];
#pragma unroll
  for (int k = 0; k < kMsFrame - 1; ++k) {
    const int r = top0 + k;
    f[k] = (r >= rlo && r <= rhi) ? base[(size_t)r * stride] : mkc(0.0, 0.0);
  }
  f[kMsFrame - 1] = mkc(0.0, 0.0);
  cplx pre[kMsPre];
#pragma unroll
  for (int d = 0; d < kMsPre; ++d) {
    const int r = top0 + d + kMsFrame - 1;
    pre[d] = (d < nsteps && r >= rlo && r <= rhi) ? base[(size_t)r * stride] : mkc(0.0, 0.0);
  }
  for (int sg0 = 0; sg0 < nsteps; sg0 += kMsPre) {
    cplx cur[kMsPre];
#pragma unroll
    for (int d = 0; d < kMsPre; ++d) {
      cur[d] = pre[d];
      const int sg = sg0 + kMsPre + d, r = top0 + sg + kMsFrame - 1;
      pre[d] = (sg < nsteps && r >= rlo && r <= rhi) ? base[(size_t)r * stride] : mkc(0.0, 0.0);
    }
#pragma unroll
    for (int d = 0; d < kMsPre; ++d) {
      const int sg = sg0 + d;
      if (sg < nsteps) {
        f[kMsFrame - 1] = cur[d];
        const int* e = sm.ix + sg * kMsShifts;
#pragma unroll
        for (int b = 0; b < kMsShifts; ++b) {
          const int slot = e[b];
          const double c = sm.lc[b * kMsLog + slot];
          const cplx sn = sm.ls[b * kMsLog + slot];
          const int kb = 3 * (kMsShifts - 1 - b);
          const cplx x = f[kb], y = f[kb + 1];
          if (kRows) {
            f[kb] = cfma(sn, y, cscale(x, c));
            f[kb + 1] = cfma(cneg(cconj(sn)), x, cscale(y, c));
          } else {
            f[kb] = cfma(cconj(sn), y, cscale(x, c));
            f[kb + 1] = cfma(cneg(sn), x, cscale(y, c));
          }
        }
        const int rt = top0 + sg;
        if (rt >= rlo && rt <= rhi) base[(size_t)rt * stride] = f[0];
#pragma unroll
        for (int k = 0; k < kMsFrame - 1; ++k) f[k] = f[k + 1];
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kMsFrame - 1; ++k) {
    const int r = top0 + nsteps + k;
    if (r >= rlo && r <= rhi) base[(size_t)r * stride] = f[k];
  }
}

// One multishift sweep over the active block [l, i] with sm.shifts[0..s).
// Bulge b sits at position p = l + t - 3b at chain step t; it is active while
// l <= p <= i-1 and its rotation acts on rows/columns (p, p+1).
// With a team of several CTAs every CTA chases the bulges through its own
// copy of the window (the same operations on the same data), the first CTA
// writes the window back, and the off-window lines are split over the team.
__device__ void ms_sweep(cplx* T, int ldt, cplx* Z, int n, int l, int i, int s, const MsSmem& sm, const Team& tm) {
  const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarp = nthr >> 5;
  const int tend = (i - l) + 3 * (s - 1);
  int t = 0;
  while (t < tend) {
    const int bmax0 = min(s - 1, t / 3);
    const int pmin = l + t - 3 * bmax0;
    // while bulges are still being introduced at l the window starts at l
    const int ws = (t < 3 * (s - 1) || pmin == l) ? l : pmin - 1;
    const int we = min(i, ws + kMsW - 1);
    const int w = we - ws + 1;
    int t1 = t;
    while (t1 < tend) {
      const int over = l + t1 - (i - 1);
      const int b0 = over > 0 ? (over + 2) / 3 : 0;
      if (we != i && l + t1 - 3 * b0 + 2 > we) break;
      ++t1;
    }
    STAT_ADD(2, 1);
#ifdef RCWA_EIG_STATS
    const long long c_start = clock64();
#endif
    if (tid < s) { sm.firstp[tid] = -1; sm.cnt[tid] = 0; }
    for (int idx = tid; idx < w * w; idx += nthr)
      cp_async16(&MSW(idx / w, idx % w), &T[(size_t)(ws + idx / w) * ldt + ws + idx % w]);
    cp_async_wait_all();
    __syncthreads();
    // every CTA holds its window before the first one writes it back
    if (tm.size > 1) tm.sync();
    for (int tt = t; tt < t1; ++tt) {
      const int over = l + tt - (i - 1);
      const int bA = over > 0 ? (over + 2) / 3 : 0;
      const int bB = min(s - 1, tt / 3);
      if (tid >= bA && tid <= bB) {
        const int b = tid, p = l + tt - 3 * b;
        cplx x, y;
        if (p == l) { x = csub(MSW(p - ws, p - ws), sm.shifts[b]); y = MSW(p + 1 - ws, p - ws); }
        else { x = MSW(p - ws, p - 1 - ws); y = MSW(p + 1 - ws, p - 1 - ws); }
        double c;
        cplx sn;
        givens_fast(x, y, c, sn);
        if (sm.firstp[b] < 0) { sm.firstp[b] = p; sm.tfirst[b] = tt - t; }
        const int k = p - sm.firstp[b];
        sm.lc[b * kMsLog + k] = c;
        sm.ls[b * kMsLog + k] = sn;
        sm.cnt[b] = k + 1;
      }
      __syncthreads();
      // row operations: bulge b on rows (p, p+1), columns max(p-1, l) .. we
      const int nact = bB - bA + 1;
      for (int idx = tid; idx < nact * kMsW; idx += nthr) {
        const int b = bA + idx / kMsW;
        const int p = l + tt - 3 * b;
        const int j = ((p == l) ? l : p - 1) + idx % kMsW;
        if (j > we) continue;
        const int k = p - sm.firstp[b];
        const double c = sm.lc[b * kMsLog + k];
        const cplx sn = sm.ls[b * kMsLog + k];
        const cplx a = MSW(p - ws, j - ws), bb = MSW(p + 1 - ws, j - ws);
        MSW(p - ws, j - ws) = cfma(sn, bb, cscale(a, c));
        MSW(p + 1 - ws, j - ws) = cfma(cneg(cconj(sn)), a, cscale(bb, c));
      }
      __syncthreads();
      if (tid >= bA && tid <= bB) {
        const int p = l + tt - 3 * tid;
        if (p > l) MSW(p + 1 - ws, p - 1 - ws) = mkc(0.0, 0.0);
      }
      // column operations: bulge b on columns (p, p+1), rows ws .. min(p+2, i)
      for (int idx = tid; idx < nact * kMsW; idx += nthr) {
        const int b = bA + idx / kMsW;
        const int p = l + tt - 3 * b;
        const int r = ws + idx % kMsW;
        if (r > min(p + 2, i)) continue;
        const int k = p - sm.firstp[b];
        const double c = sm.lc[b * kMsLog + k];
        const cplx sn = sm.ls[b * kMsLog + k];
        const cplx a = MSW(r - ws, p - ws), bb = MSW(r - ws, p + 1 - ws);
        MSW(r - ws, p - ws) = cfma(cconj(sn), bb, cscale(a, c));
        MSW(r - ws, p + 1 - ws) = cfma(cneg(sn), a, cscale(bb, c));
      }
      __syncthreads();
    }
#ifdef RCWA_EIG_STATS
    const long long c_mid = clock64();
    STAT_ADD(3, c_mid - c_start);
#endif
    if (tm.rank == 0)
      for (int idx = tid; idx < w * w; idx += nthr) T[(size_t)(ws + idx / w) * ldt + ws + idx % w] = MSW(idx / w, idx % w);
    // rows/columns touched in this pass
    int rlo = i + 1, rhi = -1;
    for (int b = 0; b < s; ++b)
      if (sm.cnt[b] > 0) { rlo = min(rlo, sm.firstp[b]); rhi = max(rhi, sm.firstp[b] + sm.cnt[b]); }
    const int nsteps = t1 - t;
    // replay table per chain step and bulge: the log slot of the bulge's
    // rotation at that step (the identity slot while it is inactive), so the
    // chains interleave without branches
    for (int idx = tid; idx < nsteps * kMsShifts; idx += nthr) {
      const int sg = idx / kMsShifts, b = idx % kMsShifts;
      int slot = kMsW;
      if (b < s) {
        const int k = sg - sm.tfirst[b];
        if (k >= 0 && k < sm.cnt[b]) slot = k;
      }
      sm.ix[idx] = slot;
    }
    __syncthreads();
    const int top0 = l + t - 3 * (kMsShifts - 1);
    const int nR = (n - 1 - we + 31) / 32, nU = (ws + 31) / 32, nZ = (n + 31) / 32;
    for (int task = warp + nwarp * tm.rank; task < nR + nU + nZ; task += nwarp * tm.size) {
      if (task < nR) {
        // T(rlo..rhi, j), j right of the window: row rotations, lane = column
        const int j = we + 1 + 32 * task + lane;
        if (j < n) replay_frame<true>(T + j, (size_t)ldt, top0, nsteps, rlo, rhi, sm);
      } else if (task < nR + nU) {
        // T(r, rlo..rhi), r above the window: column rotations, lane = row
        const int r = 32 * (task - nR) + lane;
        if (r < ws) replay_frame<false>(T + (size_t)r * ldt, (size_t)1, top0, nsteps, rlo, rhi, sm);
      } else {
        // Z(r, rlo..rhi) (column-major): column rotations, lane = row
        const int r = 32 * (task - nR - nU) + lane;
        if (r < n) replay_frame<false>(Z + r, (size_t)n, top0, nsteps, rlo, rhi, sm);
      }
    }
    tm.sync();
#ifdef RCWA_EIG_STATS
    STAT_ADD(4, clock64() - c_mid);
#endif
    t = t1;
  }
}

// Schur form by multishift sweeps on active blocks of at least ms_min rows
// (ms_min >= kMsMin) and single-shift sweeps on smaller ones.  Returns 0 or
// RCWA_ERR_NOCONV.  With a team of several CTAs the first CTA finds each
// split point and runs the single-shift sweeps, and every decision that
// steers the team's barriers comes from the first CTA through ctrl (global
// scratch of at least 8 ints), so all CTAs take the same path.
__device__ int schur_ms(cplx* T, int ldt, cplx* Z, int n, int ms_min, const MsSmem& sm, int sweep_cap,
                        const Team& tm, int* ctrl) {
  const double ulp = 2.0 * RCWA_DBL_EPS;
  const double smlnum = RCWA_DBL_MIN * ((double)n / ulp);
  const int tid = threadIdx.x;
  int i = n - 1;
  long long sweeps = 0;
  const long long budget = sweep_cap > 0 ? min(30LL * max(10, n), (long long)sweep_cap) : 30LL * max(10, n);
  int stall = 0, last_i = -1, last_l = -1;
  const bool lead = tm.rank == 0;
  int it = 0;
  while (i >= 0) {
    int l = 0;
    if (lead) {
      int best = 0;
      for (int k = 1 + tid; k <= i; k += blockDim.x)
        if (negligible(T, ldt, k, 0, i, ulp, smlnum)) best = max(best, k);
      l = block_max_int(best, sm.redi);
      if (l > 0 && tid == 0) T[(size_t)l * ldt + l - 1] = mkc(0.0, 0.0);
      if (tm.size > 1 && tid == 0) ctrl[it & 1] = l;
    }
    tm.sync();
    if (tm.size > 1) l = __ldcg(ctrl + (it & 1));  // two slots: the first CTA may run one split ahead
    ++it;
    if (l >= i) {
      --i;
      stall = 0;
      continue;
    }
    stall = (i == last_i && l == last_l) ? stall + 1 : 0;
    last_i = i;
    last_l = l;
    const int m = i - l + 1;
    if (m < ms_min) {
      // small blocks: single-shift sweeps whose off-window updates stream
      // only the rotated pairs (cheaper than full tiles for few rotations)
      cplx shift;
      if (stall == 10 || stall == 30)
        shift = cadd(T[(size_t)l * ldt + l], mkc(0.75 * cabs1(T[(size_t)(l + 1) * ldt + l]), 0.0));
      else if (stall == 20 || stall == 40)
        shift = cadd(T[(size_t)i * ldt + i], mkc(0.75 * cabs1(T[(size_t)i * ldt + i - 1]), 0.0));
      else
        shift = wilkinson_shift(T[(size_t)(i - 1) * ldt + i - 1], T[(size_t)(i - 1) * ldt + i],
                                T[(size_t)i * ldt + i - 1], T[(size_t)i * ldt + i]);
      __syncthreads();
      STAT_ADD(1, 1);
#ifdef RCWA_EIG_STATS
      const long long c_ss = clock64();
#endif
      if (lead) qr_sweep(T, ldt, Z, n, l, i, shift, reinterpret_cast<cplx(*)[kWin + 1]>(sm.Wt), sm.lc, sm.ls);
#ifdef RCWA_EIG_STATS
      STAT_ADD(9, clock64() - c_ss);
#endif
      if (++sweeps > budget) return RCWA_ERR_NOCONV;
      continue;
    }
    // aggressive early deflation on the trailing window; its undeflated
    // eigenvalues are the next sweep's shifts
    int s = kMsShifts, ib = i;
    bool have_shifts = false;
    {
#ifdef RCWA_EIG_STATS
      const long long c_aed = clock64();
#endif
      int cnt = 0;
      const int nd = aed(T, ldt, Z, n, l, i, sm, tm, ctrl, &cnt);
#ifdef RCWA_EIG_STATS
      STAT_ADD(8, clock64() - c_aed);
      STAT_ADD(11, 1);
      STAT_ADD(12, nd > 0 ? nd : 0);
#endif
      if (nd > 0) {
        stall = 0;
        if (100 * nd > kAedNibble * kAedW || i - nd - l + 1 < ms_min) {
          if (++sweeps > budget) return RCWA_ERR_NOCONV;
          continue;
        }
        ib = i - nd;
      }
      if (nd >= 0 && cnt >= kMsShifts / 2) {
        s = cnt;
        have_shifts = true;
      }
    }
    __syncthreads();
    {
      STAT_ADD(0, 1);
      if (tid < 32) {
        cplx* B = sm.work;  // s x s, stride s + 1
        const int o = ib - s + 1;
        if (stall > 0 && stall % 6 == 0) {
          for (int k = tid; k < s; k += 32)
            sm.shifts[k] = cadd(T[(size_t)(o + k) * ldt + o + k],
                                mkc(0.75 * cabs1(T[(size_t)(o + k) * ldt + o + k - 1]), 0.0));
        } else if (!have_shifts) {
          for (int idx = tid; idx < s * s; idx += 32)
            B[(idx / s) * (s + 1) + idx % s] = T[(size_t)(o + idx / s) * ldt + o + idx % s];
          __syncwarp();
          small_eigs_warp(B, s + 1, s, sm.shifts);
        }
      }
    }
    __syncthreads();
    ms_sweep(T, ldt, Z, n, l, ib, s, sm, tm);
    if (++sweeps > budget) return RCWA_ERR_NOCONV;
  }
  return 0;
}

// True when every entry of the Hessenberg matrix is finite (whole CTA).  A
// NaN or Inf never passes the deflation tests, so such a matrix would only
// burn the sweep budget; it is reported as RCWA_ERR_NONFINITE instead.
__device__ bool hessenberg_finite(const cplx* T, int ldt, int n, int* redi) {
  int bad = 0;
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
    const int r = idx / n, c = idx % n;
    if (r <= c + 1) {
      const cplx v = T[(size_t)r * ldt + c];
      if (!isfinite(v.x) || !isfinite(v.y)) bad = 1;
    }
  }
  return block_max_int(bad, redi) == 0;
}

__global__ void __launch_bounds__(kMsThreads) schur_ms_kernel(cplx* const* Aarr, int n, int lda, cplx* w_all,
                                                             void* work, int* info_all, int ms_min, int sweep_cap) {
  extern __shared__ __align__(16) unsigned char dsm[];
  const MsSmem sm = carve_ms_smem(dsm);
  // identity slot of every bulge's rotation log (inactive chain steps)
  for (int b = threadIdx.x; b < kMsShifts; b += blockDim.x) {
    sm.lc[b * kMsLog + kMsW] = 1.0;
    sm.ls[b * kMsLog + kMsW] = mkc(0.0, 0.0);
  }
  __syncthreads();
  // one matrix per team (cluster) of CTAs
  const Team tm = cluster_team();
  const int mb = blockIdx.x / tm.size;
  cplx* A = Aarr[mb];
  const Scratch s = scratch_for(work, n, mb);
  // the team's decisions go through the reflector scalars' storage, dead
  // after the Hessenberg reduction (n >= 64 doubles)
  int* ctrl = reinterpret_cast<int*>(s.tau);
#ifdef RCWA_EIG_STATS
  const long long c_schur = clock64();
#endif
  bool fin = false;
  if (tm.rank == 0) {
    fin = hessenberg_finite(A, lda, n, sm.redi);
    if (tm.size > 1 && threadIdx.x == 0) ctrl[5] = fin ? 1 : 0;
  }
  if (tm.size > 1) {
    tm.sync();
    fin = __ldcg(ctrl + 5) != 0;
  }
  const int status = fin ? schur_ms(A, lda, s.Z, n, ms_min, sm, sweep_cap, tm, ctrl) : RCWA_ERR_NONFINITE;
#ifdef RCWA_EIG_STATS
  STAT_ADD(10, clock64() - c_schur);
#endif
  if (tm.rank == 0) {
    cplx* w = w_all + (size_t)mb * n;
    for (int k = threadIdx.x; k < n; k += blockDim.x) w[k] = A[(size_t)k * lda + k];
    if (threadIdx.x == 0) info_all[mb] = status;
  }
}

// ---------------------------------------------------------------- eigenvectors
// Eigenvectors of the upper triangular T (LAPACK ztrevc, right vectors, back
// substitution with protected divisors): column k of X solves
// (T - t_kk I) x = 0 with x_k = 1 and x_j = 0 for j > k.  Blocked bottom-up
// over 64-row blocks [r0, r1): the coupling to the rows already solved,
// B = T(r0:r1, r1:) X(r1:, k), is a tile GEMM over the upper triangle of X
// (column tile by column tile, K cut at the tile's last column); the block
// itself is solved by one thread per column in two 32-row halves held in
// registers.
constexpr int kTrBlk = 64;

template <int R>
__device__ __forceinline__ void trevc_half(const cplx* T, int ldt, cplx* X, int n, int k, int h0, int hend,
                                           cplx tkk, double ulp, double smlnum, cplx (&x)[R]) {
  // rows h0 .. h0+R-1 (those < hend); X(i, k) holds the right-hand side
  const double smin = fmax(ulp * cabs1(tkk), smlnum);
#pragma unroll
  for (int ii = R - 1; ii >= 0; --ii) {
    const int i = h0 + ii;
    cplx xi = mkc(0.0, 0.0);
    if (i < hend) {
      if (i == k) {
        xi = mkc(1.0, 0.0);
      } else if (i < k) {
        cplx acc = X[(size_t)i * n + k];
#pragma unroll
        for (int jj = ii + 1; jj < R; ++jj) acc = cfma(__ldg(&T[(size_t)i * ldt + h0 + jj]), x[jj], acc);
        cplx d = csub(__ldg(&T[(size_t)i * ldt + i]), tkk);
        if (cabs1(d) < smin) d = mkc(smin, 0.0);
        xi = cneg(cdiv(acc, d));
      }
      X[(size_t)i * n + k] = xi;
    }
    x[ii] = xi;
  }
}

__device__ void trevc_blocked(const cplx* T, int ldt, cplx* X, int n, TileSmem& tsm) {
  const double ulp = 2.0 * RCWA_DBL_EPS;
  const double smlnum = RCWA_DBL_MIN * ((double)n / ulp);
  // X = 0 everywhere but the unit diagonal; rows are overwritten block by block
  for (size_t idx = threadIdx.x; idx < (size_t)n * n; idx += blockDim.x)
    X[idx] = mkc((idx / n) == (idx % n) ? 1.0 : 0.0, 0.0);
  __syncthreads();
  const int nblk = (n + kTrBlk - 1) / kTrBlk;
  for (int bi = nblk - 1; bi >= 0; --bi) {
    const int r0 = bi * kTrBlk, r1 = min(n, r0 + kTrBlk);
    // B(r0:r1, c) = sum_{j >= r1} T(r0:r1, j) X(j, c) for columns c >= r1;
    // X(j, c) = 0 for j > c, so the tile of columns [c0, c0+64) needs j < c0+64
    for (int c0 = r1; c0 < n; c0 += kTBN) {
      const int nc = min(kTBN, n - c0);
      const int K = min(n, c0 + nc) - r1;
      cta_gemm<false, false>(tsm, r1 - r0, nc, K, T + (size_t)r0 * ldt + r1, ldt, X + (size_t)r1 * n + c0, n,
                             X + (size_t)r0 * n + c0, n, nullptr, 0, mkc(1.0, 0.0), mkc(0.0, 0.0));
    }
    // columns k > r0 solve the block rows; columns inside the block start
    // from a zero right-hand side (X(i, k) = 0 for i < k there)
    for (int k = r0 + 1 + threadIdx.x; k < n; k += blockDim.x) {
      const cplx tkk = __ldg(&T[(size_t)k * ldt + k]);
      cplx xl[32], xh[32];
      // lower half [r0+32, r1)
      trevc_half<32>(T, ldt, X, n, k, r0 + 32, r1, tkk, ulp, smlnum, xh);
      // the lower half's contribution to the upper half's right-hand side
      if (k > r0) {
        for (int ii = 0; ii < 32 && r0 + ii < min(k, r1); ++ii) {
          const int i = r0 + ii;
          cplx acc = X[(size_t)i * n + k];
#pragma unroll
          for (int jj = 0; jj < 32; ++jj)
            if (r0 + 32 + jj < r1) acc = cfma(__ldg(&T[(size_t)i * ldt + r0 + 32 + jj]), xh[jj], acc);
          X[(size_t)i * n + k] = acc;
        }
      }
      trevc_half<32>(T, ldt, X, n, k, r0, min(r1, r0 + 32), tkk, ulp, smlnum, xl);
    }
    __syncthreads();
  }
}

// The Hessenberg reduction runs 512 threads: its per-column sweeps and
// matrix-vector products stream from L2/DRAM and need the loads in flight;
// the first 256 threads also run the tile products.
constexpr int kHessThreads = 512;

template <bool kTeam>
__global__ void __launch_bounds__(kHessThreads) hessenberg_kernel(cplx* const* Aarr, int n, int lda, void* work) {
  __shared__ double red[kHessThreads / 32];
  __shared__ TileSmem tsm;
  // one matrix per team (cluster) of CTAs
  const Team tm = kTeam ? cluster_team() : Team{0, 1};
  const int mb = blockIdx.x / tm.size;
  const Scratch s = scratch_for(work, n, mb);
  hessenberg_blocked<kTeam>(Aarr[mb], n, lda, s, red, tsm, tm);
}

__global__ void __launch_bounds__(kEigThreads) schur_kernel(cplx* const* Aarr, int n, int lda, cplx* w_all,
                                                           void* work, int* info_all, int sweep_cap) {
  __shared__ cplx Wt[kWin][kWin + 1];
  __shared__ int redi[kEigThreads / 32];
  __shared__ double rc[kWin];
  __shared__ cplx rs[kWin];
  cplx* A = Aarr[blockIdx.x];
  const Scratch s = scratch_for(work, n, blockIdx.x);
  const int status = hessenberg_finite(A, lda, n, redi) ? schur(A, lda, s.Z, n, Wt, rc, rs, redi, sweep_cap)
                                                       : RCWA_ERR_NONFINITE;
  cplx* w = w_all + (size_t)blockIdx.x * n;
  for (int k = threadIdx.x; k < n; k += blockDim.x) w[k] = A[(size_t)k * lda + k];
  if (threadIdx.x == 0) info_all[blockIdx.x] = status;
}

__global__ void __launch_bounds__(kEigThreads) trevc_kernel(cplx* const* Aarr, int n, int lda, void* work) {
  __shared__ TileSmem tsm;
  const Scratch s = scratch_for(work, n, blockIdx.x);
  trevc_blocked(Aarr[blockIdx.x], lda, s.X, n, tsm);
}

// unit 2-norm columns; non-finite eigenpairs flag the matrix
__global__ void normalize_kernel(cplx* const* VRarr, int n, int ldv, const cplx* w_all, int* info_all) {
  cplx* VR = VRarr[blockIdx.y];
  const cplx* w = w_all + (size_t)blockIdx.y * n;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double ss = 0.0;
  for (int i = 0; i < n; ++i) ss += cnorm2(VR[(size_t)i * ldv + j]);
  const double sc = ss > 0.0 ? 1.0 / sqrt(ss) : 1.0;
  for (int i = 0; i < n; ++i) VR[(size_t)i * ldv + j] = cscale(VR[(size_t)i * ldv + j], sc);
  if (!isfinite(sc) || !isfinite(ss) || !isfinite(w[j].x) || !isfinite(w[j].y))
    atomicCAS(&info_all[blockIdx.y], 0, RCWA_ERR_NONFINITE);
}


}  // namespace


namespace {
// QR sweep cap of every later eigensolve (0: the built-in budget), set by
// rcwa_set_qr_sweep_limit; read when the Schur kernels are launched.
std::atomic<int> g_qr_sweep_cap{0};
// CTAs per matrix of the Hessenberg and multishift Schur kernels (0: the
// automatic choice), set by rcwa_set_eig_cluster.
std::atomic<int> g_eig_team{0};

// Matrices of at least this order use a team of CTAs when the batch leaves
// SMs idle.
constexpr int kTeamMinN = 1024;

// Clusters of `size` CTAs of `kernel` that fit on the device at once.
template <class K>
int active_clusters(K kernel, int threads, size_t smem, int size) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(size);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = size;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int nc = 0;
  if (cudaOccupancyMaxActiveClusters(&nc, (void*)kernel, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nc;
}

// Team size for a batch of order-n matrices: the largest (up to 8) whose
// clusters of both kernels all fit on the device in one wave, when the batch
// alone would leave at least half of the SMs idle; 1 otherwise.
int eig_team_size(int n, int batch, int ms_smem) {
  const int forced = g_eig_team.load();
  if (forced > 0) return forced;
  if (n < kTeamMinN) return 1;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (2 * batch > sms) return 1;
  static std::mutex mu;
  static std::map<std::pair<int, int>, int> cache;  // (device, batch) -> size
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find({dev, batch});
  if (it != cache.end()) return it->second;
  int pick = 1;
  for (int c = std::min(8, sms / batch); c >= 2; --c)
    if (active_clusters(hessenberg_kernel<true>, kHessThreads, 0, c) >= batch &&
        active_clusters(schur_ms_kernel, kMsThreads, (size_t)ms_smem, c) >= batch) {
      pick = c;
      break;
    }
  cache[{dev, batch}] = pick;
  return pick;
}

// launch of kernel over batch * team CTAs in clusters of `team`
template <class K, class... Args>
cudaError_t launch_team(K kernel, int batch, int team, int threads, size_t smem, cudaStream_t st, Args... args) {
  if (team <= 1) {
    kernel<<<batch, threads, smem, st>>>(args...);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(batch * team);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = team;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}
}  // namespace

extern "C" int rcwa_set_qr_sweep_limit(int sweeps) {
  if (sweeps < 0) return RCWA_ERR_INVALID;
  g_qr_sweep_cap.store(sweeps);
  return RCWA_OK;
}

extern "C" int rcwa_set_eig_cluster(int ctas) {
  if (ctas < 0 || ctas > 8) return RCWA_ERR_INVALID;
  g_eig_team.store(ctas);
  return RCWA_OK;
}

extern "C" int rcwa_eig_cluster_size(int n, int batch) {
  if (n < kMsMin || batch <= 0) return 1;
  return eig_team_size(n, batch, (int)kMsSmemBytes);
}

cudaError_t zgeev_batched(cplx* const* A, int n, int lda, cplx* w, cplx* const* VR, int ldv, void* work,
                          int* info, int batch, cudaStream_t st, StageProf* prof, int ms_min) {
  if (batch <= 0 || n <= 0) return cudaSuccess;
  ms_min = max(ms_min, kMsMin);
  const int sweep_cap = g_qr_sweep_cap.load();
  StageProf none;
  StageProf& P = prof ? *prof : none;
  static SmemAttrOnce attr;
  cudaError_t e = attr.ensure(schur_ms_kernel, (int)kMsSmemBytes);
  if (e != cudaSuccess) return e;
  // a team of CTAs per matrix where the batch is too small to fill the GPU
  // (the single-shift kernel for small orders always runs one CTA)
  const int team = n < ms_min ? 1 : eig_team_size(n, batch, (int)kMsSmemBytes);
  e = team > 1 ? launch_team(hessenberg_kernel<true>, batch, team, kHessThreads, 0, st, A, n, lda, work)
               : launch_team(hessenberg_kernel<false>, batch, 1, kHessThreads, 0, st, A, n, lda, work);
  if (e != cudaSuccess) return e;
  ++launch_counter();
  P.mark(st, kStHessenberg);
  if (n < ms_min) {
    schur_kernel<<<batch, kEigThreads, 0, st>>>(A, n, lda, w, work, info, sweep_cap);
    ++launch_counter();
  } else {
    if ((e = launch_team(schur_ms_kernel, batch, team, kMsThreads, kMsSmemBytes, st, A, n, lda, w, work, info,
                         ms_min, sweep_cap)) != cudaSuccess)
      return e;
    ++launch_counter();
  }
  P.mark(st, kStSchur);
  trevc_kernel<<<batch, kEigThreads, 0, st>>>(A, n, lda, work);
  ++launch_counter();
  P.mark(st, kStTrevc);
  // VR = Z X for every matrix (Z column-major == transposed operand)
  GemmArgs g{};
  g.A = nullptr;
  g.A0 = (const cplx*)work;
  g.sA = workspace_bytes(n) / sizeof(cplx);
  g.B = nullptr;
  g.B0 = (const cplx*)work + (size_t)n * n;
  g.sB = g.sA;
  g.D = VR;
  g.M = n; g.N = n; g.K = n;
  g.lda = n; g.ldb = n; g.ldd = ldv; g.ldc = ldv;
  g.transA = 1; g.transB = 0;
  g.triB = 1;  // X is upper triangular
  g.alpha = mkc(1.0, 0.0); g.beta = mkc(0.0, 0.0); g.gammaI = mkc(0.0, 0.0);
  g.batch = batch;
  cudaError_t err = zgemm_batched(g, st);
  if (err != cudaSuccess) return err;
  P.mark(st, kStBackTransform);
  dim3 grid((n + 127) / 128, batch);
  normalize_kernel<<<grid, 128, 0, st>>>(VR, n, ldv, w, info);
  ++launch_counter();
  P.mark(st, kStNormalize);
  return cudaGetLastError();
}

#ifdef RCWA_EIG_STATS
extern "C" int rcwa_debug_eig_stats(unsigned long long* out, int reset) {
  unsigned long long h[32];
  if (cudaMemcpyFromSymbol(h, g_eig_stats, sizeof(h)) != cudaSuccess) return 2;
  for (int i = 0; i < 32; ++i) out[i] = h[i];
  if (reset) {
    unsigned long long z[32] = {};
    cudaMemcpyToSymbol(g_eig_stats, z, sizeof(z));
  }
  return 0;
}
#endif
