// 3xTF32 complex GEMM on tcgen05.
//
// One CTA (four warps) computes a 128 x 128 (or 128 x 256) complex output tile.  For each
// 8-deep K slab the CTA converts its FP64 operand tiles into eight TF32
// planes in shared memory (A: re hi/lo, im hi/lo; B likewise), laid out as
// K-major, unswizzled UMMA core matrices (8 rows x 16 bytes; 8-row groups
// 128 B apart, 16-byte K chunks 2048 B apart).  One thread then issues, per
// K step of 8, twelve tcgen05.mma (M=128, N=128, K=8):
//   Re += Ar*Br (3 terms) - Ai*Bi (3 terms, A negated in the descriptor)
//   Im += Ar*Bi (3 terms) + Ai*Br (3 terms)
// into two FP32 accumulators in tensor memory (256 columns), and commits to
// the stage's mbarrier.  Slabs alternate between two stages of planes, so
// the conversion of one slab overlaps the MMAs of the previous one; a stage
// is refilled only after its last commit completed.  The two stages take
// 64 KB, so two CTAs share an SM (512 tensor-memory columns) and overlap too.  The epilogue reads the accumulators with
// tcgen05.ld (warp w owns rows 32w..32w+31) and writes alpha*acc + beta*C.
// The accumulators restart every kTcKBlock of K, their block sums being added
// into D in FP64, which bounds the FP32 accumulation error independently of K.
// Every wait is bounded: a wait that runs out sets the error flag, waits
// (bounded) for the MMAs in flight, frees the tensor memory and skips the
// tile's stores.
#include <algorithm>
#include <cstdint>

#include "gemm_tc.cuh"

namespace {

// Tile: kTcM rows of D by N columns (N = 128 or 256, the tile-shape choice of
// the engine's tuner).  A plane holds rows x kTcK TF32 values; the K-major
// planes' leading byte offset (between 4-value K chunks) is rows x 16 bytes.
constexpr int kTcM = 128, kTcK = 8;
constexpr int kTcThreads = 128;
constexpr int kPlaneA = kTcM * kTcK;                     // 1024 floats = 4 KB
constexpr int kSbo = 128;                                // bytes between 8-row groups
template <int N> struct TcTile {
  static constexpr int kPlaneB = N * kTcK;
  static constexpr int kStageFloats = 4 * kPlaneA + 4 * kPlaneB;
  // two stages + barriers; the 256-wide tile takes all 512 tensor-memory
  // columns of an SM, so it asks for enough shared memory to be alone there
  static constexpr size_t kSmemUsed = 2 * kStageFloats * sizeof(float) + 64;
  static constexpr size_t kSmem = N == 256 && kSmemUsed < 120 * 1024 ? 120 * 1024 : kSmemUsed;
  static constexpr uint32_t kTmemCols = 2 * N;                              // Re and Im accumulators
  static constexpr int kLboB = N * 16;
  // instruction descriptor: D F32, A/B TF32, both K-major, N, M = 128
  static constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
                                     ((uint32_t)(kTcM >> 4) << 24);
  static constexpr uint32_t kIdescNegA = kIdesc | (1u << 13);
};
constexpr int kLboA = kTcM * 16;
constexpr long kWaitLimit = 1L << 22;
// K-block of the FP32 accumulators: after every kTcKBlock of K the tensor-
// memory sums are added into D in FP64 and the accumulators restart.  The
// tensor cores' FP32 accumulation is not round-to-nearest: its error grows
// with the number of MMAs accumulated (six per 8-deep K step), so bounding
// that number bounds the product's error independently of K.  Measured on
// the lossless 2D pillar stack (Nx = Ny = 10, n = 882, 148 points): the
// largest |R + T - 1| of the mixed plan is 2.5e-5 / 4.8e-5 / 7.5e-5 / 1.04e-4
// for K-blocks of 128 / 256 / 512 / the whole K, and the cascade products
// take 417 / 289 / 198 / 150 ms per step; 256 keeps half of the 1e-4 budget.
#ifndef RCWA_TC_KBLOCK
#define RCWA_TC_KBLOCK 256
#endif
constexpr int kTcKBlock = RCWA_TC_KBLOCK;  // a build-time parameter

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of (row r, k) in a plane whose K chunks are lbo bytes apart
__device__ __forceinline__ int plane_off(int r, int k, int lbo) {
  return (k >> 2) * lbo + (r >> 3) * kSbo + (r & 7) * 16 + (k & 3) * 4;
}

// shared-memory matrix descriptor (sm100 layout: start >> 4 at [0,14), LBO >> 4
// at [16,30), SBO >> 4 at [32,46), version 1 at [46,48), no swizzle)
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, int lbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((kSbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (long it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void split_tf32(double v, float& hi, float& lo) {
  const float f = (float)v;
  uint32_t h, l;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(f));
  const float rest = f - __uint_as_float(h);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(rest));
  hi = __uint_as_float(h);
  lo = __uint_as_float(l);
}

__device__ __forceinline__ void st_plane4(float* plane, int off, float a, float b, float c, float d) {
  *reinterpret_cast<float4*>(reinterpret_cast<char*>(plane) + off) = make_float4(a, b, c, d);
}

// Largest |re|, |im| of each batch item's A (z = 0) or B (z = 1) as a binary
// exponent e with max < 2^e, combined over blocks by atomicMax into exps
// (initialised very negative; an all-zero matrix keeps that value).
__global__ void tc_scale_kernel(GemmArgs g, int* exps) {
  __shared__ double red[8];
  const int b = blockIdx.y, isB = blockIdx.z;
  const cplx* X = isB ? (g.B ? g.B[b] : g.B0 + b * g.sB) + g.offB : (g.A ? g.A[b] : g.A0 + b * g.sA) + g.offA;
  const int rows = isB ? g.K : g.M, cols = isB ? g.N : g.K, ld = isB ? g.ldb : g.lda;
  double mx = 0.0;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < (size_t)rows * cols;
       idx += (size_t)gridDim.x * blockDim.x) {
    const cplx v = X[(idx / cols) * ld + idx % cols];
    mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
  }
  for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) mx = fmax(mx, red[w]);
    if (mx > 0.0 && mx < INFINITY) {
      int e;
      frexp(mx, &e);  // mx = f 2^e, 0.5 <= f < 1
      atomicMax(&exps[isB * gridDim.y + b], e);
    }
  }
}

// Accumulators -> D for one K-block (whole CTA; warp w reads tensor-memory
// lanes 32w..32w+31, i.e. tile rows): the first block writes
// alpha*acc*2^eAB + beta*C + gammaI*I, every later block adds alpha*acc*2^eAB
// to D in FP64.
template <int N>
__device__ __forceinline__ void tc_epilogue(const GemmArgs& g, int b, int m0, int n0, uint32_t tRe, uint32_t tIm,
                                            int eAB, bool first) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m = m0 + 32 * warp + lane;
  const uint32_t row_addr = (uint32_t)(32 * warp) << 16;
  for (int cb = 0; cb < N; cb += 16) {
    uint32_t re[16], im[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(re[0]), "=r"(re[1]), "=r"(re[2]), "=r"(re[3]), "=r"(re[4]), "=r"(re[5]), "=r"(re[6]), "=r"(re[7]),
          "=r"(re[8]), "=r"(re[9]), "=r"(re[10]), "=r"(re[11]), "=r"(re[12]), "=r"(re[13]), "=r"(re[14]),
          "=r"(re[15])
        : "r"(tRe + row_addr + cb));
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(im[0]), "=r"(im[1]), "=r"(im[2]), "=r"(im[3]), "=r"(im[4]), "=r"(im[5]), "=r"(im[6]), "=r"(im[7]),
          "=r"(im[8]), "=r"(im[9]), "=r"(im[10]), "=r"(im[11]), "=r"(im[12]), "=r"(im[13]), "=r"(im[14]),
          "=r"(im[15])
        : "r"(tIm + row_addr + cb));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    if (m < g.M) {
      cplx* Drow = (g.D ? g.D[b] : g.D0 + b * g.sD) + g.offD + (size_t)m * g.ldd;
      const cplx* Crow =
          (first && (g.beta.x != 0.0 || g.beta.y != 0.0)) ? g.C[b] + g.offC + (size_t)m * g.ldc : nullptr;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int n = n0 + cb + j;
        if (n < g.N) {
          cplx v = cmul(g.alpha, mkc(ldexp((double)__uint_as_float(re[j]), eAB),
                                     ldexp((double)__uint_as_float(im[j]), eAB)));
          if (first) {
            if (Crow) v = cfma(g.beta, Crow[n], v);
            if (m == n) v = cadd(v, g.gammaI);
          } else {
            v = cadd(v, Drow[n]);
          }
          Drow[n] = v;
        }
      }
    }
  }
}

template <int N>
__global__ void __launch_bounds__(kTcThreads, N == 128 ? 2 : 1) zgemm_tf32x3_kernel(GemmArgs g, const int* exps,
                                                                                   int* err) {
  using Tile = TcTile<N>;
  constexpr int kPlaneB = Tile::kPlaneB;
  constexpr int kLboB = Tile::kLboB;
  constexpr uint32_t kTmemCols = Tile::kTmemCols;
  constexpr uint32_t kIdesc = Tile::kIdesc, kIdescNegA = Tile::kIdescNegA;
  extern __shared__ __align__(1024) unsigned char tsm[];
  // two stages of eight planes (A: re hi, re lo, im hi, im lo; then B)
  float* planes = reinterpret_cast<float*>(tsm);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(tsm + 2 * Tile::kStageFloats * sizeof(float));  // one per stage
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 2);
  int* s_fail = reinterpret_cast<int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int b = blockIdx.z;
  const int m0 = blockIdx.y * kTcM, n0 = blockIdx.x * N;
  const cplx* A = (g.A ? g.A[b] : g.A0 + b * g.sA) + g.offA;
  const cplx* B = (g.B ? g.B[b] : g.B0 + b * g.sB) + g.offB;
  const uint32_t mb0 = smem_u32(mbar), mb1 = smem_u32(mbar + 1);
  // exact power-of-two operand scales (an all-zero operand keeps scale 1)
  const int eA = max(exps[b], -1000), eB = max(exps[g.batch + b], -1000);
  const double sA = ldexp(1.0, eA > -1000 ? -eA : 0), sB = ldexp(1.0, eB > -1000 ? -eB : 0);
  const int eAB = (eA > -1000 ? eA : 0) + (eB > -1000 ? eB : 0);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *s_fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t tRe = tmem, tIm = tmem + N;

  // slab i goes to stage i % 2; before stage s is refilled, the MMAs of slab
  // i - 2 (its previous contents) must have completed.  The conversion of
  // slab i thus overlaps the MMAs of slab i - 1.
  uint32_t phase[2] = {0u, 0u};
  int pending[2] = {0, 0};  // uniform across the CTA
  int slab = 0;
  int kblock0 = 0;          // first K of the accumulators' current block
  for (int k0 = 0; k0 < g.K; k0 += kTcK, ++slab) {
    const int st = slab & 1;
    const uint32_t mbs = st ? mb1 : mb0;
    if (pending[st]) {
      if (mbar_wait(mbs, phase[st])) {
        phase[st] ^= 1u;
        pending[st] = 0;
      } else {
        *s_fail = 1;
      }
    }
    __syncthreads();
    if (*s_fail) break;
    float* P = planes + st * Tile::kStageFloats;
    float *Arh = P, *Arl = P + kPlaneA, *Aih = P + 2 * kPlaneA, *Ail = P + 3 * kPlaneA;
    float* PB = P + 4 * kPlaneA;
    float *Brh = PB, *Brl = PB + kPlaneB, *Bih = PB + 2 * kPlaneB, *Bil = PB + 3 * kPlaneB;
    // A: row tid, K chunks q (4 consecutive k each)
    {
      const int gm = m0 + tid;
#pragma unroll
      for (int q = 0; q < kTcK / 4; ++q) {
        float rh[4], rl[4], ih[4], il[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int gk = k0 + 4 * q + j;
          cplx v = mkc(0.0, 0.0);
          if (gm < g.M && gk < g.K) v = A[(size_t)gm * g.lda + gk];
          split_tf32(v.x * sA, rh[j], rl[j]);
          split_tf32(v.y * sA, ih[j], il[j]);
        }
        const int off = plane_off(tid, 4 * q, kLboA);
        st_plane4(Arh, off, rh[0], rh[1], rh[2], rh[3]);
        st_plane4(Arl, off, rl[0], rl[1], rl[2], rl[3]);
        st_plane4(Aih, off, ih[0], ih[1], ih[2], ih[3]);
        st_plane4(Ail, off, il[0], il[1], il[2], il[3]);
      }
    }
    // B: columns tid + 128 c (rows of the K-major plane), K chunks q
#pragma unroll
    for (int cc = 0; cc < N / kTcThreads; ++cc) {
      const int col = tid + kTcThreads * cc;
      const int gn = n0 + col;
#pragma unroll
      for (int q = 0; q < kTcK / 4; ++q) {
        float rh[4], rl[4], ih[4], il[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int gk = k0 + 4 * q + j;
          cplx v = mkc(0.0, 0.0);
          if (gn < g.N && gk < g.K) v = B[(size_t)gk * g.ldb + gn];
          split_tf32(v.x * sB, rh[j], rl[j]);
          split_tf32(v.y * sB, ih[j], il[j]);
        }
        const int off = plane_off(col, 4 * q, kLboB);
        st_plane4(Brh, off, rh[0], rh[1], rh[2], rh[3]);
        st_plane4(Brl, off, rl[0], rl[1], rl[2], rl[3]);
        st_plane4(Bih, off, ih[0], ih[1], ih[2], ih[3]);
        st_plane4(Bil, off, il[0], il[1], il[2], il[3]);
      }
    }
    // make the generic-proxy writes visible to the tensor cores
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int ks = 0; ks < kTcK / 8; ++ks) {
        const uint32_t oa = (uint32_t)(2 * ks * kLboA), ob = (uint32_t)(2 * ks * kLboB);
        const uint64_t arh = make_desc(smem_u32(Arh) + oa, kLboA), arl = make_desc(smem_u32(Arl) + oa, kLboA);
        const uint64_t aih = make_desc(smem_u32(Aih) + oa, kLboA), ail = make_desc(smem_u32(Ail) + oa, kLboA);
        const uint64_t brh = make_desc(smem_u32(Brh) + ob, kLboB), brl = make_desc(smem_u32(Brl) + ob, kLboB);
        const uint64_t bih = make_desc(smem_u32(Bih) + ob, kLboB), bil = make_desc(smem_u32(Bil) + ob, kLboB);
        const uint32_t acc = (k0 > kblock0 || ks > 0) ? 1u : 0u;
        mma_tf32(tRe, arh, brh, kIdesc, acc);
        mma_tf32(tRe, arh, brl, kIdesc, 1u);
        mma_tf32(tRe, arl, brh, kIdesc, 1u);
        mma_tf32(tRe, aih, bih, kIdescNegA, 1u);
        mma_tf32(tRe, aih, bil, kIdescNegA, 1u);
        mma_tf32(tRe, ail, bih, kIdescNegA, 1u);
        mma_tf32(tIm, arh, bih, kIdesc, acc);
        mma_tf32(tIm, arh, bil, kIdesc, 1u);
        mma_tf32(tIm, arl, bih, kIdesc, 1u);
        mma_tf32(tIm, aih, brh, kIdesc, 1u);
        mma_tf32(tIm, aih, brl, kIdesc, 1u);
        mma_tf32(tIm, ail, brh, kIdesc, 1u);
      }
      mma_commit(mbs);
    }
    pending[st] = 1;
    if (k0 + kTcK < g.K && k0 + kTcK - kblock0 >= kTcKBlock) {
      // end of a K-block: wait for its MMAs, add the accumulators into D in
      // FP64, and let the next slab's MMAs start fresh accumulators
      for (int s2 = 0; s2 < 2; ++s2) {
        if (!pending[s2]) continue;
        if (mbar_wait(s2 ? mb1 : mb0, phase[s2])) {
          phase[s2] ^= 1u;
          pending[s2] = 0;
        } else {
          *s_fail = 1;
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (*s_fail) break;
      tc_epilogue<N>(g, b, m0, n0, tRe, tIm, eAB, kblock0 == 0);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      kblock0 = k0 + kTcK;
    }
  }
  // the outstanding slabs' MMAs (after a failure too: nothing may still write
  // the tensor memory or the planes when they are freed); the commit of the
  // last slab also covers every earlier MMA
  for (int s2 = 0; s2 < 2; ++s2)
    if (pending[s2] && !mbar_wait(s2 ? mb1 : mb0, phase[s2])) *s_fail = 1;

  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const bool good = *s_fail == 0;
  if (!good && tid == 0) atomicExch(err, 1);
  if (good) tc_epilogue<N>(g, b, m0, n0, tRe, tIm, eAB, kblock0 == 0);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

// ------------------------------------------------------------ pre-split operands
// The operands are split into TF32 planes once per product instead of once
// per output tile: for row tile rt (128 rows of op(A), or 128 columns of B)
// and K slab ks (8 values) each plane (re hi, re lo, im hi, im lo) holds a
// 4 KB block already in the UMMA no-swizzle K-major layout, so a CTA moves a
// slab into shared memory with plain bulk copies (cp.async.bulk, the TMA
// engine, from this GPU's memory; no tensor map, no multicast) and its
// threads do no conversion at all.
#ifndef RCWA_TC_STAGES
#define RCWA_TC_STAGES 3
#endif
constexpr int kV2Stages = RCWA_TC_STAGES;  // a build-time parameter
constexpr size_t kV2StageBytes = 8 * 4096;  // 4 A planes + 4 B planes
constexpr size_t kV2Smem = kV2Stages * kV2StageBytes + 64;

__host__ __device__ inline size_t plane_blocks(int rows, int K) {
  return (size_t)((rows + kTcM - 1) / kTcM) * ((K + kTcK - 1) / kTcK);
}

// Planes of op A (isB = 0: rows = M, A row-major) or of B (isB = 1: rows = N,
// B row-major K x N, read column-wise) for every batch item, scaled by the
// item's power of two; zero outside the matrix.  One thread per (row, 4-value
// K chunk) of a (row tile, K slab) block.
__global__ void tc_split_kernel(GemmArgs g, const int* exps, int isB, float* planes) {
  const int b = blockIdx.y;
  const int rows = isB ? g.N : g.M;
  const int RT = (rows + kTcM - 1) / kTcM, KS = (g.K + kTcK - 1) / kTcK;
  const size_t nblk = (size_t)RT * KS;
  const int e = max(exps[isB * g.batch + b], -1000);
  const double sc = ldexp(1.0, e > -1000 ? -e : 0);
  const cplx* X = isB ? (g.B ? g.B[b] : g.B0 + b * g.sB) + g.offB : (g.A ? g.A[b] : g.A0 + b * g.sA) + g.offA;
  float* P = planes + (size_t)b * 4 * nblk * 1024;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nblk * 256; t += (size_t)gridDim.x * blockDim.x) {
    const size_t blk = t / 256;
    const int within = (int)(t % 256);
    const int r = within % kTcM, q = within / kTcM;  // row in the tile, K chunk (0 or 1)
    const int rt = (int)(blk / KS), ks = (int)(blk % KS);
    const int gr = rt * kTcM + r;
    float rh[4], rl[4], ih[4], il[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gk = ks * kTcK + 4 * q + j;
      cplx v = mkc(0.0, 0.0);
      if (gr < rows && gk < g.K) v = isB ? X[(size_t)gk * g.ldb + gr] : X[(size_t)gr * g.lda + gk];
      split_tf32(v.x * sc, rh[j], rl[j]);
      split_tf32(v.y * sc, ih[j], il[j]);
    }
    const int off = plane_off(r, 4 * q, kLboA) / 4;
    float* base = P + blk * 1024 + off;
    *reinterpret_cast<float4*>(base) = make_float4(rh[0], rh[1], rh[2], rh[3]);
    *reinterpret_cast<float4*>(base + nblk * 1024) = make_float4(rl[0], rl[1], rl[2], rl[3]);
    *reinterpret_cast<float4*>(base + 2 * nblk * 1024) = make_float4(ih[0], ih[1], ih[2], ih[3]);
    *reinterpret_cast<float4*>(base + 3 * nblk * 1024) = make_float4(il[0], il[1], il[2], il[3]);
  }
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(dst), "l"(src), "r"(bytes), "r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

// 128 x 128 output tile from pre-split planes.  Thread 0 runs a three-stage
// pipeline: the bulk copies of slab i are issued while the MMAs of slab
// i - 2 run; a stage is refilled once the commit of its previous MMAs has
// arrived.  At each K-block boundary the whole CTA adds the accumulators
// into D in FP64 (tc_epilogue).  Every wait is bounded.
__global__ void __launch_bounds__(kTcThreads, 2) zgemm_tf32x3_split_kernel(GemmArgs g, const int* exps,
                                                                          const float* planesA,
                                                                          const float* planesB, int* err) {
  using Tile = TcTile<128>;
  constexpr uint32_t kIdesc = Tile::kIdesc, kIdescNegA = Tile::kIdescNegA;
  extern __shared__ __align__(1024) unsigned char tsm[];
  uint64_t* full = reinterpret_cast<uint64_t*>(tsm + kV2Stages * kV2StageBytes);
  uint64_t* empty = full + kV2Stages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(empty + kV2Stages);
  int* s_fail = reinterpret_cast<int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int b = blockIdx.z;
  const int m0 = blockIdx.y * kTcM, n0 = blockIdx.x * 128;
  const int KS = (g.K + kTcK - 1) / kTcK;
  const size_t nblkA = plane_blocks(g.M, g.K), nblkB = plane_blocks(g.N, g.K);
  const float* PA = planesA + (size_t)b * 4 * nblkA * 1024 + (size_t)blockIdx.y * KS * 1024;
  const float* PB = planesB + (size_t)b * 4 * nblkB * 1024 + (size_t)blockIdx.x * KS * 1024;
  const int eA = max(exps[b], -1000), eB = max(exps[g.batch + b], -1000);
  const int eAB = (eA > -1000 ? eA : 0) + (eB > -1000 ? eB : 0);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(Tile::kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < kV2Stages; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(full + i)) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(empty + i)) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *s_fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t tRe = tmem, tIm = tmem + 128;
  uint32_t fphase[kV2Stages] = {}, ephase[kV2Stages] = {};
  int epending[kV2Stages] = {};  // a commit on empty[s] not yet waited for (thread 0)
  int fpending[kV2Stages] = {};  // bulk copies into stage s not yet waited for (thread 0)
  const int slabs_per_block = kTcKBlock / kTcK;
  int issued = 0;  // slabs whose copies thread 0 has issued (they run across K-blocks)
  for (int kb0 = 0; kb0 < KS; kb0 += slabs_per_block) {
    const int kb1 = min(KS, kb0 + slabs_per_block);
    if (tid == 0 && !*s_fail) {
      bool fail = false;
      // pipeline over the block's slabs: copies run kV2Stages - 1 slabs ahead,
      // into the next K-block too, so its first slabs arrive during the drain
      for (int j = kb0; j < kb1 && !fail; ++j) {
        while (issued < KS && issued <= j + kV2Stages - 1) {
          const int i = issued;
          const int stg = i % kV2Stages;
          if (epending[stg]) {
            if (!mbar_wait(smem_u32(empty + stg), ephase[stg])) { fail = true; break; }
            ephase[stg] ^= 1u;
            epending[stg] = 0;
          }
          const uint32_t fb = smem_u32(full + stg);
          mbar_expect_tx(fb, (uint32_t)kV2StageBytes);
          const uint32_t dst = smem_u32(tsm + stg * kV2StageBytes);
          for (int p = 0; p < 4; ++p) {
            bulk_g2s(dst + p * 4096, PA + (size_t)p * nblkA * 1024 + (size_t)i * 1024, 4096, fb);
            bulk_g2s(dst + (4 + p) * 4096, PB + (size_t)p * nblkB * 1024 + (size_t)i * 1024, 4096, fb);
          }
          fpending[stg] = 1;
          ++issued;
        }
        if (fail) break;
        {
          const int stg = j % kV2Stages;
          if (!mbar_wait(smem_u32(full + stg), fphase[stg])) { fail = true; break; }
          fphase[stg] ^= 1u;
          fpending[stg] = 0;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t base = smem_u32(tsm + stg * kV2StageBytes);
          const uint64_t arh = make_desc(base, kLboA), arl = make_desc(base + 4096, kLboA);
          const uint64_t aih = make_desc(base + 8192, kLboA), ail = make_desc(base + 12288, kLboA);
          const uint64_t brh = make_desc(base + 16384, kLboA), brl = make_desc(base + 20480, kLboA);
          const uint64_t bih = make_desc(base + 24576, kLboA), bil = make_desc(base + 28672, kLboA);
          const uint32_t acc = j > kb0 ? 1u : 0u;
          mma_tf32(tRe, arh, brh, kIdesc, acc);
          mma_tf32(tRe, arh, brl, kIdesc, 1u);
          mma_tf32(tRe, arl, brh, kIdesc, 1u);
          mma_tf32(tRe, aih, bih, kIdescNegA, 1u);
          mma_tf32(tRe, aih, bil, kIdescNegA, 1u);
          mma_tf32(tRe, ail, bih, kIdescNegA, 1u);
          mma_tf32(tIm, arh, bih, kIdesc, acc);
          mma_tf32(tIm, arh, bil, kIdesc, 1u);
          mma_tf32(tIm, arl, bih, kIdesc, 1u);
          mma_tf32(tIm, aih, brh, kIdesc, 1u);
          mma_tf32(tIm, aih, brl, kIdesc, 1u);
          mma_tf32(tIm, ail, brh, kIdesc, 1u);
          mma_commit(smem_u32(empty + stg));
          epending[stg] = 1;
        }
      }
      // the block's MMAs complete before the accumulators are read: the
      // commit of its last slab covers every earlier MMA
      for (int s2 = 0; s2 < kV2Stages && !fail; ++s2) {
        if (!epending[s2]) continue;
        if (!mbar_wait(smem_u32(empty + s2), ephase[s2])) { fail = true; break; }
        ephase[s2] ^= 1u;
        epending[s2] = 0;
      }
      if (fail) *s_fail = 1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (*s_fail) break;
    tc_epilogue<128>(g, b, m0, n0, tRe, tIm, eAB, kb0 == 0);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (*s_fail) {
    // nothing may still write the stages or the tensor memory when they are
    // released: wait (bounded) for every outstanding copy and commit
    if (tid == 0) {
      for (int s2 = 0; s2 < kV2Stages; ++s2) {
        if (fpending[s2]) mbar_wait(smem_u32(full + s2), fphase[s2]);
        if (epending[s2]) mbar_wait(smem_u32(empty + s2), ephase[s2]);
      }
      atomicExch(err, 1);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Tile::kTmemCols)
                 : "memory");
}

}  // namespace

size_t zgemm_tf32x3_planes_bytes(int M, int N, int K, int batch) {
  return sizeof(float) * 4 * 1024 * (plane_blocks(M, K) + plane_blocks(N, K)) * (size_t)batch;
}

cudaError_t zgemm_tf32x3_batched(const GemmArgs& g, int* scale_ws, int* err, cudaStream_t st, int tile_n,
                                 float* planes, size_t planes_bytes) {
  if (g.batch <= 0 || g.M <= 0 || g.N <= 0) return cudaSuccess;
  if (g.K <= 0 || g.transA || g.transB || g.s || !err || !scale_ws || (tile_n != 128 && tile_n != 256))
    return cudaErrorInvalidValue;
  if (planes && tile_n == 128 && planes_bytes >= zgemm_tf32x3_planes_bytes(g.M, g.N, g.K, g.batch)) {
    // operands split once into TF32 planes, slabs moved by bulk copies
    static SmemAttrOnce attr_split;
    cudaError_t e = attr_split.ensure(zgemm_tf32x3_split_kernel, (int)kV2Smem);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(scale_ws, 0x80, sizeof(int) * 2 * g.batch, st);
    if (e != cudaSuccess) return e;
    tc_scale_kernel<<<dim3(16, g.batch, 2), 256, 0, st>>>(g, scale_ws);
    ++launch_counter();
    float* pA = planes;
    float* pB = planes + 4 * 1024 * plane_blocks(g.M, g.K) * (size_t)g.batch;
    const size_t thrA = plane_blocks(g.M, g.K) * 256, thrB = plane_blocks(g.N, g.K) * 256;
    tc_split_kernel<<<dim3((unsigned)std::min<size_t>((thrA + 255) / 256, 4096), g.batch), 256, 0, st>>>(g, scale_ws,
                                                                                                      0, pA);
    ++launch_counter();
    tc_split_kernel<<<dim3((unsigned)std::min<size_t>((thrB + 255) / 256, 4096), g.batch), 256, 0, st>>>(g, scale_ws,
                                                                                                      1, pB);
    ++launch_counter();
    dim3 grid((g.N + 127) / 128, (g.M + kTcM - 1) / kTcM, g.batch);
    zgemm_tf32x3_split_kernel<<<grid, kTcThreads, kV2Smem, st>>>(g, scale_ws, pA, pB, err);
    ++launch_counter();
    return cudaGetLastError();
  }
  static SmemAttrOnce attr128, attr256;
  cudaError_t e = tile_n == 128 ? attr128.ensure(zgemm_tf32x3_kernel<128>, (int)TcTile<128>::kSmem)
                                : attr256.ensure(zgemm_tf32x3_kernel<256>, (int)TcTile<256>::kSmem);
  if (e != cudaSuccess) return e;
  // 0x80 bytes: every exponent starts at a very negative value
  e = cudaMemsetAsync(scale_ws, 0x80, sizeof(int) * 2 * g.batch, st);
  if (e != cudaSuccess) return e;
  tc_scale_kernel<<<dim3(16, g.batch, 2), 256, 0, st>>>(g, scale_ws);
  ++launch_counter();
  dim3 grid((g.N + tile_n - 1) / tile_n, (g.M + kTcM - 1) / kTcM, g.batch);
  if (tile_n == 128)
    zgemm_tf32x3_kernel<128><<<grid, kTcThreads, TcTile<128>::kSmem, st>>>(g, scale_ws, err);
  else
    zgemm_tf32x3_kernel<256><<<grid, kTcThreads, TcTile<256>::kSmem, st>>>(g, scale_ws, err);
  ++launch_counter();
  return cudaGetLastError();
}
