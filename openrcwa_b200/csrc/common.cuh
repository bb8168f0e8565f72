// Shared device helpers for the RCWA engine: complex FP64 arithmetic on
// double2, status codes and launch checking.  All matrices are complex128
// stored as double2 (re, im); unless a kernel says otherwise they are
// row-major with an explicit leading dimension.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "../../include/rcwa_b200.h"

typedef double2 cplx;

#define RCWA_HD __host__ __device__ __forceinline__

RCWA_HD cplx mkc(double re, double im) { return make_double2(re, im); }
RCWA_HD cplx cadd(cplx a, cplx b) { return mkc(a.x + b.x, a.y + b.y); }
RCWA_HD cplx csub(cplx a, cplx b) { return mkc(a.x - b.x, a.y - b.y); }
RCWA_HD cplx cneg(cplx a) { return mkc(-a.x, -a.y); }
RCWA_HD cplx cconj(cplx a) { return mkc(a.x, -a.y); }
RCWA_HD cplx cscale(cplx a, double s) { return mkc(a.x * s, a.y * s); }
RCWA_HD cplx cmul(cplx a, cplx b) { return mkc(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
// a*b + c with fused multiply-adds
RCWA_HD cplx cfma(cplx a, cplx b, cplx c) {
  return mkc(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
// conj(a)*b + c
RCWA_HD cplx cfmaconj(cplx a, cplx b, cplx c) {
  return mkc(fma(a.x, b.x, fma(a.y, b.y, c.x)), fma(a.x, b.y, fma(-a.y, b.x, c.y)));
}
RCWA_HD double cabs1(cplx a) { return fabs(a.x) + fabs(a.y); }
RCWA_HD double cnorm2(cplx a) { return a.x * a.x + a.y * a.y; }
RCWA_HD double cabs(cplx a) { return hypot(a.x, a.y); }

// Complex division by Smith's algorithm (R. L. Smith, CACM 5(8), 1962).
RCWA_HD cplx cdiv(cplx a, cplx b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, d = b.x + b.y * r;
    return mkc((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  } else {
    double r = b.x / b.y, d = b.y + b.x * r;
    return mkc((a.x * r + a.y) / d, (a.y * r - a.x) / d);
  }
}

// Principal complex square root (branch cut on the negative real axis, the
// sign of a zero imaginary part selects the side), from the half-angle
// identities: for z = x + iy, t = sqrt((|x| + |z|)/2); if x >= 0 the root is
// (t, y/(2t)), otherwise (|y|/(2t), copysign(t, y)).
RCWA_HD cplx csqrt_principal(cplx z) {
  double x = z.x, y = z.y;
  if (x == 0.0 && y == 0.0) return mkc(0.0, y);
  double t = sqrt(0.5 * (fabs(x) + hypot(x, y)));
  if (x >= 0.0) return mkc(t, y / (2.0 * t));
  return mkc(fabs(y) / (2.0 * t), copysign(t, y));
}

RCWA_HD cplx cexp_(cplx z) {
  double e = exp(z.x);
  double s, c;
  sincos(z.y, &s, &c);
  return mkc(e * c, e * s);
}

// GammaSqrtOp of the reference: principal root, negated when Im < 0, then
// negated again when |Im| < |Re| and Re < 0.
RCWA_HD cplx gamma_sqrt(cplx g) {
  cplx v = csqrt_principal(g);
  if (v.y < 0) v = cneg(v);
  if (fabs(v.y) < fabs(v.x) && v.x < 0) v = cneg(v);
  return v;
}

#define RCWA_DBL_EPS 1.1102230246251565e-16   // unit roundoff 2^-53
#define RCWA_DBL_MIN 2.2250738585072014e-308

// Kernel launches issued by the calling host thread; plan execution reports
// the difference over its launch sequence.
inline long long& launch_counter() {
  static thread_local long long count = 0;
  return count;
}

// Raises a kernel's dynamic shared-memory limit once per device (the
// attribute is held per device and per kernel).  Several host threads may make
// their first launch at the same time, so the per-device flags sit behind a
// mutex; later calls only take the uncontended lock.
struct SmemAttrOnce {
  std::mutex mu;
  bool done[64] = {};
  template <class Kernel>
  cudaError_t ensure(Kernel kernel, int bytes) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev] = true;
    return e;
  }
};

// Host-side launch check used by the engine.
#define RCWA_CUDA_TRY(expr)                                   \
  do {                                                        \
    cudaError_t err__ = (expr);                               \
    if (err__ != cudaSuccess) return RCWA_ERR_CUDA;           \
  } while (0)

// Stage timer: CUDA events recorded on the launching stream between groups of
// launches; the time between consecutive marks is charged to the stage named
// by the later mark.  Used only when the caller enables plan profiling.
enum RcwaStage {
  kStConvTables = 0, kStConvGather, kStConvInverse, kStPQGemm, kStAssemble, kStHessenberg, kStSchur,
  kStTrevc, kStBackTransform, kStNormalize, kStModes, kStHalfspace, kStInterface, kStPhase, kStCascadeGemm,
  kStTau, kStScatter, kStInterfaceLU, kStTauLU, kStCount
};

struct StageProf {
  bool on = false;
  int used = 0;
  cudaEvent_t ev[8192];
  int stage[8192];
  bool created = false;
  void begin(cudaStream_t st) {
    if (!on) return;
    if (!created) {
      for (int i = 0; i < 8192; ++i) cudaEventCreate(&ev[i]);
      created = true;
    }
    used = 0;
    stage[used] = -1;
    record(ev[used++], st);
  }
  void mark(cudaStream_t st, int s) {
    if (!on || used >= 8192) return;
    stage[used] = s;
    record(ev[used++], st);
  }
  // While the stream is being captured into a graph the record becomes an
  // external event node, so stage times also come out of graph launches (the
  // external flag is only valid during capture).
  static void record(cudaEvent_t e, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusActive)
      cudaEventRecordWithFlags(e, st, cudaEventRecordExternal);
    else
      cudaEventRecord(e, st);
  }
  void collect(double* ms_per_stage) {
    for (int i = 0; i < kStCount; ++i) ms_per_stage[i] = 0.0;
    for (int i = 1; i < used; ++i) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[i - 1], ev[i]);
      if (stage[i] >= 0 && stage[i] < kStCount) ms_per_stage[stage[i]] += t;
    }
  }
  ~StageProf() {
    if (created)
      for (int i = 0; i < 8192; ++i) cudaEventDestroy(ev[i]);
  }
};

// Asynchronous 16-byte global->shared copies (cp.async, bypassing L1); many
// can be in flight per thread.  cp_async_wait_all() waits for the calling
// thread's copies; a barrier then publishes them to the other threads.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
