// Eigensolver entry point for callers that cannot allocate device memory.
//
// Some hosts of this library run where cudaMalloc is not available to them:
// code that executes inside another framework's memory pool or arena (which
// hands out buffers but forbids new device allocations), real-time loops where
// an allocation may stall or fail, or applications that must bound their
// device footprint up front.  rcwa_zgeev_batched_noalloc serves them: the
// caller passes its own device buffers for the inputs and outputs, and the
// eigensolver's scratch (Schur vectors, the triangular eigenvector matrix,
// Householder vectors and the per-matrix pointer tables) lives in one
// file-scope __device__ array that every GPU loading the library reserves
// until the process exits.
#include <mutex>

#include "eig.cuh"
#include "engine_internal.cuh"

namespace {

constexpr int kMaxN = RCWA_NOALLOC_MAX_N;
constexpr int kMaxBatch = RCWA_NOALLOC_MAX_BATCH;
constexpr size_t kPtrBytes = 2 * sizeof(void*) * kMaxBatch;

size_t scratch_bytes_needed(int n, int batch) { return kPtrBytes + zgeev_workspace_bytes(n) * (size_t)batch; }

// pointer tables (A and VR per matrix) followed by the eigensolver workspace;
// sized for the largest accepted call: n = 64, batch = 64 (about 38 MB)
constexpr size_t kScratchBytes = kPtrBytes + zgeev_workspace_bytes(kMaxN) * kMaxBatch;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch per device.  In host code the symbol
// name is only a stand-in, so the address is looked up once per device with
// that device current.  Under CUDA's lazy module loading (the default since
// CUDA 12.2) the driver loads this library's device code, and reserves the
// array, at that first lookup: the first call on a device is where the
// reservation can fail (a device already full), and it must not come during
// a stream capture.  Later calls touch no allocator at all.
constexpr int kMaxDevices = 64;
unsigned char* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

__global__ void fill_ptrs_kernel(cplx* A, cplx* VR, int n, int batch, cplx** ptrA, cplx** ptrV) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < batch) {
    ptrA[b] = A + (size_t)b * n * n;
    ptrV[b] = VR + (size_t)b * n * n;
  }
}

}  // namespace

extern "C" int rcwa_zgeev_batched_noalloc(int n, int batch, rcwa_cplx* A, rcwa_cplx* w, rcwa_cplx* VR, int* info,
                                          void* stream) {
  if (n < 1 || batch < 1 || !A || !w || !VR || !info) return RCWA_ERR_INVALID;
  if (n > kMaxN || batch > kMaxBatch || scratch_bytes_needed(n, batch) > kScratchBytes)
    return RCWA_ERR_UNSUPPORTED;  // beyond the static scratch: n <= 64 and batch <= 64
  // an error left pending by the caller's own earlier work is reported, not
  // cleared: it stays readable with cudaGetLastError after this call
  if (cudaPeekAtLastError() != cudaSuccess) return RCWA_ERR_CUDA;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return RCWA_ERR_CUDA;
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return RCWA_ERR_CUDA;
      g_scratch_addr[dev] = (unsigned char*)p;
    }
    base = g_scratch_addr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  cplx** ptrA = (cplx**)base;
  cplx** ptrV = ptrA + kMaxBatch;
  void* work = base + kPtrBytes;
  fill_ptrs_kernel<<<(batch + 127) / 128, 128, 0, st>>>((cplx*)A, (cplx*)VR, n, batch, ptrA, ptrV);
  ++launch_counter();
  if (cudaGetLastError() != cudaSuccess) return RCWA_ERR_CUDA;
  // every scratch region is written before it is read inside the eigensolver
  // (Z starts as the identity, X is initialised by the back-substitution),
  // so nothing left by an earlier call needs clearing
  if (zgeev_batched(ptrA, n, n, (cplx*)w, ptrV, n, work, info, batch, st) != cudaSuccess) return RCWA_ERR_CUDA;
  return RCWA_OK;
}
