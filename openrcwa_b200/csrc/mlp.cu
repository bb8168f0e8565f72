// Learned surrogate: a fully connected network (GELU hidden layers) that maps
// grating parameters to per-order efficiencies, trained and evaluated on the
// GPU by the kernels of this file.
//
//   training    FP32 master weights; forward and backward products by a tiled
//               FP32 GEMM; GELU, bias, mean-squared-error and Adam kernels
//   inference   BF16 weights and activations, FP32 accumulation, on tcgen05
//               (kind::f16): one 128-row CTA tile per launch row block, the
//               whole layer width N (<= 256) in one TMEM accumulator, bias and
//               GELU fused into the epilogue
//
// No counterpart in the reference; the engine's plain FP64 solve is the
// surrogate's fallback and the reference for its error (host side,
// openrcwa_b200/surrogate.py).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_bf16.h>

#include "engine_internal.cuh"

namespace {

// ---------------------------------------------------------------- FP32 training kernels
constexpr int kSgT = 64, kSgK = 16;

// C = alpha * op(A) * op(B) + beta * C, row-major, op = transpose when t = 1;
// op(A) is M x K, op(B) is K x N.  64 x 64 tile per CTA of 256 threads, 4 x 4
// outputs per thread.
__global__ void __launch_bounds__(256) sgemm_kernel(int M, int N, int K, const float* __restrict__ A, int lda, int ta,
                                                    const float* __restrict__ B, int ldb, int tb, float* C, int ldc,
                                                    float alpha, float beta) {
  __shared__ float As[kSgK][kSgT + 1];
  __shared__ float Bs[kSgK][kSgT + 1];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.y * kSgT, n0 = blockIdx.x * kSgT;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += kSgK) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int idx = tid + 256 * r;
      int mm, kk;
      if (!ta) { kk = idx & 15; mm = idx >> 4; } else { mm = idx & 63; kk = idx >> 6; }
      const int gm = m0 + mm, gk = k0 + kk;
      float v = 0.f;
      if (gm < M && gk < K) v = ta ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
      As[kk][mm] = v;
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int idx = tid + 256 * r;
      int nn, kk;
      if (!tb) { nn = idx & 63; kk = idx >> 6; } else { kk = idx & 15; nn = idx >> 4; }
      const int gn = n0 + nn, gk = k0 + kk;
      float v = 0.f;
      if (gn < N && gk < K) v = tb ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn];
      Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kSgK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty + 16 * i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx + 16 * j;
      if (n >= N) continue;
      float v = alpha * acc[i][j];
      if (beta != 0.f) v = fmaf(beta, C[(size_t)m * ldc + n], v);
      C[(size_t)m * ldc + n] = v;
    }
  }
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// Z += bias (per column); H = gelu(Z) when act (H may be null)
__global__ void bias_act_kernel(float* Z, float* H, const float* bias, int rows, int cols, int act) {
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < (size_t)rows * cols;
       idx += (size_t)gridDim.x * blockDim.x) {
    const float z = Z[idx] + bias[idx % cols];
    Z[idx] = z;
    if (H) H[idx] = act ? gelu(z) : z;
  }
}

// dZ = dH * gelu'(Z)
__global__ void gelu_back_kernel(float* dZ, const float* dH, const float* Z, size_t count) {
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < count; idx += (size_t)gridDim.x * blockDim.x)
    dZ[idx] = dH[idx] * gelu_grad(Z[idx]);
}

// D = (P - Y) * 2 / (rows * cols), loss partial sums of (P - Y)^2
__global__ void mse_kernel(const float* P, const float* Y, float* D, int rows, int cols, double* loss) {
  double part = 0.0;
  const float s = 2.f / ((float)rows * (float)cols);
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < (size_t)rows * cols;
       idx += (size_t)gridDim.x * blockDim.x) {
    const float d = P[idx] - Y[idx];
    D[idx] = d * s;
    part += (double)d * d;
  }
  for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(0xffffffffu, part, off);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, part);
}

// db[c] = sum over rows of dZ[r][c]
__global__ void colsum_kernel(const float* dZ, float* db, int rows, int cols) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (int r = 0; r < rows; ++r) s += dZ[(size_t)r * cols + c];
  db[c] = s;
}

// Adam (Kingma and Ba, ICLR 2015) on every parameter
__global__ void adam_kernel(float* w, const float* g, float* m, float* v, size_t count, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// gather rows idx[r] of X (cols wide) into out
__global__ void gather_rows_kernel(const float* X, const int* idx, float* out, int rows, int cols) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < (size_t)rows * cols;
       k += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(k / cols), c = (int)(k % cols);
    out[k] = X[(size_t)idx[r] * cols + c];
  }
}

inline dim3 ew(size_t count) {
  size_t b = (count + 255) / 256;
  return dim3((unsigned)(b > 4096 ? 4096 : (b ? b : 1)));
}

}  // namespace

namespace {

// ---------------------------------------------------------------- BF16 inference on tcgen05
constexpr int kInfM = 128, kInfK = 64, kInfThreads = 128;
constexpr long kInfWait = 1L << 22;

__device__ __forceinline__ uint32_t s_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// byte offset of (row r, k) in a K-major BF16 plane of 8 x 16-byte core matrices
__device__ __forceinline__ uint32_t bf_off(int r, int k, uint32_t lbo) {
  return (uint32_t)(k >> 3) * lbo + (uint32_t)(r >> 3) * 128u + (uint32_t)(r & 7) * 16u + (uint32_t)(k & 7) * 2u;
}

__device__ __forceinline__ bool inf_wait(uint32_t mbar, uint32_t parity) {
  for (long it = 0; it < kInfWait; ++it) {
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

// Y[rows x N] = act(X[rows x K] W[N x K]^T + b); X, W BF16 with leading
// dimensions that are multiples of 8 and K padded with zeros to kp (a
// multiple of 16); Y BF16 (yb) or FP32 (yf).  np = N rounded up to 16 (<= 256),
// tcols = TMEM columns (power of two >= np).
__global__ void __launch_bounds__(kInfThreads, 1) mlp_layer_tc_kernel(const __nv_bfloat16* X, int ldx, int rows,
                                                                      const __nv_bfloat16* W, int ldw, int N, int np,
                                                                      int kp, const float* bias, int act,
                                                                      __nv_bfloat16* yb, float* yf, int ldy, int tcols,
                                                                      int* err) {
  extern __shared__ __align__(1024) unsigned char ism[];
  const uint32_t lboA = (kInfM / 8) * 128u, lboB = (uint32_t)(np / 8) * 128u;
  unsigned char* As = ism;                                  // kInfM x kInfK
  unsigned char* Bs = ism + kInfM * kInfK * 2;              // np x kInfK
  uint64_t* mbar = reinterpret_cast<uint64_t*>(Bs + 256 * kInfK * 2);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
  int* fail = reinterpret_cast<int*>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kInfM;
  const uint32_t mb = s_u32(mbar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s_u32(tslot)), "r"(tcols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(np >> 3) << 17) | ((uint32_t)(kInfM >> 4) << 24);
  uint32_t phase = 0;
  int pending = 0;
  for (int k0 = 0; k0 < kp; k0 += kInfK) {
    if (pending) {
      if (inf_wait(mb, phase)) { phase ^= 1u; pending = 0; } else { *fail = 1; }
    }
    __syncthreads();
    if (*fail) break;
    const int kc = min(kInfK, kp - k0);  // multiple of 16
    // A rows: thread = row, 16-byte chunks of 8 elements
    {
      const int gm = m0 + tid;
      for (int q = 0; q < kc / 8; ++q) {
        uint4 v = make_uint4(0, 0, 0, 0);
        if (gm < rows) v = *reinterpret_cast<const uint4*>(X + (size_t)gm * ldx + k0 + 8 * q);
        *reinterpret_cast<uint4*>(As + bf_off(tid, 8 * q, lboA)) = v;
      }
    }
    for (int r = tid; r < np; r += kInfThreads) {
      for (int q = 0; q < kc / 8; ++q) {
        uint4 v = make_uint4(0, 0, 0, 0);
        if (r < N) v = *reinterpret_cast<const uint4*>(W + (size_t)r * ldw + k0 + 8 * q);
        *reinterpret_cast<uint4*>(Bs + bf_off(r, 8 * q, lboB)) = v;
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int ks = 0; ks < kc / 16; ++ks) {
        const uint64_t da = umma_desc(s_u32(As) + 2 * ks * lboA, lboA, 128);
        const uint64_t db = umma_desc(s_u32(Bs) + 2 * ks * lboB, lboB, 128);
        const uint32_t acc = (k0 > 0 || ks > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
            :
            : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb)
                   : "memory");
    }
    pending = 1;
  }
  if (pending && !inf_wait(mb, phase)) *fail = 1;
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (*fail) {
    if (tid == 0) atomicExch(err, 1);
  } else {
    const int m = m0 + 32 * warp + lane;
    for (int cb = 0; cb < np; cb += 16) {
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(tmem + ((uint32_t)(32 * warp) << 16) + cb));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (m < rows) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = cb + j;
          if (n < N) {
            float z = __uint_as_float(v[j]) + bias[n];
            if (act) z = gelu(z);
            if (yb) yb[(size_t)m * ldy + n] = __float2bfloat16(z);
            else yf[(size_t)m * ldy + n] = z;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tcols) : "memory");
}

// FP32 -> BF16 with zero padding: out[r][c] for c < cout (c >= cin -> 0)
__global__ void to_bf16_pad_kernel(const float* in, int cin, __nv_bfloat16* out, int cout, int rows) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < (size_t)rows * cout;
       k += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(k / cout), c = (int)(k % cout);
    out[k] = __float2bfloat16(c < cin ? in[(size_t)r * cin + c] : 0.f);
  }
}

}  // namespace

// ---------------------------------------------------------------- host side
struct rcwa_mlp {
  rcwa_engine* e = nullptr;
  int n_in = 0, n_hidden = 0, n_layers = 0, n_out = 0;  // n_layers hidden layers
  std::vector<int> dims;                                 // n_in, n_hidden x n_layers, n_out
  std::vector<size_t> w_off, b_off;                      // parameter offsets per layer
  size_t n_params = 0;
  float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  long long adam_t = 0;
  // training set
  float *X = nullptr, *Y = nullptr;
  int n_data = 0;
  // per-batch work (sized for max_batch rows)
  int max_batch = 0;
  std::vector<float*> Z, H;  // Z[l]: pre-activation of layer l; H[l]: its input (H[0] = batch inputs)
  float *Yb = nullptr, *D = nullptr, *dH = nullptr, *dZ = nullptr;
  int* idx = nullptr;
  double* loss = nullptr;
  // inference (BF16 on tcgen05)
  std::vector<__nv_bfloat16*> Wb;   // per layer, out x round16(in)
  int inf_rows = 0;
  std::vector<__nv_bfloat16*> act;  // per layer input, rows x round16(width), zero padded
  float* out = nullptr;
  int* err = nullptr;
};

namespace {

int round16(int x) { return (x + 15) / 16 * 16; }

template <class T>
bool dalloc(T** p, size_t count) {
  return cudaMalloc((void**)p, sizeof(T) * (count ? count : 1)) == cudaSuccess;
}

int mlp_fail(rcwa_mlp* m, int code, const char* msg) {
  if (m && m->e) m->e->last_error = msg;
  return code;
}

cudaError_t sgemm(int M, int N, int K, const float* A, int lda, int ta, const float* B, int ldb, int tb, float* C,
                  int ldc, float alpha, float beta, cudaStream_t st) {
  dim3 grid((N + kSgT - 1) / kSgT, (M + kSgT - 1) / kSgT);
  sgemm_kernel<<<grid, 256, 0, st>>>(M, N, K, A, lda, ta, B, ldb, tb, C, ldc, alpha, beta);
  ++launch_counter();
  return cudaGetLastError();
}

void free_batch(rcwa_mlp* m) {
  for (auto p : m->Z) cudaFree(p);
  for (auto p : m->H) cudaFree(p);
  m->Z.clear();
  m->H.clear();
  cudaFree(m->Yb); cudaFree(m->D); cudaFree(m->dH); cudaFree(m->dZ); cudaFree(m->idx);
  m->Yb = m->D = m->dH = m->dZ = nullptr;
  m->idx = nullptr;
  m->max_batch = 0;
}

bool ensure_batch(rcwa_mlp* m, int rows) {
  if (rows <= m->max_batch) return true;
  free_batch(m);
  const int L = (int)m->dims.size() - 1;
  m->Z.assign(L, nullptr);
  m->H.assign(L, nullptr);
  int wmax = 0;
  for (int d : m->dims) wmax = std::max(wmax, d);
  bool ok = true;
  for (int l = 0; l < L; ++l) {
    ok = ok && dalloc(&m->Z[l], (size_t)rows * m->dims[l + 1]);
    ok = ok && dalloc(&m->H[l], (size_t)rows * m->dims[l]);
  }
  ok = ok && dalloc(&m->Yb, (size_t)rows * m->n_out) && dalloc(&m->D, (size_t)rows * m->n_out) &&
       dalloc(&m->dH, (size_t)rows * wmax) && dalloc(&m->dZ, (size_t)rows * wmax) && dalloc(&m->idx, rows);
  if (ok) m->max_batch = rows;
  else free_batch(m);
  return ok;
}

// forward over H[0] (rows x n_in); the outputs land in Z[L-1]
cudaError_t forward_fp32(rcwa_mlp* m, int rows, cudaStream_t st) {
  const int L = (int)m->dims.size() - 1;
  cudaError_t err = cudaSuccess;
  for (int l = 0; l < L && err == cudaSuccess; ++l) {
    const int in = m->dims[l], out = m->dims[l + 1];
    err = sgemm(rows, out, in, m->H[l], in, 0, m->params + m->w_off[l], in, 1, m->Z[l], out, 1.f, 0.f, st);
    if (err != cudaSuccess) break;
    const bool hidden = l + 1 < L;
    bias_act_kernel<<<ew((size_t)rows * out), 256, 0, st>>>(m->Z[l], hidden ? m->H[l + 1] : nullptr,
                                                            m->params + m->b_off[l], rows, out, hidden ? 1 : 0);
    ++launch_counter();
    err = cudaGetLastError();
  }
  return err;
}

// mean squared error against Yb and its gradient with respect to every parameter
cudaError_t backward_fp32(rcwa_mlp* m, int rows, cudaStream_t st) {
  const int L = (int)m->dims.size() - 1;
  cudaError_t err = cudaMemsetAsync(m->loss, 0, sizeof(double), st);
  mse_kernel<<<ew((size_t)rows * m->n_out), 256, 0, st>>>(m->Z[L - 1], m->Yb, m->D, rows, m->n_out, m->loss);
  ++launch_counter();
  const float* dz = m->D;
  for (int l = L - 1; l >= 0 && err == cudaSuccess; --l) {
    const int in = m->dims[l], out = m->dims[l + 1];
    // dW = dZ^T H, db = column sums of dZ
    err = sgemm(out, in, rows, dz, out, 1, m->H[l], in, 0, m->grads + m->w_off[l], in, 1.f, 0.f, st);
    colsum_kernel<<<(out + 127) / 128, 128, 0, st>>>(dz, m->grads + m->b_off[l], rows, out);
    ++launch_counter();
    if (l > 0 && err == cudaSuccess) {
      // dH = dZ W, then dZ of the layer below = dH * gelu'(Z); stream order
      // lets the new dZ overwrite the buffer this iteration read
      err = sgemm(rows, in, out, dz, out, 0, m->params + m->w_off[l], in, 0, m->dH, in, 1.f, 0.f, st);
      gelu_back_kernel<<<ew((size_t)rows * in), 256, 0, st>>>(m->dZ, m->dH, m->Z[l - 1], (size_t)rows * in);
      ++launch_counter();
      dz = m->dZ;
    }
    if (err == cudaSuccess) err = cudaGetLastError();
  }
  return err;
}

}  // namespace

extern "C" {

void rcwa_mlp_destroy(rcwa_mlp* m) {
  if (!m) return;
  cudaSetDevice(m->e->device);
  cudaDeviceSynchronize();
  free_batch(m);
  cudaFree(m->params); cudaFree(m->grads); cudaFree(m->adam_m); cudaFree(m->adam_v);
  cudaFree(m->X); cudaFree(m->Y); cudaFree(m->loss);
  for (auto p : m->Wb) cudaFree(p);
  for (auto p : m->act) cudaFree(p);
  cudaFree(m->out); cudaFree(m->err);
  delete m;
}

int rcwa_mlp_create(rcwa_engine* e, int n_in, int n_hidden, int n_layers, int n_out, unsigned long long seed,
                    rcwa_mlp** out) {
  if (!e || !out || n_in < 1 || n_hidden < 1 || n_hidden > 256 || n_layers < 1 || n_out < 1 || n_out > 256)
    return RCWA_ERR_INVALID;
  *out = nullptr;
  if (cudaSetDevice(e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  rcwa_mlp* m = new rcwa_mlp();
  m->e = e;
  m->n_in = n_in; m->n_hidden = n_hidden; m->n_layers = n_layers; m->n_out = n_out;
  m->dims.push_back(n_in);
  for (int l = 0; l < n_layers; ++l) m->dims.push_back(n_hidden);
  m->dims.push_back(n_out);
  const int L = (int)m->dims.size() - 1;
  for (int l = 0; l < L; ++l) {
    m->w_off.push_back(m->n_params);
    m->n_params += (size_t)m->dims[l + 1] * m->dims[l];
    m->b_off.push_back(m->n_params);
    m->n_params += m->dims[l + 1];
  }
  // uniform initialisation with bound sqrt(6 / fan_in) (He et al. 2015), zero biases;
  // a 64-bit linear congruential generator keeps it reproducible
  std::vector<float> h(m->n_params, 0.f);
  unsigned long long s = seed * 6364136223846793005ull + 1442695040888963407ull;
  for (int l = 0; l < L; ++l) {
    const float bound = std::sqrt(6.f / (float)m->dims[l]);
    for (size_t i = 0; i < (size_t)m->dims[l + 1] * m->dims[l]; ++i) {
      s = s * 6364136223846793005ull + 1442695040888963407ull;
      const float u = (float)((s >> 11) * (1.0 / 9007199254740992.0));
      h[m->w_off[l] + i] = bound * (2.f * u - 1.f);
    }
  }
  bool ok = dalloc(&m->params, m->n_params) && dalloc(&m->grads, m->n_params) && dalloc(&m->adam_m, m->n_params) &&
            dalloc(&m->adam_v, m->n_params) && dalloc(&m->loss, 1) && dalloc(&m->err, 1);
  ok = ok && cudaMemcpy(m->params, h.data(), sizeof(float) * m->n_params, cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemset(m->adam_m, 0, sizeof(float) * m->n_params) == cudaSuccess &&
       cudaMemset(m->adam_v, 0, sizeof(float) * m->n_params) == cudaSuccess &&
       cudaDeviceSynchronize() == cudaSuccess;
  if (!ok) {
    rcwa_mlp_destroy(m);
    return RCWA_ERR_NOMEM;
  }
  *out = m;
  return RCWA_OK;
}

long long rcwa_mlp_param_count(const rcwa_mlp* m) { return m ? (long long)m->n_params : 0; }

int rcwa_mlp_get_params(rcwa_mlp* m, float* params) {
  if (!m || !params) return RCWA_ERR_INVALID;
  if (cudaSetDevice(m->e->device) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return RCWA_ERR_CUDA;
  return cudaMemcpy(params, m->params, sizeof(float) * m->n_params, cudaMemcpyDeviceToHost) == cudaSuccess
             ? RCWA_OK : RCWA_ERR_CUDA;
}

int rcwa_mlp_set_params(rcwa_mlp* m, const float* params) {
  if (!m || !params) return RCWA_ERR_INVALID;
  if (cudaSetDevice(m->e->device) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return RCWA_ERR_CUDA;
  return cudaMemcpy(m->params, params, sizeof(float) * m->n_params, cudaMemcpyHostToDevice) == cudaSuccess
             ? RCWA_OK : RCWA_ERR_CUDA;
}

}  // extern "C"

namespace {
// Squared distance from every query row to its nearest row of the training
// set (both n_in features, FP32).  A block takes 128 queries and a slice of
// the training rows, staged through shared memory 128 rows at a time; the
// per-slice minima combine by atomicMin on the (non-negative) float bits.
// With skip_self, a training row at distance exactly 0 (the query itself,
// for leave-one-out distances of training rows) is not counted.
constexpr int kNnThreads = 128;
constexpr int kNnMaxDim = 32;

__global__ void __launch_bounds__(kNnThreads) nn_distance_kernel(const float* __restrict__ ref, int n_ref,
                                                                 const float* __restrict__ q, int n_q, int dim,
                                                                 int slice, int skip_self, unsigned* d2_bits) {
  __shared__ float tile[kNnThreads * kNnMaxDim];
  const int qi = blockIdx.x * kNnThreads + threadIdx.x;
  float x[kNnMaxDim];
#pragma unroll
  for (int k = 0; k < kNnMaxDim; ++k) x[k] = (qi < n_q && k < dim) ? q[(size_t)qi * dim + k] : 0.0f;
  float best = INFINITY;
  const int r0 = blockIdx.y * slice, r1 = min(n_ref, r0 + slice);
  for (int t0 = r0; t0 < r1; t0 += kNnThreads) {
    const int rows = min(kNnThreads, r1 - t0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < rows * dim; idx += kNnThreads) tile[idx] = ref[(size_t)t0 * dim + idx];
    __syncthreads();
    for (int r = 0; r < rows; ++r) {
      float d = 0.0f;
#pragma unroll
      for (int k = 0; k < kNnMaxDim; ++k)
        if (k < dim) {
          const float e = x[k] - tile[r * dim + k];
          d = fmaf(e, e, d);
        }
      if (!(skip_self && d == 0.0f)) best = fminf(best, d);
    }
  }
  if (qi < n_q) atomicMin(&d2_bits[qi], __float_as_uint(best));
}
}  // namespace

extern "C" {

// Nearest-neighbour distances of query rows Q [n][n_in] (host, the features
// the network was trained on) to the training set of rcwa_mlp_set_data: d2[n]
// receives the squared Euclidean distance to the nearest training row.  With
// skip_self, distances of exactly 0 are ignored (queries that are training
// rows get their leave-one-out distance).  The surrogate's hull test.
int rcwa_mlp_nn_distance(rcwa_mlp* m, const float* Q, int n, int skip_self, float* d2) {
  if (!m || !Q || !d2 || n < 1) return RCWA_ERR_INVALID;
  if (!m->X || m->n_data < 1) return mlp_fail(m, RCWA_ERR_INVALID, "no training set");
  if (m->n_in > kNnMaxDim) return mlp_fail(m, RCWA_ERR_UNSUPPORTED, "more than 32 input features");
  if (cudaSetDevice(m->e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  float* dq = nullptr;
  unsigned* dd = nullptr;
  if (!dalloc(&dq, (size_t)n * m->n_in) || !dalloc(&dd, (size_t)n)) {
    cudaFree(dq);
    return mlp_fail(m, RCWA_ERR_NOMEM, "query allocation failed");
  }
  cudaStream_t st = m->e->stream;
  int rc = RCWA_OK;
  if (cudaMemcpyAsync(dq, Q, sizeof(float) * n * m->n_in, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemsetAsync(dd, 0x7f, sizeof(unsigned) * n, st) != cudaSuccess) {
    rc = RCWA_ERR_CUDA;
  } else {
    // training rows split into slices so that the grid covers the SMs
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->e->device);
    const int qblocks = (n + kNnThreads - 1) / kNnThreads;
    const int nslices = std::max(1, std::min((m->n_data + kNnThreads - 1) / kNnThreads, (4 * sms + qblocks - 1) / qblocks));
    const int slice = ((m->n_data + nslices - 1) / nslices + kNnThreads - 1) / kNnThreads * kNnThreads;
    const int ns = (m->n_data + slice - 1) / slice;
    nn_distance_kernel<<<dim3(qblocks, ns), kNnThreads, 0, st>>>(m->X, m->n_data, dq, n, m->n_in, slice,
                                                                 skip_self ? 1 : 0, dd);
    ++launch_counter();
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(d2, dd, sizeof(float) * n, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      rc = RCWA_ERR_CUDA;
  }
  cudaFree(dq);
  cudaFree(dd);
  return rc;
}

int rcwa_mlp_set_data(rcwa_mlp* m, const float* X, const float* Y, int n) {
  if (!m || !X || !Y || n < 1) return RCWA_ERR_INVALID;
  if (cudaSetDevice(m->e->device) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return RCWA_ERR_CUDA;
  cudaFree(m->X);
  cudaFree(m->Y);
  m->X = m->Y = nullptr;
  m->n_data = 0;
  if (!dalloc(&m->X, (size_t)n * m->n_in) || !dalloc(&m->Y, (size_t)n * m->n_out))
    return mlp_fail(m, RCWA_ERR_NOMEM, "training set allocation failed");
  if (cudaMemcpy(m->X, X, sizeof(float) * n * m->n_in, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(m->Y, Y, sizeof(float) * n * m->n_out, cudaMemcpyHostToDevice) != cudaSuccess)
    return RCWA_ERR_CUDA;
  m->n_data = n;
  return RCWA_OK;
}

// Loss (mean squared error) and its gradient for the rows X, Y (host); grad
// has rcwa_mlp_param_count entries in the parameter layout (per layer W then b).
int rcwa_mlp_loss_grad(rcwa_mlp* m, const float* X, const float* Y, int n, double* loss, float* grad) {
  if (!m || !X || !Y || n < 1) return RCWA_ERR_INVALID;
  if (cudaSetDevice(m->e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  if (!ensure_batch(m, n)) return mlp_fail(m, RCWA_ERR_NOMEM, "batch allocation failed");
  cudaStream_t st = m->e->stream;
  if (cudaMemcpyAsync(m->H[0], X, sizeof(float) * n * m->n_in, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(m->Yb, Y, sizeof(float) * n * m->n_out, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return RCWA_ERR_CUDA;
  if (forward_fp32(m, n, st) != cudaSuccess || backward_fp32(m, n, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return mlp_fail(m, RCWA_ERR_CUDA, "training kernels failed");
  double h = 0.0;
  if (cudaMemcpy(&h, m->loss, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return RCWA_ERR_CUDA;
  if (loss) *loss = h / ((double)n * m->n_out);
  if (grad && cudaMemcpy(grad, m->grads, sizeof(float) * m->n_params, cudaMemcpyDeviceToHost) != cudaSuccess)
    return RCWA_ERR_CUDA;
  return RCWA_OK;
}

// Adam epochs over the training set in shuffled minibatches; loss[epoch] = mean
// squared error averaged over the epoch's batches.
int rcwa_mlp_train(rcwa_mlp* m, int epochs, int batch, float lr, unsigned long long seed, float* loss) {
  if (!m || epochs < 1 || batch < 1 || !(lr > 0.f) || m->n_data < 1) return RCWA_ERR_INVALID;
  if (cudaSetDevice(m->e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  batch = std::min(batch, m->n_data);
  if (!ensure_batch(m, batch)) return mlp_fail(m, RCWA_ERR_NOMEM, "batch allocation failed");
  cudaStream_t st = m->e->stream;
  std::vector<int> perm(m->n_data);
  unsigned long long s = seed * 6364136223846793005ull + 1442695040888963407ull;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int ep = 0; ep < epochs; ++ep) {
    for (int i = 0; i < m->n_data; ++i) perm[i] = i;
    for (int i = m->n_data - 1; i > 0; --i) {  // Fisher-Yates
      s = s * 6364136223846793005ull + 1442695040888963407ull;
      const int j = (int)((s >> 33) % (unsigned long long)(i + 1));
      std::swap(perm[i], perm[j]);
    }
    double sum = 0.0;
    int nb = 0;
    for (int b0 = 0; b0 + batch <= m->n_data; b0 += batch) {
      if (cudaMemcpyAsync(m->idx, perm.data() + b0, sizeof(int) * batch, cudaMemcpyHostToDevice, st) !=
          cudaSuccess)
        return RCWA_ERR_CUDA;
      gather_rows_kernel<<<ew((size_t)batch * m->n_in), 256, 0, st>>>(m->X, m->idx, m->H[0], batch, m->n_in);
      gather_rows_kernel<<<ew((size_t)batch * m->n_out), 256, 0, st>>>(m->Y, m->idx, m->Yb, batch, m->n_out);
      launch_counter() += 2;
      if (forward_fp32(m, batch, st) != cudaSuccess || backward_fp32(m, batch, st) != cudaSuccess)
        return mlp_fail(m, RCWA_ERR_CUDA, "training kernels failed");
      ++m->adam_t;
      const float c1 = 1.f - std::pow(b1, (float)m->adam_t), c2 = 1.f - std::pow(b2, (float)m->adam_t);
      adam_kernel<<<ew(m->n_params), 256, 0, st>>>(m->params, m->grads, m->adam_m, m->adam_v, m->n_params, lr, b1, b2,
                                                   eps, c1, c2);
      ++launch_counter();
      double h = 0.0;
      // the pageable copy waits for the batch (one sync per batch keeps the
      // index upload above from racing the next batch's gather)
      if (cudaMemcpyAsync(&h, m->loss, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess)
        return mlp_fail(m, RCWA_ERR_CUDA, "training step failed");
      sum += h / ((double)batch * m->n_out);
      ++nb;
    }
    if (loss) loss[ep] = nb ? (float)(sum / nb) : 0.f;
  }
  return RCWA_OK;
}

// FP32 forward of the training path (host rows in and out).
int rcwa_mlp_predict_fp32(rcwa_mlp* m, const float* X, int n, float* Y) {
  if (!m || !X || !Y || n < 1) return RCWA_ERR_INVALID;
  if (cudaSetDevice(m->e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  if (!ensure_batch(m, n)) return mlp_fail(m, RCWA_ERR_NOMEM, "batch allocation failed");
  cudaStream_t st = m->e->stream;
  const int L = (int)m->dims.size() - 1;
  if (cudaMemcpyAsync(m->H[0], X, sizeof(float) * n * m->n_in, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      forward_fp32(m, n, st) != cudaSuccess ||
      cudaMemcpyAsync(Y, m->Z[L - 1], sizeof(float) * n * m->n_out, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return mlp_fail(m, RCWA_ERR_CUDA, "forward failed");
  return RCWA_OK;
}

}  // extern "C"

namespace {
constexpr size_t kInfSmem = (size_t)kInfM * kInfK * 2 + (size_t)256 * kInfK * 2 + 64;

int pow2_cols(int np) {
  int c = 32;
  while (c < np) c <<= 1;
  return c;
}

bool ensure_inference(rcwa_mlp* m, int rows) {
  if (rows <= m->inf_rows) return true;
  for (auto p : m->act) cudaFree(p);
  cudaFree(m->out);
  m->act.assign(m->dims.size() - 1, nullptr);
  m->out = nullptr;
  m->inf_rows = 0;
  bool ok = true;
  for (size_t l = 0; l + 1 < m->dims.size(); ++l) {
    const size_t cnt = (size_t)rows * round16(m->dims[l]);
    ok = ok && dalloc(&m->act[l], cnt) && cudaMemset(m->act[l], 0, sizeof(__nv_bfloat16) * cnt) == cudaSuccess;
  }
  ok = ok && dalloc(&m->out, (size_t)rows * m->n_out);
  if (ok) m->inf_rows = rows;
  return ok;
}
}  // namespace

extern "C" {

// Inference on the tensor cores: BF16 weights and activations, FP32
// accumulation (tcgen05 kind::f16), bias and GELU in the epilogue.
int rcwa_mlp_predict(rcwa_mlp* m, const float* X, int n, float* Y) {
  if (!m || !X || !Y || n < 1) return RCWA_ERR_INVALID;
  if (cudaSetDevice(m->e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  static SmemAttrOnce attr;
  if (attr.ensure(mlp_layer_tc_kernel, (int)kInfSmem) != cudaSuccess) return RCWA_ERR_CUDA;
  const int L = (int)m->dims.size() - 1;
  if (m->Wb.empty()) {
    m->Wb.assign(L, nullptr);
    for (int l = 0; l < L; ++l)
      if (!dalloc(&m->Wb[l], (size_t)m->dims[l + 1] * round16(m->dims[l])))
        return mlp_fail(m, RCWA_ERR_NOMEM, "inference weight allocation failed");
  }
  if (!ensure_inference(m, n))
    return mlp_fail(m, RCWA_ERR_NOMEM, "inference allocation failed");
  cudaStream_t st = m->e->stream;
  float* xin = nullptr;
  if (!dalloc(&xin, (size_t)n * m->n_in)) return mlp_fail(m, RCWA_ERR_NOMEM, "input allocation failed");
  cudaError_t err = cudaMemcpyAsync(xin, X, sizeof(float) * n * m->n_in, cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess) err = cudaMemsetAsync(m->err, 0, sizeof(int), st);
  for (int l = 0; l < L && err == cudaSuccess; ++l) {
    const int kp = round16(m->dims[l]);
    to_bf16_pad_kernel<<<ew((size_t)m->dims[l + 1] * kp), 256, 0, st>>>(m->params + m->w_off[l], m->dims[l], m->Wb[l],
                                                                        kp, m->dims[l + 1]);
    ++launch_counter();
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) {
    to_bf16_pad_kernel<<<ew((size_t)n * round16(m->n_in)), 256, 0, st>>>(xin, m->n_in, m->act[0], round16(m->n_in), n);
    ++launch_counter();
    err = cudaGetLastError();
  }
  for (int l = 0; l < L && err == cudaSuccess; ++l) {
    const bool hidden = l + 1 < L;
    const int kp = round16(m->dims[l]), N = m->dims[l + 1], np = round16(N);
    mlp_layer_tc_kernel<<<(n + kInfM - 1) / kInfM, kInfThreads, kInfSmem, st>>>(
        m->act[l], kp, n, m->Wb[l], kp, N, np, kp, m->params + m->b_off[l], hidden ? 1 : 0,
        hidden ? m->act[l + 1] : nullptr, hidden ? nullptr : m->out, hidden ? np : m->n_out, pow2_cols(np), m->err);
    ++launch_counter();
    err = cudaGetLastError();
  }
  int herr = 0;
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(Y, m->out, sizeof(float) * n * m->n_out, cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaMemcpyAsync(&herr, m->err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  cudaFree(xin);
  if (err != cudaSuccess) return mlp_fail(m, RCWA_ERR_CUDA, "inference kernels failed");
  if (herr) return mlp_fail(m, RCWA_ERR_CUDA, "a tensor-core completion wait ran out");
  return RCWA_OK;
}

}  // extern "C"
