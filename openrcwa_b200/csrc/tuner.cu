// Schedule autotuner: timing of the candidate schedules on this GPU, the
// engine's lookup, and the C ABI of the schedule table (create, set, get,
// list, save, load, measure).  The reference has no counterpart: its CPU path
// calls LAPACK with fixed blocking.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "eig.cuh"
#include "engine_internal.cuh"
#include "gemm_tc.cuh"
#include "linalg.cuh"
#include "tuner.cuh"

namespace {

constexpr int kSchurCand[kTuneMaxCand] = {64, 96, 128, 192};
constexpr int kSchurTuneMax = 512;
constexpr const char* kOpName[kTuneOps] = {"lu", "schur", "product"};
// device memory one measurement may take
constexpr size_t kTuneBytes = (size_t)6 << 30;

// splitmix64 of the element index: entries uniform in [-1, 1) per component
__global__ void fill_random_kernel(cplx* p, size_t count, unsigned long long seed) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (2 * i + 1);
    double v[2];
    for (int c = 0; c < 2; ++c) {
      z += 0x9E3779B97F4A7C15ull;
      unsigned long long x = z;
      x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
      x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
      x ^= x >> 31;
      v[c] = (double)(x >> 11) * (2.0 / 9007199254740992.0) - 1.0;
    }
    p[i] = mkc(v[0], v[1]);
  }
}

struct Buf {
  void* p = nullptr;
  Buf() = default;
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
  bool alloc(size_t bytes) {
    if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();  // a failed allocation must not surface at a later launch check
      return false;
    }
    return true;
  }
  ~Buf() { if (p) cudaFree(p); }
  template <class T> T* as() const { return (T*)p; }
};

struct Events {
  cudaEvent_t a = nullptr, b = nullptr;
  Events() { cudaEventCreate(&a); cudaEventCreate(&b); }
  ~Events() { if (a) cudaEventDestroy(a); if (b) cudaEventDestroy(b); }
};

cudaError_t fill(cplx* p, size_t count, unsigned long long seed, cudaStream_t st) {
  fill_random_kernel<<<1024, 256, 0, st>>>(p, count, seed);
  ++launch_counter();
  return cudaGetLastError();
}

cudaError_t upload_ptrs(Buf& dst, cplx* base, size_t stride, int count) {
  std::vector<cplx*> h(count);
  for (int i = 0; i < count; ++i) h[i] = base + stride * i;
  if (!dst.alloc(sizeof(cplx*) * count)) return cudaErrorMemoryAllocation;
  // a pageable upload may still be in flight when cudaMemcpy returns, and the
  // engine's stream does not wait for the legacy stream
  cudaError_t err = cudaMemcpy(dst.p, h.data(), sizeof(cplx*) * count, cudaMemcpyHostToDevice);
  return err == cudaSuccess ? cudaStreamSynchronize(cudaStreamLegacy) : err;
}

bool valid_op(int op) { return op >= 0 && op < kTuneOps; }

bool valid_choice(int op, int n, int choice) {
  int c[kTuneMaxCand];
  const int k = tune_candidates(op, n, c);
  for (int i = 0; i < k; ++i)
    if (c[i] == choice) return true;
  return false;
}

}  // namespace

int tune_batch_class(int batch, int sms) {
  if (sms <= 0) sms = 148;
  const int waves = (std::max(batch, 1) + sms - 1) / sms;
  return waves <= 3 ? waves : (waves < 8 ? 4 : 8);
}

int tune_candidates(int op, int n, int* out) {
  switch (op) {
    case kTuneLU:
      // 128-column blocks need room for a block and a trailing matrix
      out[0] = 0; out[1] = 1;
      if (n < 256) return 2;
      out[2] = 2;
      return 3;
    case kTuneSchur:
      // the crossover only matters while small active blocks are a large part
      // of the iteration; from 512 rows on the multishift phase dominates
      // (measured on B200: 64 fastest at n = 450, 882 and 1250), and a
      // measurement there would cost seconds per candidate
      if (n < kSchurCrossover || n >= kSchurTuneMax) { out[0] = kSchurCrossover; return 1; }
      for (int i = 0; i < kTuneMaxCand; ++i) out[i] = kSchurCand[i];
      return kTuneMaxCand;
    case kTuneProduct: out[0] = 0; out[1] = 1; out[2] = 2; return 3;
    default: return 0;
  }
}

int tune_default_sms(int op, int n, int batch, int sms) {
  switch (op) {
    case kTuneLU: return zgetrf_default_schedule(n, batch, sms);
    // whole matrices below 128 rows: the single-shift kernel (measured on
    // B200: n = 98 in 61% of the multishift kernel's time; n = 242 slower)
    case kTuneSchur: return (n >= kSchurCrossover && n < 128) ? 128 : kSchurCrossover;
    case kTuneProduct: return 0;
    default: return -1;
  }
}

int tune_default(int op, int n, int batch) { return tune_default_sms(op, n, batch, 0); }

cudaError_t tune_measure(rcwa_engine* e, int op, int n, int batch, TuneEntry& out) {
  out = TuneEntry();
  out.ncand = tune_candidates(op, n, out.cand);
  if (out.ncand <= 0 || n <= 0 || batch <= 0) return cudaErrorInvalidValue;
  if (out.ncand == 1) { out.choice = out.cand[0]; return cudaSuccess; }
  cudaStream_t st = e->stream;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
  const size_t nn = (size_t)n * n;
  const size_t per = nn * sizeof(cplx);
  // buffers per matrix: LU source + work; eigensolver source + work + vectors
  // + scratch; products A, B, D
  const size_t per_item = op == kTuneLU ? 2 * per
                          : op == kTuneSchur ? 3 * per + zgeev_workspace_bytes(n) + (size_t)n * sizeof(cplx) + 64
                                             : 3 * per + zgemm_tf32x3_planes_bytes(n, n, n, 1);
  int mb = op == kTuneSchur ? std::min(batch, sms) : batch;
  mb = (int)std::max<size_t>(1, std::min<size_t>((size_t)mb, kTuneBytes / per_item));
  Events ev;
  if (!ev.a || !ev.b) return cudaErrorUnknown;
  cudaError_t err = cudaSuccess;
  auto timed = [&](auto&& prepare, auto&& run, int reps, double& best) -> cudaError_t {
    best = 0.0;
    for (int r = 0; r < reps; ++r) {
      cudaError_t x = prepare();
      if (x != cudaSuccess) return x;
      if ((x = cudaEventRecord(ev.a, st)) != cudaSuccess) return x;
      if ((x = run()) != cudaSuccess) return x;
      if ((x = cudaEventRecord(ev.b, st)) != cudaSuccess) return x;
      if ((x = cudaEventSynchronize(ev.b)) != cudaSuccess) return x;
      float ms = 0.f;
      if ((x = cudaEventElapsedTime(&ms, ev.a, ev.b)) != cudaSuccess) return x;
      if (r == 0 || ms < best) best = ms;
    }
    return cudaSuccess;
  };

  if (op == kTuneLU) {
    Buf src, work, ipiv, info, ptrs;
    if (!src.alloc(per * mb) || !work.alloc(per * mb) || !ipiv.alloc(sizeof(int) * n * (size_t)mb) ||
        !info.alloc(sizeof(int) * mb))
      return cudaErrorMemoryAllocation;
    if ((err = upload_ptrs(ptrs, work.as<cplx>(), nn, mb)) != cudaSuccess) return err;
    if ((err = fill(src.as<cplx>(), nn * mb, 0x5EEDull + n, st)) != cudaSuccess) return err;
    for (int c = 0; c < out.ncand; ++c) {
      auto restore = [&]() { return cudaMemcpyAsync(work.p, src.p, per * mb, cudaMemcpyDeviceToDevice, st); };
      double warm = 0.0;
      // first launch of each kernel (module loading) on one matrix, then the batch
      err = timed(restore, [&]() {
        return zgetrf_batched(ptrs.as<cplx*>(), n, n, ipiv.as<int>(), info.as<int>(), 1, st, out.cand[c]); }, 1, warm);
      if (err == cudaSuccess)
        err = timed(restore, [&]() {
          return zgetrf_batched(ptrs.as<cplx*>(), n, n, ipiv.as<int>(), info.as<int>(), mb, st, out.cand[c]); },
          2, out.ms[c]);
      if (err != cudaSuccess) return err;
    }
  } else if (op == kTuneSchur) {
    Buf src, a, vr, w, wk, info, pa, pv;
    if (!src.alloc(per * mb) || !a.alloc(per * mb) || !vr.alloc(per * mb) || !w.alloc(sizeof(cplx) * n * (size_t)mb) ||
        !wk.alloc(zgeev_workspace_bytes(n) * mb) || !info.alloc(sizeof(int) * mb))
      return cudaErrorMemoryAllocation;
    if ((err = upload_ptrs(pa, a.as<cplx>(), nn, mb)) != cudaSuccess) return err;
    if ((err = upload_ptrs(pv, vr.as<cplx>(), nn, mb)) != cudaSuccess) return err;
    if ((err = fill(src.as<cplx>(), nn * mb, 0xE16ull + n, st)) != cudaSuccess) return err;
    auto restore = [&]() { return cudaMemcpyAsync(a.p, src.p, per * mb, cudaMemcpyDeviceToDevice, st); };
    for (int c = 0; c < out.ncand; ++c) {
      auto run = [&](int b) {
        return zgeev_batched(pa.as<cplx*>(), n, n, w.as<cplx>(), pv.as<cplx*>(), n, wk.p, info.as<int>(), b, st,
                             nullptr, out.cand[c]);
      };
      double warm = 0.0;
      err = timed(restore, [&]() { return run(1); }, 1, warm);
      if (err == cudaSuccess) err = timed(restore, [&]() { return run(mb); }, 1, out.ms[c]);
      if (err != cudaSuccess) return err;
    }
  } else {
    Buf A, B, D, scale, tcerr, planes;
    const size_t pbytes = zgemm_tf32x3_planes_bytes(n, n, n, mb);
    if (!A.alloc(per * mb) || !B.alloc(per * mb) || !D.alloc(per * mb) || !scale.alloc(sizeof(int) * 2 * mb) ||
        !tcerr.alloc(sizeof(int)) || !planes.alloc(pbytes))
      return cudaErrorMemoryAllocation;
    if ((err = fill(A.as<cplx>(), nn * mb, 0xA11ull + n, st)) != cudaSuccess) return err;
    if ((err = fill(B.as<cplx>(), nn * mb, 0xB22ull + n, st)) != cudaSuccess) return err;
    if ((err = cudaMemsetAsync(tcerr.p, 0, sizeof(int), st)) != cudaSuccess) return err;
    GemmArgs g{};
    g.A0 = A.as<cplx>(); g.B0 = B.as<cplx>(); g.D0 = D.as<cplx>();
    g.sA = g.sB = g.sD = nn;
    g.M = g.N = g.K = n;
    g.lda = g.ldb = g.ldc = g.ldd = n;
    g.alpha = mkc(1.0, 0.0); g.beta = mkc(0.0, 0.0); g.gammaI = mkc(0.0, 0.0);
    auto nop = []() { return cudaSuccess; };
    for (int c = 0; c < out.ncand; ++c) {
      auto run = [&](int b) {
        GemmArgs x = g;
        x.batch = b;
        return out.cand[c] == 1 ? zgemm_batched(x, st)
               : out.cand[c] == 2 ? zgemm_tf32x3_batched(x, scale.as<int>(), tcerr.as<int>(), st, 256)
                                  : zgemm_tf32x3_batched(x, scale.as<int>(), tcerr.as<int>(), st, 128,
                                                         planes.as<float>(), pbytes);
      };
      double warm = 0.0;
      err = timed(nop, [&]() { return run(1); }, 1, warm);
      if (err == cudaSuccess) err = timed(nop, [&]() { return run(mb); }, 2, out.ms[c]);
      if (err != cudaSuccess) return err;
    }
  }
  int best = 0;
  for (int c = 1; c < out.ncand; ++c)
    if (out.ms[c] < out.ms[best]) best = c;
  out.choice = out.cand[best];
  return cudaSuccess;
}

int tune_resolve(rcwa_engine* e, int op, int n, int batch) {
  int only[kTuneMaxCand];
  if (tune_candidates(op, n, only) == 1) return only[0];
  if (!e || !e->tuner || e->tuning == kTuningOff) return tune_default(op, n, batch);
  rcwa_tuner* t = e->tuner;
  const auto key = std::make_tuple(op, n, tune_batch_class(batch, t->sms));
  {
    std::lock_guard<std::mutex> lk(t->mu);
    auto it = t->table.find(key);
    if (it != t->table.end() && it->second.choice >= 0) return it->second.choice;
  }
  if (e->tuning != kTuningAuto) return tune_default(op, n, batch);
  TuneEntry ent;
  if (tune_measure(e, op, n, batch, ent) != cudaSuccess || ent.choice < 0) {
    cudaGetLastError();
    return tune_default(op, n, batch);
  }
  std::lock_guard<std::mutex> lk(t->mu);
  t->table[key] = ent;
  return ent.choice;
}

// ------------------------------------------------------------------ C ABI

extern "C" int rcwa_tuner_create(rcwa_tuner** out) {
  if (!out) return RCWA_ERR_INVALID;
  *out = new rcwa_tuner();
  return RCWA_OK;
}

extern "C" void rcwa_tuner_destroy(rcwa_tuner* t) { delete t; }

extern "C" int rcwa_tuner_set_sms(rcwa_tuner* t, int sms) {
  if (!t || sms <= 0) return RCWA_ERR_INVALID;
  std::lock_guard<std::mutex> lk(t->mu);
  t->sms = sms;
  return RCWA_OK;
}

extern "C" int rcwa_tuner_candidates(int op, int n, int* choices) {
  if (!valid_op(op) || n <= 0 || !choices) return -1;
  return tune_candidates(op, n, choices);
}

extern "C" int rcwa_tuner_default(const rcwa_tuner* t, int op, int n, int batch) {
  if (!t || !valid_op(op) || n <= 0 || batch <= 0) return -1;
  return tune_default_sms(op, n, batch, t->sms);
}

extern "C" int rcwa_tuner_set(rcwa_tuner* t, int op, int n, int batch, int choice) {
  if (!t || !valid_op(op) || n <= 0 || batch <= 0 || !valid_choice(op, n, choice)) return RCWA_ERR_INVALID;
  std::lock_guard<std::mutex> lk(t->mu);
  TuneEntry ent;
  ent.ncand = tune_candidates(op, n, ent.cand);
  ent.choice = choice;
  t->table[std::make_tuple(op, n, tune_batch_class(batch, t->sms))] = ent;
  return RCWA_OK;
}

extern "C" int rcwa_tuner_get(const rcwa_tuner* t, int op, int n, int batch, int* choice) {
  if (!t || !valid_op(op) || n <= 0 || batch <= 0 || !choice) return RCWA_ERR_INVALID;
  std::lock_guard<std::mutex> lk(t->mu);
  auto it = t->table.find(std::make_tuple(op, n, tune_batch_class(batch, t->sms)));
  *choice = it == t->table.end() ? -1 : it->second.choice;
  return RCWA_OK;
}

extern "C" int rcwa_tuner_count(const rcwa_tuner* t) {
  if (!t) return 0;
  std::lock_guard<std::mutex> lk(t->mu);
  return (int)t->table.size();
}

extern "C" int rcwa_tuner_entry(const rcwa_tuner* t, int index, int* op, int* n, int* batch_class, int* choice,
                                int* ncand, int* cand, double* ms) {
  if (!t || index < 0) return RCWA_ERR_INVALID;
  std::lock_guard<std::mutex> lk(t->mu);
  if (index >= (int)t->table.size()) return RCWA_ERR_INVALID;
  auto it = t->table.begin();
  std::advance(it, index);
  if (op) *op = std::get<0>(it->first);
  if (n) *n = std::get<1>(it->first);
  if (batch_class) *batch_class = std::get<2>(it->first);
  if (choice) *choice = it->second.choice;
  if (ncand) *ncand = it->second.ncand;
  for (int c = 0; c < kTuneMaxCand; ++c) {
    if (cand) cand[c] = c < it->second.ncand ? it->second.cand[c] : -1;
    if (ms) ms[c] = c < it->second.ncand ? it->second.ms[c] : 0.0;
  }
  return RCWA_OK;
}

// Text format, one entry per line after a header:
//   <op name> <n> <batch class> <choice> [<candidate> <ms>]...
extern "C" int rcwa_tuner_save(const rcwa_tuner* t, const char* path) {
  if (!t || !path) return RCWA_ERR_INVALID;
  std::ofstream f(path);
  if (!f) return RCWA_ERR_INVALID;
  std::lock_guard<std::mutex> lk(t->mu);
  f << "# rcwa_b200 schedule table v1 sms " << t->sms << "\n";
  char line[512];
  for (const auto& kv : t->table) {
    const TuneEntry& en = kv.second;
    int w = std::snprintf(line, sizeof(line), "%s %d %d %d", kOpName[std::get<0>(kv.first)], std::get<1>(kv.first),
                          std::get<2>(kv.first), en.choice);
    for (int c = 0; c < en.ncand && w > 0 && w < (int)sizeof(line); ++c)
      w += std::snprintf(line + w, sizeof(line) - w, " %d %.6g", en.cand[c], en.ms[c]);
    f << line << "\n";
  }
  return f.good() ? RCWA_OK : RCWA_ERR_INVALID;
}

// Entries of the file replace those with the same key; the whole file is
// checked before anything is inserted.
extern "C" int rcwa_tuner_load(rcwa_tuner* t, const char* path) {
  if (!t || !path) return RCWA_ERR_INVALID;
  std::ifstream f(path);
  if (!f) return RCWA_ERR_INVALID;
  std::vector<std::pair<std::tuple<int, int, int>, TuneEntry>> got;
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream is(line);
    std::string name;
    int n = 0, cls = 0, choice = -1;
    if (!(is >> name >> n >> cls >> choice)) return RCWA_ERR_INVALID;
    int op = -1;
    for (int k = 0; k < kTuneOps; ++k)
      if (name == kOpName[k]) op = k;
    if (op < 0 || n <= 0 || (cls != 1 && cls != 2 && cls != 3 && cls != 4 && cls != 8) || !valid_choice(op, n, choice))
      return RCWA_ERR_INVALID;
    TuneEntry en;
    en.ncand = tune_candidates(op, n, en.cand);
    en.choice = choice;
    int c = 0;
    double ms = 0.0;
    while (is >> c >> ms) {
      for (int k = 0; k < en.ncand; ++k)
        if (en.cand[k] == c) en.ms[k] = ms;
    }
    got.push_back({std::make_tuple(op, n, cls), en});
  }
  std::lock_guard<std::mutex> lk(t->mu);
  for (auto& g : got) t->table[g.first] = g.second;
  return RCWA_OK;
}

extern "C" int rcwa_engine_set_tuner(rcwa_engine* e, rcwa_tuner* t, int mode) {
  if (!e || mode < kTuningOff || mode > kTuningAuto || (mode != kTuningOff && !t)) return RCWA_ERR_INVALID;
  if (t) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device) == cudaSuccess && sms > 0) {
      std::lock_guard<std::mutex> lk(t->mu);
      t->sms = sms;
    }
  }
  e->tuner = mode == kTuningOff ? nullptr : t;
  e->tuning = mode;
  return RCWA_OK;
}

extern "C" int rcwa_tuner_measure(rcwa_engine* e, rcwa_tuner* t, int op, int n, int batch, int* choice, double* ms) {
  if (!e || !t || !valid_op(op) || n <= 0 || batch <= 0) return RCWA_ERR_INVALID;
  if (cudaSetDevice(e->device) != cudaSuccess) return RCWA_ERR_CUDA;
  TuneEntry ent;
  const cudaError_t err = tune_measure(e, op, n, batch, ent);
  if (err == cudaErrorMemoryAllocation) {
    e->last_error = "tuner: device allocation failed";
    return RCWA_ERR_NOMEM;
  }
  if (err != cudaSuccess) {
    e->last_error = std::string("tuner: ") + cudaGetErrorString(err);
    return RCWA_ERR_CUDA;
  }
  {
    std::lock_guard<std::mutex> lk(t->mu);
    t->table[std::make_tuple(op, n, tune_batch_class(batch, t->sms))] = ent;
  }
  if (choice) *choice = ent.choice;
  if (ms)
    for (int c = 0; c < kTuneMaxCand; ++c) ms[c] = c < ent.ncand ? ent.ms[c] : 0.0;
  return RCWA_OK;
}
