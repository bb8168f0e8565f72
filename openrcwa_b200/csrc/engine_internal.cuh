// Engine object shared by the C-ABI translation units.
#pragma once
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "common.cuh"

struct rcwa_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;
  // plan workspace kept between plans (grow only); lent to one plan at a time
  void* work_cache = nullptr;
  size_t work_cache_bytes = 0;
  bool work_cache_busy = false;
  // schedule table consulted when plans are built (not owned), and its mode
  // (kTuningOff: built-in rules; kTuningTable: table, else the rules;
  // kTuningAuto: table, else measure and record)
  struct rcwa_tuner* tuner = nullptr;
  int tuning = 0;
  // small device blocks of finished plans (inputs, outputs, metadata) kept
  // for the next plan, so that a stream of small solves does not pay a
  // cudaMalloc/cudaFree pair per buffer
  std::vector<std::pair<void*, size_t>> block_pool;
  size_t block_pool_bytes = 0;
  std::mutex pool_mu;
};

// A device block of at least `bytes` from the engine's pool, else a new
// allocation (nullptr when that fails); *got receives its size.
void* engine_take_block(rcwa_engine* e, size_t bytes, size_t* got);
// Returns a block to the pool (or frees it when the pool is full).  The
// caller guarantees no kernel still uses it.
void engine_release_block(rcwa_engine* e, void* p, size_t bytes);
