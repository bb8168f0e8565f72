// Engine object shared by the C-ABI translation units.
#pragma once
#include <string>

#include "common.cuh"

struct rcwa_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;
  // plan workspace kept between plans (grow only); lent to one plan at a time
  void* work_cache = nullptr;
  size_t work_cache_bytes = 0;
  bool work_cache_busy = false;
};
