// Engine object shared by the C-ABI translation units.
#pragma once
#include <string>

#include "common.cuh"

struct rcwa_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;
};
