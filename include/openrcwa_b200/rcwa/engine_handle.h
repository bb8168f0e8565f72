// Process-wide engine used by the header-only RCWA API adapters.  The device
// is RCWA_B200_DEVICE from the environment (default 0).  A missing or failed
// device is reported on std::cerr, and the calls then leave their outputs
// empty, as the reference does on its own error paths.
#pragma once
#include <cstdlib>
#include <iostream>
#include <mutex>

#include "../../rcwa_b200.h"

namespace rcwa_b200 {
inline rcwa_engine* engine() {
  static rcwa_engine* e = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    const char* d = std::getenv("RCWA_B200_DEVICE");
    const int rc = rcwa_engine_create(d ? std::atoi(d) : 0, &e);
    if (rc != RCWA_OK) {
      std::cerr << "[rcwa_b200] engine unavailable: " << rcwa_status_string(rc) << "\n";
      e = nullptr;
    }
  });
  return e;
}
}  // namespace rcwa_b200
