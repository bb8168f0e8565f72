// HDF5 writers of the reference's callers (include/rcwa_hdf5.h), stubbed for
// the drop-in test binaries: HDF5 output is outside the engine and libhdf5 is
// not installed, so the writers report failure and the callers keep their CSV
// output.  TEST INFRASTRUCTURE ONLY (linked into oracle/_ref by
// oracle/build_ref.sh).
#include "rcwa_hdf5.h"

extern "C" {
int rcwa_write_hdf5(const char*, const rcwa_meta_t*, const rcwa_spectrum_row_t*, int, int, const char* const*) {
  return 1;
}
int rcwa_write_hdf5_orders(const char*, int, int, int, int, const double*, const double*) { return 1; }
}
