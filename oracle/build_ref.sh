#!/bin/sh
# Builds the reference-side test binary into oracle/_ref/ (kept out of git,
# shipped with the tree to the GPU box).  Needs the reference sources at
# $REF (default /root/reference) and the engine library already built.
# "build_ref.sh --print-ref" prints the sources' location and exits; without
# the sources the script prints a note and exits 0 (nothing to build).
#
#   rcwa_bridge_dropin : the reference's sol/rcwa_bridge.cpp, unmodified,
#                        compiled against include/openrcwa_b200/rcwa/*.h and
#                        linked with librcwa_b200.so plus dropin_harness.cpp.
#   rcwa_driver_dropin : the reference's orcwa_rcwa (rcwa/RCWADriver.cpp,
#                        rcwa/RCWAInput.cpp, src/rcwa_Main.cpp), unmodified,
#                        against the same headers and library.
# Both link hdf5_stub.cpp in place of the HDF5 writers.
#
# The reference's RCWA core (rcwa/*.cpp) itself is not built: it needs Eigen3
# and LAPACKE, which this image does not have.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=$(dirname "$HERE")
REF=${REF:-/root/reference}
if [ "$1" = "--print-ref" ]; then echo "$REF"; exit 0; fi
[ -f "$REF/sol/rcwa_bridge.cpp" ] || { echo "reference sources not found at $REF: nothing to build"; exit 0; }
OUT="$HERE/_ref"
mkdir -p "$OUT"
CXXFLAGS="-std=c++17 -O2 -DRCWA_B200_NO_EIGEN -I$ROOT/include/openrcwa_b200 -I$REF/include"
g++ $CXXFLAGS -c "$REF/sol/rcwa_bridge.cpp" -o "$OUT/rcwa_bridge.o"
g++ $CXXFLAGS -c "$HERE/dropin_harness.cpp" -o "$OUT/dropin_harness.o"
g++ $CXXFLAGS -c "$HERE/hdf5_stub.cpp" -o "$OUT/hdf5_stub.o"
g++ "$OUT/rcwa_bridge.o" "$OUT/dropin_harness.o" "$OUT/hdf5_stub.o" -L"$ROOT/openrcwa_b200/lib" -lrcwa_b200 \
    -Wl,-rpath,'$ORIGIN/../../openrcwa_b200/lib' -o "$OUT/rcwa_bridge_dropin"
DRV="-std=c++17 -O2 -DRCWA_B200_NO_EIGEN -I$ROOT/include/openrcwa_b200 -I$REF -I$REF/include"
g++ $DRV -c "$REF/rcwa/RCWADriver.cpp" -o "$OUT/RCWADriver.o"
g++ $DRV -c "$REF/rcwa/RCWAInput.cpp" -o "$OUT/RCWAInput.o"
g++ $DRV -c "$REF/src/rcwa_Main.cpp" -o "$OUT/rcwa_Main.o"
g++ "$OUT/RCWADriver.o" "$OUT/RCWAInput.o" "$OUT/rcwa_Main.o" "$OUT/hdf5_stub.o" -L"$ROOT/openrcwa_b200/lib" \
    -lrcwa_b200 -Wl,-rpath,'$ORIGIN/../../openrcwa_b200/lib' -o "$OUT/rcwa_driver_dropin"
rm -f "$OUT/rcwa_bridge.o" "$OUT/dropin_harness.o" "$OUT/hdf5_stub.o" "$OUT/RCWADriver.o" "$OUT/RCWAInput.o" \
    "$OUT/rcwa_Main.o"
echo "$OUT/rcwa_bridge_dropin"
echo "$OUT/rcwa_driver_dropin"
