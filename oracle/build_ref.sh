#!/bin/sh
# Compiles the reference's own pixel-inserter source (libEM/reconstructor_tools.cpp,
# which pulls in libEM/reconstructor_tools.h and libEM/emdata_core.h) from where it
# lies in the reference tree, against the stand-in headers in oracle/refshim/, into
# oracle/_ref/libfr_ref.so (strict IEEE, for the bitwise pin) and
# oracle/_ref/libfr_ref_fast.so (release flags, for timing).  Test infrastructure only.  -I- stops the compiler from
# resolving "emdata.h" next to the reference source, so the stand-in is used.
# Strict IEEE flags (no contraction) so results compare bitwise with fr_oracle.c.
# The reference tree's location is the first argument or $EMAN2_REFERENCE;
# without either (or without the tree) nothing is built.
set -e
REF=${1:-$EMAN2_REFERENCE}
HERE=$(cd "$(dirname "$0")" && pwd)
if [ -z "$REF" ] || [ ! -f "$REF/libEM/reconstructor_tools.cpp" ]; then
  echo "reference tree not given or not found ('$REF'); oracle/_ref not built" >&2
  exit 0
fi
mkdir -p "$HERE/_ref"
g++ -std=c++17 -O2 -Wl,--no-undefined -fPIC -shared -ffp-contract=off -fno-fast-math -w \
  -I- -I"$HERE/refshim" -I"$REF/libEM" \
  "$REF/libEM/reconstructor_tools.cpp" "$HERE/ref_driver.cpp" \
  -o "$HERE/_ref/libfr_ref.so"
echo "built $HERE/_ref/libfr_ref.so"
# The same source with the reference's default release flags (its
# CMakeLists.txt: -O3 -ffast-math): the timed CPU reference arm of bench.py.
g++ -std=c++17 -O3 -ffast-math -Wl,--no-undefined -fPIC -shared -w \
  -I- -I"$HERE/refshim" -I"$REF/libEM" \
  "$REF/libEM/reconstructor_tools.cpp" "$HERE/ref_driver.cpp" \
  -o "$HERE/_ref/libfr_ref_fast.so"
echo "built $HERE/_ref/libfr_ref_fast.so"
