#!/bin/sh
# Compiles the reference's own propagator sources (libnestutil/iaf_propagator.cpp,
# libnestutil/numerics.cpp) with g++ directly into oracle/_ref/libnestprop.so,
# for pinning the oracle's and the engine's FP64 coefficients.  The
# reference's build system is not used; its generated config.h is replaced by
# an empty header (these two files need none of its macros).
# Usage: oracle/build_ref.sh [--if-present] [reference root]
# The reference root defaults to $NEST_REFERENCE_ROOT, else /root/reference.
# With --if-present a missing source tree is not an error (nothing is built).
set -e
IF_PRESENT=0
if [ "$1" = "--if-present" ]; then IF_PRESENT=1; shift; fi
REF=${1:-${NEST_REFERENCE_ROOT:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
if [ ! -f "$REF/libnestutil/iaf_propagator.cpp" ]; then
  [ "$IF_PRESENT" = 1 ] && exit 0
  echo "reference sources not found under $REF" >&2
  exit 1
fi
mkdir -p "$OUT/include"
: > "$OUT/include/config.h"
CXX=${CXX:-/usr/bin/g++}
$CXX -std=c++20 -O2 -fPIC -ffp-contract=off -shared -I"$OUT/include" -I"$REF/libnestutil" \
  -o "$OUT/libnestprop.so" "$REF/libnestutil/iaf_propagator.cpp" "$REF/libnestutil/numerics.cpp" "$HERE/ref_shim.cpp"
echo "built $OUT/libnestprop.so"
