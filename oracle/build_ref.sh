#!/bin/sh
# Compile GARLI's own eigensolver (garli/trunk/src/linalg.cpp, standalone: it
# needs only defs.h) plus oracle/ref_eigen_shim.cpp into oracle/_ref/libref_linalg.so.
# The rest of GARLI's CPU path needs NCL (an external library, not vendored)
# and is restated in oracle/garli_oracle.c instead.
set -e
REF=${1:-/root/reference/garli/trunk/src}
HERE=$(cd "$(dirname "$0")" && pwd)
[ -f "$REF/linalg.cpp" ] || { echo "reference sources not found at $REF" >&2; exit 1; }
mkdir -p "$HERE/_ref"
g++ -O2 -fPIC -shared -DUNIX -DNDEBUG -I"$REF" -o "$HERE/_ref/libref_linalg.so" \
    "$REF/linalg.cpp" "$HERE/ref_eigen_shim.cpp"
echo "$HERE/_ref/libref_linalg.so"
