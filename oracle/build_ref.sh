#!/bin/sh
# Compile GARLI's own eigensolver (garli/trunk/src/linalg.cpp, standalone: it
# needs only defs.h) plus oracle/ref_eigen_shim.cpp into oracle/_ref/libref_linalg.so.
# The rest of GARLI's CPU path needs NCL (an external library, not vendored)
# and is restated in oracle/garli_oracle.c instead.
#
#   sh oracle/build_ref.sh [garli/trunk/src directory]
# The directory defaults to $GARLI_REFERENCE/garli/trunk/src, GARLI_REFERENCE
# defaulting to the checkout this build was set up with (/root/reference).
# Without the sources it prints a note and exits 0: the oracle's own
# restatement does not need them.
set -e
REF=${1:-${GARLI_REFERENCE:-/root/reference}/garli/trunk/src}
HERE=$(cd "$(dirname "$0")" && pwd)
[ -f "$REF/linalg.cpp" ] || { echo "reference sources not found at $REF: oracle/_ref not built" >&2; exit 0; }
mkdir -p "$HERE/_ref"
g++ -O2 -fPIC -shared -DUNIX -DNDEBUG -I"$REF" -o "$HERE/_ref/libref_linalg.so" \
    "$REF/linalg.cpp" "$HERE/ref_eigen_shim.cpp"
echo "$HERE/_ref/libref_linalg.so"
