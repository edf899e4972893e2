#!/bin/sh
# Compiles the reference's own host code for the golden-vector harness from
# the SOP-GPU source tree where it lies (read only), into oracle/_ref/.
# Nothing from the reference tree is copied into this repository.
# Usage: oracle/build_ref.sh [path-to-SOP-GPU]   (default /root/reference)
set -e
REF=${1:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
if [ ! -d "$REF/src" ]; then
    echo "reference tree not found at $REF; skipping" >&2
    exit 0
fi
mkdir -p "$OUT"
/usr/bin/g++ -O2 -w -std=c++11 -I"$REF/src" -I/usr/local/cuda/include \
    -o "$OUT/ref_host" "$HERE/ref_host_harness.cpp" \
    "$REF/src/Integrators/ran2.cpp" "$REF/src/IO/configreader.cpp" \
    "$REF/src/IO/topio.cpp" "$REF/src/IO/pdbio.cpp" \
    "$REF/src/Util/wrapper.cpp" "$REF/src/Util/mystl.cpp"
echo "built $OUT/ref_host"
