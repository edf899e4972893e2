#!/bin/sh
# Compiles the reference's own host code for the golden-vector harness from
# the SOP-GPU source tree where it lies (read only), into oracle/_ref/.
# Nothing from the reference tree is copied into this repository.
# Usage: oracle/build_ref.sh [path-to-SOP-GPU]
# (default: $SOPB_REFERENCE_DIR, else the build container's /root/reference)
set -e
REF=${1:-${SOPB_REFERENCE_DIR:-/root/reference}}
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

# The reference's topology creator (src/sop-top.cpp, host code only), for
# the golden files of the topology tool.
/usr/bin/g++ -O2 -w -std=c++11 -I"$REF/src" -I/usr/local/cuda/include \
    -o "$OUT/ref_sop_top" "$REF/src/sop-top.cpp" "$REF/src/IO/configreader.cpp" \
    "$REF/src/IO/topio.cpp" "$REF/src/IO/pdbio.cpp" \
    "$REF/src/Util/wrapper.cpp" "$REF/src/Util/mystl.cpp"
echo "built $OUT/ref_sop_top"
/usr/bin/g++ -O2 -w -std=c++11 -I"$REF/src" -I/usr/local/cuda/include \
    -o "$OUT/ref_sop_top2" "$REF/src/sop-top2.cpp" "$REF"/src/TopologyCreator/*.cpp \
    "$REF/src/IO/configreader.cpp" "$REF/src/Util/wrapper.cpp" "$REF/src/Util/mystl.cpp" \
    "$REF/src/Util/parameters.cpp"
echo "built $OUT/ref_sop_top2"

# The reference's CUDA path for sm_100a (golden harness ref_gpu).  As
# shipped it targets sm_30 with texture references, both gone from CUDA 12:
# -DNOTEXTURE selects its plain-load path and ref_texture_shim.h covers the
# TEA integrator's three texture references.  Flags otherwise follow the
# reference Makefile (-O3, -use_fast_math).
NVCC=/usr/local/cuda/bin/nvcc
if [ -x "$NVCC" ]; then
    OBJ="$OUT/obj"
    mkdir -p "$OBJ"
    "$NVCC" -O3 -gencode arch=compute_100a,code=sm_100a -use_fast_math -w -DNOTEXTURE \
        -ccbin /usr/bin/g++ -include "$HERE/ref_texture_shim.h" -I"$REF/src" \
        -c "$REF/src/gsop.cu" -o "$OBJ/gsop.o"
    for f in Integrators/ran2.cpp IO/dcdio.cpp IO/pdbio.cpp IO/topio.cpp IO/configreader.cpp \
             Util/wrapper.cpp Util/mystl.cpp Util/parameters.cpp Updaters/dcd_manager.cpp; do
        /usr/bin/g++ -O3 -w -DNOTEXTURE -I"$REF/src" -I/usr/local/cuda/include -c "$REF/src/$f" \
            -o "$OBJ/$(basename "$f" .cpp).o"
    done
    /usr/bin/g++ -O2 -w -DNOTEXTURE -I"$REF/src" -I/usr/local/cuda/include -c "$HERE/ref_gpu_harness.cpp" \
        -o "$OBJ/ref_gpu_harness.o"
    /usr/bin/g++ -o "$OUT/ref_gpu" "$OBJ"/*.o -L/usr/local/cuda/lib64 -lcudart -lrt -lm -ldl -lpthread
    echo "built $OUT/ref_gpu"
fi
