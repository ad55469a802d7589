#!/usr/bin/env bash
# Builds the checker library oracle/_ref/libzsph_ref.so from the reference's
# own hot-path sources, in place and unmodified, for sm_100a.  The reference's
# CMake build needs VTK, the un-vendored nlohmann/json submodule and the
# removed FindCUDA module, so this recipe compiles the six hot-path files
# directly with the reference's own flags (-lineinfo -maxrregcount 64, -rdc),
# sm_100a in place of sm_75, and ref_shim.cuh in place of std_header.cuh.
# Output goes only to oracle/_ref/ (git-ignored).  Test infrastructure only.
set -euo pipefail
HERE=$(cd "$(dirname "$0")" && pwd)
# the reference checkout: ZSPH_REFERENCE, else a "reference" directory beside this repository
REF=${ZSPH_REFERENCE:-$(cd "$HERE/../.." && pwd)/reference}
SG="$REF/single_gpu_sph_src"
OUT="$HERE/_ref"
if [ ! -d "$SG" ]; then
  echo "reference sources not found at $SG; oracle/_ref not built" >&2
  exit 0
fi
NVCC=${NVCC:-nvcc}
ARCH="-gencode arch=compute_100a,code=sm_100a"
# deltasph (-DZSPH_DELTA, delta_ns.cu) and simplesph (-DZSPH_SIMPLE, simple_ns.cu),
# as the reference's two CMake targets select them
build() {
  local macro=$1 eqfile=$2 lib=$3 obj="$OUT/obj_$3"
  mkdir -p "$obj"
  local FLAGS="-std=c++17 -rdc=true $ARCH -lineinfo -maxrregcount 64 -Xcompiler -fPIC -D__STD_HEADER_CUH__ -D$macro -include $HERE/ref_shim.cuh -I $SG/header"
  for f in lib/hash.cu lib/sort.cu "$eqfile" lib/time_int.cu lib/init.cu lib/check.cu; do
    "$NVCC" $FLAGS -c "$SG/$f" -o "$obj/$(basename "$f" .cu).o"
  done
  "$NVCC" $FLAGS -c "$HERE/ref_driver.cu" -o "$obj/ref_driver.o"
  "$NVCC" -shared -rdc=true $ARCH -Xcompiler -fPIC "$obj"/*.o -o "$OUT/$lib.so"
  echo "built $OUT/$lib.so"
}
build ZSPH_DELTA equation/delta_ns.cu libzsph_ref
build ZSPH_SIMPLE equation/simple_ns.cu libzsph_ref_simple
