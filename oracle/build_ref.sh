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
REF=${ZSPH_REFERENCE:-/root/reference}
SG="$REF/single_gpu_sph_src"
OUT="$HERE/_ref"
if [ ! -d "$SG" ]; then
  echo "reference sources not found at $SG; oracle/_ref not built" >&2
  exit 0
fi
mkdir -p "$OUT/obj"
NVCC=${NVCC:-nvcc}
ARCH="-gencode arch=compute_100a,code=sm_100a"
FLAGS="-std=c++17 -rdc=true $ARCH -lineinfo -maxrregcount 64 -Xcompiler -fPIC -D__STD_HEADER_CUH__ -DZSPH_DELTA -include $HERE/ref_shim.cuh -I $SG/header"
for f in lib/hash.cu lib/sort.cu equation/delta_ns.cu lib/time_int.cu lib/init.cu lib/check.cu; do
  "$NVCC" $FLAGS -c "$SG/$f" -o "$OUT/obj/$(basename "$f" .cu).o"
done
"$NVCC" $FLAGS -c "$HERE/ref_driver.cu" -o "$OUT/obj/ref_driver.o"
"$NVCC" -shared -rdc=true $ARCH -Xcompiler -fPIC "$OUT"/obj/*.o -o "$OUT/libzsph_ref.so"
echo "built $OUT/libzsph_ref.so"
