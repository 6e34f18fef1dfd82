#!/bin/bash
# Builds the reference's own CUDA library (mumax/2 src/libmumax2) for sm_100a into
# oracle/_ref/libmumax2_ref.so.  Test infrastructure only: the library is the
# reference-side checker of the libmumax2-compatible entry points.  Sources are
# compiled where they lie; nothing is copied into this repository.
# The reference targets sm_20/sm_30 (src/Make.inc:11-17); only the architecture flag
# changes, and <stdio.h> is force-included because gpu_safe.h uses printf without it.
set -e
[ -n "$REF_ROOT" ] || { echo "set REF_ROOT to the mumax/2 source tree" >&2; exit 1; }
REF=$REF_ROOT/src/libmumax2
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$HERE/_ref
[ -d "$REF" ] || { echo "reference sources not found at $REF" >&2; exit 1; }
mkdir -p "$OUT/obj"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
FLAGS="-gencode arch=compute_100a,code=sm_100a -std=c++14 -O3 --use_fast_math -Xcompiler -fPIC -include stdio.h -I$REF"
objs=""
for f in "$REF"/*.cu "$REF"/*.cpp; do
  b=$(basename "$f")
  o="$OUT/obj/$b.o"
  if [ ! -f "$o" ] || [ "$f" -nt "$o" ]; then
    $NVCC $FLAGS -c "$f" -o "$o" &
  fi
  objs="$objs $o"
done
wait
$NVCC -gencode arch=compute_100a,code=sm_100a -shared -o "$OUT/libmumax2_ref.so" $objs -lcudart -lcufft -lcurand
echo "built $OUT/libmumax2_ref.so"
