#!/bin/sh
# Compile the reference's own solver sources (buuugyellow/MultiGridSoftBody,
# MultiGridSoftBody/src) headless, together with oracle/ref_driver.cu, into
# oracle/_ref/libmgsb_ref.so.  Test infrastructure only.
#
# The sources are GBK-encoded; they are transcoded into a temporary directory
# (deleted afterwards) next to oracle/ref_shim/global.h, which replaces the
# reference's GUI/glog global.h.  Nothing from the reference is kept in the
# repository; only the built library lands in oracle/_ref/ (git-ignored).
set -eu
HERE=$(cd "$(dirname "$0")" && pwd)
# the reference checkout: MGSB_REFERENCE_DIR, else a directory "reference" beside the repository
REF=${MGSB_REFERENCE_DIR:-$(cd "$HERE/../.." && pwd)/reference}/MultiGridSoftBody/src
OUT="$HERE/_ref"
if [ ! -d "$REF" ]; then
    echo "ref_build: reference sources not found at $REF; skipping" >&2
    exit 0
fi
NVCC=$(command -v nvcc || echo /usr/local/cuda/bin/nvcc)
TMP=$(mktemp -d)
trap 'rm -rf "$TMP"' EXIT
for f in utils.cu PDSolver.cu PDSolverAc.cu PDSolver.cpp PDSolver_MG.cpp Collider.cpp SoftObject.cpp \
         simpleMath.h Simulator.h PDSolver.h PDSolver_MG.h Collider.h SoftObject.h; do
    iconv -f GBK -t UTF-8 -c "$REF/$f" | sed '1s/^\xEF\xBB\xBF//' > "$TMP/$f"
done
cp "$HERE/ref_shim/global.h" "$HERE/ref_driver.cu" "$TMP/"
FLAGS="-std=c++17 -rdc=true -x cu -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -O2 -w"
OBJS=""
for f in utils.cu PDSolver.cu PDSolverAc.cu PDSolver.cpp PDSolver_MG.cpp Collider.cpp SoftObject.cpp ref_driver.cu; do
    "$NVCC" $FLAGS -I"$TMP" -c "$TMP/$f" -o "$TMP/$f.o"
    OBJS="$OBJS $TMP/$f.o"
done
mkdir -p "$OUT"
"$NVCC" -shared -rdc=true -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -o "$OUT/libmgsb_ref.so.tmp" $OBJS
mv "$OUT/libmgsb_ref.so.tmp" "$OUT/libmgsb_ref.so"
echo "$OUT/libmgsb_ref.so"
