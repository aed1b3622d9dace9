#!/bin/sh
# Builds the reference's own code, from its sources where they lie, into
# oracle/_ref/ (git-ignored).  Checker infrastructure only.
#   oracle/ref_build.sh [REFERENCE_TREE]
#
#   libpredref.so                     predicates.h compiled for the host
#   parallelac-largeData              AlphaComplexLargeData.cu, default flags
#                                     (as the reference's CMakeLists.txt builds it)
#   parallelac-largeData-nofma        ... with -fmad=false
#   parallelac-largeData-rr128        ... with -maxrregcount=128, so that
#                                     checkTetsOrthosphere fits its 512-thread
#                                     launch and actually runs
#   parallelac-largeData-rr128-nofma  ... both
# The plain binary (AlphaComplexParallel.cu) needs GMP headers that are not
# installed, so it is not built.
set -e
REF=${1:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
CXX=/usr/bin/g++
[ -x "$CXX" ] || CXX=g++
[ -f "$REF/predicates.h" ] || { echo "no reference tree at $REF" >&2; exit 1; }
mkdir -p "$OUT"
if [ ! -f "$OUT/libpredref.so" ] || [ "$HERE/predref_wrap.cpp" -nt "$OUT/libpredref.so" ]; then
    $CXX -O2 -ffp-contract=off -fPIC -shared -w -I"$REF" -o "$OUT/libpredref.so" "$HERE/predref_wrap.cpp"
fi
build() {  # name flags...
    name=$1; shift
    [ -x "$OUT/$name" ] && return 0
    $NVCC -gencode arch=compute_100a,code=sm_100a -ccbin "$CXX" -w "$@" \
        -o "$OUT/$name.tmp" "$REF/AlphaComplexLargeData.cu" && mv "$OUT/$name.tmp" "$OUT/$name"
}
build parallelac-largeData &
build parallelac-largeData-nofma -fmad=false &
build parallelac-largeData-rr128 -maxrregcount=128 &
build parallelac-largeData-rr128-nofma -maxrregcount=128 -fmad=false &
wait
for b in parallelac-largeData parallelac-largeData-nofma parallelac-largeData-rr128 parallelac-largeData-rr128-nofma; do
    [ -x "$OUT/$b" ] || { echo "reference build failed: $b" >&2; exit 1; }
done
echo "reference builds in $OUT"
