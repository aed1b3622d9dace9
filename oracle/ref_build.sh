#!/bin/sh
# Builds the reference's own code, from its sources where they lie, into
# oracle/_ref/ (git-ignored).  Checker infrastructure only.
#   oracle/ref_build.sh [--if-present] [REFERENCE_TREE]
# The tree is the argument, else $PAC_REFERENCE_TREE, else the container's
# read-only mount.  --if-present: exit quietly when no tree is there.
#
#   libpredref.so                     predicates.h compiled for the host
#   parallelac-largeData              AlphaComplexLargeData.cu, default flags
#                                     (as the reference's CMakeLists.txt builds it)
#   parallelac-largeData-nofma        ... with -fmad=false
#   parallelac-largeData-rr128        ... with -maxrregcount=128, so that
#                                     checkTetsOrthosphere fits its 512-thread
#                                     launch and actually runs
#   parallelac-largeData-rr128-nofma  ... both
#   parallelac-rr128                  AlphaComplexParallel.cu (the plain
#   parallelac-rr128-nofma            binary) with -maxrregcount=128, and
#                                     with -fmad=false too.  It includes
#                                     <gmp.h> through its vendored CGBN; the
#                                     declarations come from oracle/gmp_shim
#                                     and the link is against the system's
#                                     runtime libgmp.so.10 (no GMP headers are
#                                     installed).
set -e
IF_PRESENT=0
if [ "$1" = "--if-present" ]; then IF_PRESENT=1; shift; fi
REF=${1:-${PAC_REFERENCE_TREE:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
CXX=/usr/bin/g++
[ -x "$CXX" ] || CXX=g++
if [ ! -f "$REF/predicates.h" ]; then
    if [ $IF_PRESENT = 1 ]; then echo "no reference tree at $REF: oracle/_ref not built"; exit 0; fi
    echo "no reference tree at $REF" >&2; exit 1
fi
GMP_SO=/usr/lib/x86_64-linux-gnu/libgmp.so.10
mkdir -p "$OUT"
if [ ! -f "$OUT/libpredref.so" ] || [ "$HERE/predref_wrap.cpp" -nt "$OUT/libpredref.so" ]; then
    $CXX -O2 -ffp-contract=off -fPIC -shared -w -I"$REF" -o "$OUT/libpredref.so" "$HERE/predref_wrap.cpp"
fi
build() {  # name source flags...
    name=$1; src=$2; shift 2
    [ -x "$OUT/$name" ] && return 0
    $NVCC -gencode arch=compute_100a,code=sm_100a -ccbin "$CXX" -w "$@" \
        -o "$OUT/$name.tmp" "$REF/$src" && mv "$OUT/$name.tmp" "$OUT/$name"
}
LD=AlphaComplexLargeData.cu
PLAIN=AlphaComplexParallel.cu
build parallelac-largeData $LD &
build parallelac-largeData-nofma $LD -fmad=false &
build parallelac-largeData-rr128 $LD -maxrregcount=128 &
build parallelac-largeData-rr128-nofma $LD -maxrregcount=128 -fmad=false &
wait
names="parallelac-largeData parallelac-largeData-nofma parallelac-largeData-rr128 parallelac-largeData-rr128-nofma"
if [ -f "$GMP_SO" ]; then
    build parallelac-rr128 $PLAIN -maxrregcount=128 -I"$HERE/gmp_shim" -Xlinker "$GMP_SO" &
    build parallelac-rr128-nofma $PLAIN -maxrregcount=128 -fmad=false -I"$HERE/gmp_shim" \
        -Xlinker "$GMP_SO" &
    wait
    names="$names parallelac-rr128 parallelac-rr128-nofma"
else
    echo "no $GMP_SO: the plain binary is not built" >&2
fi
for b in $names; do
    [ -x "$OUT/$b" ] || { echo "reference build failed: $b" >&2; exit 1; }
done
echo "reference builds in $OUT"
