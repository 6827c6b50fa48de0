#!/bin/bash
# Builds the reference's own J/K libraries (libgint.so, libgvhf.so of
# cuobc/lib) for sm_100a directly from their source files where they lie in
# the read-only reference tree, into oracle/_ref/ (git-ignored).  They serve
# as a second checker: a GPU test drives the reference's GINTbuild_jk through
# the same C ABI as this package's and compares J/K.  Test infrastructure
# only.  Usage: bash oracle/build_ref.sh [reference root]; the root defaults
# to $BYTEQC_REFERENCE_ROOT, else to where this build image mounts it.
set -e
REF=${1:-${BYTEQC_REFERENCE_ROOT:-/root/reference}}
SRC=$REF/cuobc/lib
OUT=$(cd "$(dirname "$0")" && pwd)/_ref
[ -d "$SRC/gint" ] || { echo "reference sources not found under $SRC"; exit 0; }
mkdir -p "$OUT"
ARCH="-gencode arch=compute_100a,code=sm_100a"
FLAGS="-O2 -std=c++17 -Xcompiler -fPIC -I $SRC -I $SRC/gint -ccbin g++"
if [ ! -f "$OUT/libgint.so" ]; then
  gcc -O2 -fPIC -I "$SRC/gint" -c "$SRC/gint/g2e.c" -o "$OUT/g2e.o"
  gcc -O2 -fPIC -I "$SRC/gint" -c "$SRC/gint/pair_data.c" -o "$OUT/pair_data.o"
  nvcc $ARCH $FLAGS -c "$SRC/gint/nr_fill_ao_ints.cu" -o "$OUT/nr_fill_ao_ints.o"
  nvcc $ARCH -shared -o "$OUT/libgint.so" "$OUT/g2e.o" "$OUT/pair_data.o" "$OUT/nr_fill_ao_ints.o"
fi
if [ ! -f "$OUT/libgvhf.so" ]; then
  nvcc $ARCH $FLAGS -c "$SRC/gvhf/nr_jk_driver.cu" -o "$OUT/nr_jk_driver.o"
  nvcc $ARCH -shared -o "$OUT/libgvhf.so" "$OUT/nr_jk_driver.o" -L "$OUT" -lgint -Xlinker -rpath='$ORIGIN'
fi
echo "built $OUT/libgint.so $OUT/libgvhf.so"
