#!/bin/sh
# Build recipe for the checker's reference library, oracle/_ref/libterrace_ref.so.
#
# It compiles the reference Terrace sources where they lie (read-only, nothing
# is copied) together with oracle/ref_driver.cc.  The reference Makefile is not
# used: it needs clang/OpenCilk (absent) and links -lomp; the reference's own
# OpenMP backend (include/parallel.h:26-40) is selected instead with g++ and
# libgomp, and three command-line shims:
#   -DOPENMP=1 -DCILK=0   the reference's OpenMP build (Makefile:51-55)
#   -Dcilk_for=for        src/PMA.cc:2583,2788 use a bare cilk_for
#   -include memfix.h     overlapping memcpy in the reference -> memmove
# -march=x86-64-v3 (AVX2) instead of the Makefile's -march=native: the library
# travels to other hosts; src/PMA.cc uses AVX2 intrinsics.
#
# Usage: oracle/build_ref.sh <reference_root>   (or TERRACE_REF=<reference_root>)
set -e
REF=${1:-${TERRACE_REF:-}}
if [ -z "$REF" ]; then
  echo "build_ref.sh: give the reference tree as the first argument or in TERRACE_REF" >&2
  exit 2
fi
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
if [ ! -f "$REF/include/graph.h" ]; then
  echo "build_ref.sh: reference tree not found at $REF" >&2
  exit 1
fi
mkdir -p "$OUT"
FLAGS="-std=c++17 -Ofast -DNDEBUG -march=x86-64-v3 -fopenmp -DOPENMP=1 -DCILK=0 \
 -Dcilk_for=for -include $HERE/memfix.h -fPIC -w -I$REF/include"
g++ $FLAGS -c "$REF/src/PMA.cc" -o "$OUT/PMA.o"
g++ $FLAGS -c "$REF/src/PMA_Lock.cc" -o "$OUT/PMA_Lock.o"
g++ $FLAGS -c "$REF/src/util.cc" -o "$OUT/util.o"
g++ $FLAGS -x c++ -c "$REF/src/partitioned_counter.c" -o "$OUT/partitioned_counter.o"
g++ $FLAGS -c "$HERE/ref_driver.cc" -o "$OUT/ref_driver.o"
# Linked without -Ofast so no fast-math start-up code enters the host process.
g++ -shared -fopenmp -o "$OUT/libterrace_ref.so" "$OUT/PMA.o" "$OUT/PMA_Lock.o" \
  "$OUT/util.o" "$OUT/partitioned_counter.o" "$OUT/ref_driver.o"
rm -f "$OUT"/*.o
echo "built $OUT/libterrace_ref.so"
