#!/usr/bin/env bash
# Test infrastructure only (oracle). Compiles the reference's own CPU sources
# for the ISDF path, unmodified, where they lie under the reference checkout,
# together with the single-rank MPI / FFTW shims and BLAS forwarders in
# oracle/shims, into oracle/_ref/libisdf_ref.so, and once more with the
# p-rank MPI stand-in of oracle/shims_mp into oracle/_ref/libisdf_ref_mp.so.
# The reference's flags are kept (-O2 -std=c++14, no -march, so no FMA
# contraction: Makefile:102,159).
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]
# REFERENCE_ROOT: the argument, else $ISDF_REFERENCE_ROOT, else the read-only
# checkout this recipe was written against (/root/reference). Nothing else in
# the repository names that location.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${ISDF_REFERENCE_ROOT:-/root/reference}}"
OUT="$HERE/_ref"
if [ ! -d "$REF/src" ]; then
  echo "reference sources not found under $REF; skipping oracle/_ref build" >&2
  exit 0
fi
OPENBLAS_DIR="$(python3 -c 'import scipy, os; print(os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs"))')"
OPENBLAS="$(ls "$OPENBLAS_DIR"/libscipy_openblas*.so | head -1)"
mkdir -p "$OUT/obj"
CXXFLAGS="-O2 -std=c++14 -fPIC -w -I$HERE/shims -I$REF/include -I$REF/include/common"
SRCS="src/common/utility.cpp src/common/global.cpp src/common/fourier.cpp src/common/checkcode.cpp
      src/cpu/getpoints_Kmeans_MPI.cpp src/cpu/getbasis_MPI.cpp src/cpu/blas.cpp src/cpu/lapack.cpp"
OBJS=""
for s in $SRCS; do
  o="$OUT/obj/$(echo "$s" | tr '/' '_' ).o"
  g++ $CXXFLAGS -c "$REF/$s" -o "$o"
  OBJS="$OBJS $o"
done
g++ $CXXFLAGS -c "$HERE/ref_driver.cpp" -o "$OUT/obj/ref_driver.o"
g++ -O2 -std=c++14 -fPIC -c "$HERE/shims/minifft.cpp" -o "$OUT/obj/minifft.o"
gcc -O2 -fPIC -c "$HERE/shims/blas_alias.c" -o "$OUT/obj/blas_alias.o"
g++ -shared -o "$OUT/libisdf_ref.so" $OBJS "$OUT/obj/ref_driver.o" "$OUT/obj/minifft.o" \
    "$OUT/obj/blas_alias.o" "$OPENBLAS" -Wl,-rpath,"$OPENBLAS_DIR"
echo "built $OUT/libisdf_ref.so"

# The same sources against the p-rank MPI stand-in of oracle/shims_mp (ranks
# as forked processes over shared memory): the p-rank reference KMEAN.
mkdir -p "$OUT/obj_mp"
MPFLAGS="-O2 -std=c++14 -fPIC -w -I$HERE/shims_mp -I$HERE/shims -I$REF/include -I$REF/include/common"
OBJS_MP=""
for s in $SRCS; do
  o="$OUT/obj_mp/$(echo "$s" | tr '/' '_' ).o"
  g++ $MPFLAGS -c "$REF/$s" -o "$o"
  OBJS_MP="$OBJS_MP $o"
done
g++ $MPFLAGS -c "$HERE/ref_mp_driver.cpp" -o "$OUT/obj_mp/ref_mp_driver.o"
g++ -O2 -std=c++14 -fPIC -I"$HERE/shims_mp" -c "$HERE/shims_mp/mpi_mp.cpp" -o "$OUT/obj_mp/mpi_mp.o"
g++ -shared -Wl,-Bsymbolic -o "$OUT/libisdf_ref_mp.so" $OBJS_MP "$OUT/obj_mp/ref_mp_driver.o" \
    "$OUT/obj_mp/mpi_mp.o" "$OUT/obj/minifft.o" "$OUT/obj/blas_alias.o" "$OPENBLAS" -lpthread \
    -Wl,-rpath,"$OPENBLAS_DIR"
echo "built $OUT/libisdf_ref_mp.so"
