#!/bin/sh
# Relink the reference's own example driver against the drop-in library.
#
#   oracle/build_relink.sh [REFERENCE_DIR]      (default: $HAZ_REF)
#
# Needs oracle/_ref/obj (oracle/build_ref.sh) and hazmath_b200/libhazb200.so.
# Compiles examples/solvers/solvers.c of the reference (read in place, never
# copied) once and links it three ways, all into oracle/_ref/ (git-ignored):
#
#   solvers_ref           the reference library alone (libhazmath.so)
#   solvers_b200          -lhazb200 before -lhazmath (shared): the dynamic
#                         linker binds every symbol libhazb200.so exports --
#                         linear_solver_dcsr_krylov_amg and the rest of the
#                         drop-in -- to it, the rest (input parsing, COO
#                         reading, vectors) to the reference
#   solvers_b200_static   the same with the static archive: a copy of
#                         libhazmath.a whose definitions of the exported
#                         names are made local (objcopy --localize-symbol), so
#                         that the archive members pulled in for other
#                         functions do not bring the reference's versions
#
# The run paths are relative ($ORIGIN), so the binaries work wherever the
# repository is copied.
set -e
REF=${1:-$HAZ_REF}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
HZB="$HERE/../hazmath_b200"
if [ ! -f "$REF/examples/solvers/solvers.c" ]; then
    echo "build_relink.sh: reference sources not found at $REF" >&2
    exit 2
fi
if [ ! -f "$HZB/libhazb200.so" ] || [ ! -f "$OUT/libhazmath.a" ]; then
    echo "build_relink.sh: build hazmath_b200/libhazb200.so and oracle/_ref first" >&2
    exit 2
fi
CFLAGS="-O2 -w -I$OUT/include -I$REF/include"
gcc -shared -o "$OUT/libhazmath.so" "$OUT"/obj/*.o -lm
gcc $CFLAGS -c "$REF/examples/solvers/solvers.c" -o "$OUT/solvers.o"
gcc -o "$OUT/solvers_ref" "$OUT/solvers.o" -L"$OUT" -lhazmath -lm \
    -Wl,-rpath,'$ORIGIN'
gcc -o "$OUT/solvers_b200" "$OUT/solvers.o" -Wl,--no-as-needed -L"$HZB" -lhazb200 \
    -L"$OUT" -lhazmath -lm -Wl,-rpath,'$ORIGIN/../../hazmath_b200' -Wl,-rpath,'$ORIGIN'
# static route: localize the drop-in's names in a copy of the archive
nm -D --defined-only "$HZB/libhazb200.so" | awk '$2 == "T" {print $3}' | sort -u \
    > "$OUT/hzb_exports.txt"
cp "$OUT/libhazmath.a" "$OUT/libhazmath_rest.a"
objcopy --localize-symbols="$OUT/hzb_exports.txt" "$OUT/libhazmath_rest.a"
gcc -o "$OUT/solvers_b200_static" "$OUT/solvers.o" -Wl,--no-as-needed -L"$HZB" -lhazb200 \
    "$OUT/libhazmath_rest.a" -lm -Wl,-rpath,'$ORIGIN/../../hazmath_b200'
echo "built $OUT/solvers_ref $OUT/solvers_b200 $OUT/solvers_b200_static"
