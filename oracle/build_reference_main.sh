#!/bin/sh
# Builds the reference's own main program, mg_NS_solver.c, in two forms, for
# the tests that run it as a whole program (TEST INFRASTRUCTURE ONLY):
#   <out>/{timple,fs}_ref  the reference's C code alone (its own headers; CPU)
#   <out>/{timple,fs}_mgm  the same main with only the include swap that
#                          INTEGRATION.md describes, linked against libmgm.so
# "timple" is the main as shipped (time_implicit_solver); "fs" the variant its
# own comments select (fractional_step_solver.h and fractional_step_explicit,
# mg_NS_solver.c:9-10 and 71-72).  The sources are edited in a temporary
# directory; only the binaries are written into <out>.
#
#   sh oracle/build_reference_main.sh <reference tree> <out dir> <dir of libmgm.so, or "">
set -e
REF="$1"
OUT="$2"
LIBDIR="$3"
[ -f "$REF/mg_NS_solver.c" ] || { echo "no mg_NS_solver.c under '$REF': reference main not built"; exit 0; }
mkdir -p "$OUT"
T=$(mktemp -d)
trap 'rm -rf "$T"' EXIT
cp "$REF/mg_NS_solver.c" "$T/timple.c"
# the fractional-step variant: the two commented alternatives of the main swapped in
sed -e 's|^// #include "header_files/fractional_step_solver.h"|#include "header_files/fractional_step_solver.h"|' \
    -e 's|^#include "header_files/timple_solver.h"|// #include "header_files/timple_solver.h"|' \
    -e 's|^\( *\)// steady_state_error = fractional_step_explicit(|\1steady_state_error = fractional_step_explicit(|' \
    -e 's|^\( *\)steady_state_error = time_implicit_solver(|\1// steady_state_error = time_implicit_solver(|' \
    "$REF/mg_NS_solver.c" > "$T/fs.c"
grep -q '^#include "header_files/fractional_step_solver.h"' "$T/fs.c"
grep -q '^ *steady_state_error = fractional_step_explicit(' "$T/fs.c"
for v in timple fs; do
    gcc -O2 -w -I"$REF" -o "$OUT/${v}_ref" "$T/$v.c" -lm
    echo "built $OUT/${v}_ref"
done
if [ -n "$LIBDIR" ] && [ -f "$LIBDIR/libmgm.so" ]; then
    REPO=$(cd "$(dirname "$0")/.." && pwd)
    for v in timple fs; do
        # the include swap: the solver header becomes mgm_reference.h, the
        # OpenACC data functions come from the same header
        sed -e 's|^#include "header_files/timple_solver.h"|#include "mgm_reference.h"|' \
            -e 's|^#include "header_files/fractional_step_solver.h"|#include "mgm_reference.h"|' \
            -e 's|^#include "header_files/openACC_functions.h"|/* openACC_functions.h: in mgm_reference.h */|' \
            "$T/$v.c" > "$T/${v}_mgm.c"
        grep -q '^#include "mgm_reference.h"' "$T/${v}_mgm.c"
        gcc -O2 -w -I"$REPO/include" -I"$REF" -o "$OUT/${v}_mgm" "$T/${v}_mgm.c" \
            -L"$LIBDIR" -lmgm -Wl,-rpath,'$ORIGIN/../../../multigrid_meshless_b200' -lm
        echo "built $OUT/${v}_mgm"
    done
else
    echo "libmgm.so not found in '$LIBDIR': include-swapped mains not built"
fi
