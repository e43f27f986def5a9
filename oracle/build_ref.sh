#!/bin/sh
# Builds oracle/_ref/ref_harness: the reference's own solver functions, compiled from the
# reference sources where they lie, driven by oracle/ref_harness.c (test infrastructure), and
# oracle/_ref/in3mg, the reference's initial-condition program.
# Two changes, both in temporary copies removed after compilation: the static array sizes of
# head3mg.c:8-20 (the shipped sizes need 78 GB of static storage), and an optional cap on the
# outer iteration blocks of titerate (heat3mg.c:463-560 loops until heatsum <= HEATMIN, which
# its racy multi-threaded relaxation may never reach); the cap is unlimited unless the
# harness's sample command sets it.  Outputs go to oracle/_ref/ only.
set -e
REF=${I3G_REFERENCE_DIR:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
if [ ! -f "$REF/move3mg.c" ]; then
    echo "reference sources not found in $REF; oracle/_ref not rebuilt" >&2
    exit 0
fi
mkdir -p "$OUT/gen"
sed -e 's/^#define MAXMAT .*/#define MAXMAT  160000000/' \
    -e 's/^#define MAXNOD .*/#define MAXNOD   5000000/' \
    -e 's/^#define MAXNNN .*/#define MAXNNN   2300000/' \
    -e 's/^#define MAXPAR .*/#define MAXPAR  40000000/' \
    -e 's/^#define MAXPPP .*/#define MAXPPP  16000000/' \
    -e 's/^#define MAXMRK .*/#define MAXMRK  60000000/' \
    -e 's/^#define MAXBON .*/#define MAXBON   4000000/' \
    "$REF/head3mg.c" > "$OUT/gen/head3mg.c"
sed -e 's/^while(heatsum>HEATMIN);/while(heatsum>HEATMIN \&\& ++i3g_heat_blocks < i3g_heat_block_cap);/' \
    "$REF/heat3mg.c" > "$OUT/gen/heat3mg.c"
grep -q "i3g_heat_block_cap" "$OUT/gen/heat3mg.c" || { echo "heat3mg.c loop not found" >&2; exit 1; }
gcc -O2 -fopenmp -mcmodel=medium -w -I"$OUT/gen" -I"$REF" "$HERE/ref_harness.c" \
    -o "$OUT/ref_harness" -lm
rm -f "$OUT/gen/head3mg.c" "$OUT/gen/heat3mg.c"
rmdir "$OUT/gen" 2>/dev/null || true
echo "built $OUT/ref_harness"
# oracle/_ref/in3mg: the reference's initial-condition program (init.t3c -> first .prn), unchanged
# but for the same array sizes.  Its quoted includes resolve next to the including file first, so
# in3mg.c is compiled from a temporary copy beside the resized head3mg.c; the other files it
# includes come from the reference directory through -I.
mkdir -p "$OUT/gen_in3mg"
sed -e 's/^#define MAXMAT .*/#define MAXMAT  160000000/' \
    -e 's/^#define MAXNOD .*/#define MAXNOD   5000000/' \
    -e 's/^#define MAXNNN .*/#define MAXNNN   2300000/' \
    -e 's/^#define MAXPAR .*/#define MAXPAR  40000000/' \
    -e 's/^#define MAXPPP .*/#define MAXPPP  16000000/' \
    -e 's/^#define MAXMRK .*/#define MAXMRK  60000000/' \
    -e 's/^#define MAXBON .*/#define MAXBON   4000000/' \
    "$REF/head3mg.c" > "$OUT/gen_in3mg/head3mg.c"
cp "$REF/in3mg.c" "$OUT/gen_in3mg/in3mg.c"
gcc -O2 -fopenmp -mcmodel=medium -w -I"$OUT/gen_in3mg" -I"$REF" "$OUT/gen_in3mg/in3mg.c" -o "$OUT/in3mg" -lm
rm -f "$OUT/gen_in3mg/head3mg.c" "$OUT/gen_in3mg/in3mg.c"
rmdir "$OUT/gen_in3mg" 2>/dev/null || true
echo "built $OUT/in3mg"
