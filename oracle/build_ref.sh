#!/usr/bin/env bash
# Builds the reference FASES 3D solver (vitorotri/fases v0.9) from its own sources, unmodified,
# for sm_100a, into oracle/_ref/fases3D, and its 2D legacy solver into oracle/_ref/phases2D. It is the checker the CPU restatement is pinned
# against (tests/golden/make_golden.py runs it on a B200); it is never part of the product.
# The source tree is read in place; nothing is copied into this repository.
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]
#   REFERENCE_ROOT defaults to $FZ_REFERENCE_ROOT, else to a checkout named "reference" beside this
#   repository's directory.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${FZ_REFERENCE_ROOT:-$(cd "$HERE/../.." && pwd)/reference}}"
OUT="$HERE/_ref"
mkdir -p "$OUT"
if [ ! -f "$REF/3D-solver/core/main3D.cu" ]; then
  echo "reference sources not found under $REF" >&2
  exit 2
fi
# Same flags as 3D-solver/Makefile:1-32 with ARCH set to sm_100a.
nvcc -std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fopenmp \
  -I"$REF/3D-solver/include" -I"$REF/common" \
  "$REF/3D-solver/core/main3D.cu" -o "$OUT/fases3D" 2> "$OUT/build.log" || {
    cat "$OUT/build.log" >&2; exit 1; }
echo "built $OUT/fases3D"
# The 2D solver as 2D-solver/Makefile:1-31 builds it, with ARCH sm_100a and the one missing
# definition (flat) supplied by a pre-include (oracle/ref2d_flat.h); the sources stay untouched.
nvcc -std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a -include "$HERE/ref2d_flat.h" \
  -I"$REF/2D-solver/include" -I"$REF/common" \
  "$REF/2D-solver/core/main.cu" -o "$OUT/phases2D" 2> "$OUT/build2d.log" || {
    cat "$OUT/build2d.log" >&2; exit 1; }
echo "built $OUT/phases2D"
