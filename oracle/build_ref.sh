#!/usr/bin/env bash
# Builds the reference's own noblockage programs (10 MHz and 1 MHz) from their sources, unmodified,
# into oracle/_ref/ (a git-ignored build output).
# Used only to generate golden fixtures (tests/golden/make_reference_fixtures.py).
# Only these variants are built: their kernels stay in bounds on valid inputs, while
# the blockage variants' calculateDcf reads R[nr], mb[nr] one past the end
# (vissgen3d_blockage.cu:138) and pix2ang.cu reads jrll[12] / pix2x[1024].
# The reference sources are read from $REF, by default a "reference" folder
# beside the repository.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF=${REF:-$(cd "$HERE/../.." && pwd)/reference}
OUT="$HERE/_ref"
[ -d "$REF" ] || { echo "reference sources not found at $REF" >&2; exit 0; }
mkdir -p "$OUT"
for prog in vissgen3d_noblockage_10m vissgen3d_noblockage; do
  src="$REF/$prog.cu"
  exe="$OUT/$prog"
  if [ ! -x "$exe" ] || [ "$src" -nt "$exe" ]; then
    nvcc -O2 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fopenmp -I "$REF" "$src" -o "$exe" -lgomp
  fi
  echo "$exe"
done
