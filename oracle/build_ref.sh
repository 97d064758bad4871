#!/usr/bin/env bash
# Builds the reference's own noblockage_10m program from its sources, unmodified,
# into oracle/_ref/ (git-ignored; it travels with the tree to the GPU host).
# Used only to generate golden fixtures (tests/golden/make_reference_fixtures.py).
# Only this variant is built: its kernels stay in bounds on valid inputs, while
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
src="$REF/vissgen3d_noblockage_10m.cu"
exe="$OUT/vissgen3d_noblockage_10m"
if [ ! -x "$exe" ] || [ "$src" -nt "$exe" ]; then
  nvcc -O2 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fopenmp -I "$REF" "$src" -o "$exe" -lgomp
fi
echo "$exe"
