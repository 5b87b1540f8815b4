#!/bin/bash
# ORACLE / TEST INFRASTRUCTURE ONLY.
# Builds the reference replay driver (oracle/ref_driver.cu) against the
# unmodified reference sources under REF_DIR, output only into oracle/_ref/.
# The reference's own build system (Makefile, mpicxx, sm_52) is not used.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF_DIR="${REF_DIR:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF_DIR/cell.h" ]; then
  echo "reference sources not found at $REF_DIR; skipping oracle/_ref build" >&2
  exit 0
fi
mkdir -p "$OUT"
nvcc -std=c++14 -O2 -shared -Xcompiler -fPIC,-fopenmp -Wno-deprecated-gpu-targets -w \
  -gencode arch=compute_100a,code=sm_100a \
  -include "$HERE/ref_shim/surface_shim.h" -I"$REF_DIR" \
  "$HERE/ref_driver.cu" "$REF_DIR/archAPI.cu" "$REF_DIR/load_data.cu" "$REF_DIR/maxwell.cu" \
  -o "$OUT/libref0buf.so.tmp" -lgomp
mv "$OUT/libref0buf.so.tmp" "$OUT/libref0buf.so"
echo "built $OUT/libref0buf.so"
