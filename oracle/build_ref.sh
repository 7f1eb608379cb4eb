#!/usr/bin/env bash
# Builds the reference library (shangar21/cuhc, src/capi.cu and the headers it
# includes) from its own sources for sm_100a, into oracle/_ref/libcuhc.so.
#
# Test infrastructure only: the parity tests load it as the bit-parity oracle
# for the GPU path (with spatial pruning forced off, cuhc_set_pruning(2), the
# reference breaks ties by original point index exactly as this library does),
# and `bench.py --impl reference` times it. Nothing in the product links it.
#
# The reference sources are read where they lie; nothing is copied. Same flags
# as the reference's CMake Release build (CMakeLists.txt:15-41): C++17, -O3,
# -lineinfo, position-independent shared library.
#
# Usage: oracle/build_ref.sh [reference root]
# The root defaults to $CUHC_REFERENCE_ROOT, else /root/reference (where this
# recipe finds the read-only checkout of the reference).
set -euo pipefail
REF="${1:-${CUHC_REFERENCE_ROOT:-/root/reference}}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
if [ ! -f "$REF/src/capi.cu" ]; then
  echo "reference sources not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
# Rebuild only when a reference source is newer than the library.
if [ -f "$OUT/libcuhc.so" ] && [ -z "$(find "$REF/src" -newer "$OUT/libcuhc.so" -print -quit)" ]; then
  exit 0
fi
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
"$NVCC" -std=c++17 -O3 -DNDEBUG -lineinfo -shared -Xcompiler -fPIC \
  -gencode arch=compute_100a,code=sm_100a \
  -I"$REF/src" "$REF/src/capi.cu" -o "$OUT/libcuhc.so.tmp"
mv "$OUT/libcuhc.so.tmp" "$OUT/libcuhc.so"
echo "built $OUT/libcuhc.so"
