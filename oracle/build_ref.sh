#!/usr/bin/env bash
# Builds oracle/_ref/libastcref.so from the reference's own CPU sources, where
# they lie in the read-only reference checkout, plus oracle/ref_shim.cpp.
# Test infrastructure only: the product never links this library.
# The reference's GPU path (WebGPU/Dawn) is not built; only these four sources:
#   code/metadata_structures.cpp  code/partition_tables.cpp
#   code/physical_compression.cpp code/astc_store.cpp
# Usage: oracle/build_ref.sh <reference_root>   (the checkout holding code/ and shaders/)
set -euo pipefail
if [ $# -lt 1 ]; then
  echo "usage: $0 <reference_root>" >&2
  exit 2
fi
REF="$1"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
if [ ! -d "$REF/code" ]; then
  echo "build_ref: reference sources not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
g++ -std=c++20 -O2 -fPIC -shared -fpermissive -w \
    -include string -include cmath -include limits -include algorithm -include set \
    -I "$HERE/stub" -I "$REF/code" \
    "$REF/code/metadata_structures.cpp" "$REF/code/partition_tables.cpp" \
    "$REF/code/physical_compression.cpp" "$REF/code/astc_store.cpp" \
    "$HERE/ref_shim.cpp" -o "$OUT/libastcref.so.tmp"
mv "$OUT/libastcref.so.tmp" "$OUT/libastcref.so"
echo "build_ref: built $OUT/libastcref.so"
