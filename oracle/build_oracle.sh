#!/usr/bin/env bash
# Builds the CPU oracle (test infrastructure) into oracle/liboracle.so.
# -ffp-contract=off keeps every a*b+c as two IEEE operations, as the oracle's
# semantics require; OpenMP parallelises over blocks for the CPU baseline.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
g++ -std=c++17 -O3 -march=native -ffp-contract=off -fno-fast-math -fopenmp -fPIC -shared \
    -Wall -Wno-unused-function "$HERE/astc_oracle.cpp" -o "$HERE/liboracle.so.tmp"
mv "$HERE/liboracle.so.tmp" "$HERE/liboracle.so"
echo "build_oracle: built $HERE/liboracle.so"
