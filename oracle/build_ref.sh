#!/usr/bin/env bash
# Compiles the reference's galaxy_sim for sm_100a straight from its sources
# (nvcc on src/*.cu with the flags of its CMakeLists.txt:18, no CMake) into
# oracle/_ref/.  A comparison binary for timing the reference's own GPU code
# on a B200; never linked by the product.
# Usage: build_ref.sh <reference dir>   (or NBODYSSEY_REFERENCE=<dir> build_ref.sh)
set -euo pipefail
REF=${1:-${NBODYSSEY_REFERENCE:-}}
if [ -z "$REF" ]; then
  echo "usage: build_ref.sh <reference dir>" >&2
  exit 2
fi
OUT="$(cd "$(dirname "$0")" && pwd)/_ref"
mkdir -p "$OUT"
BIN="$OUT/galaxy_sim"
if [ -x "$BIN" ] && [ -z "$(find "$REF/src" -newer "$BIN" -print -quit)" ]; then
  exit 0
fi
nvcc -O3 --use_fast_math -std=c++17 -rdc=true -gencode arch=compute_100a,code=sm_100a \
  "$REF"/src/main.cu "$REF"/src/simulation.cu "$REF"/src/forces.cu \
  "$REF"/src/forces_bh.cu "$REF"/src/integrator.cu -o "$BIN"
