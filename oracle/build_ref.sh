#!/usr/bin/env bash
# Compile the reference's own C++ sources (its pybind11 module Cvortrace) into
# oracle/_ref/.  Test infrastructure only: the module is the ground truth the
# C restatement in oracle/vt_oracle.c is pinned against, and the CPU arm of
# bench.py.  The recipe is the plain g++ line over the reference's src/*.cpp;
# the reference's CMake build is not used.  No -march / -ffast-math, so x86-64
# SSE2 FP64 code has no FMA contraction.
set -euo pipefail
REF="${VT_REFERENCE_DIR:-/root/reference}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
if [ ! -d "$REF/src" ]; then
  echo "reference sources not found at $REF; skipping" >&2
  exit 0
fi
PY="${PYTHON:-python3}"
SUFFIX="$($PY -c 'import sysconfig;print(sysconfig.get_config_var("EXT_SUFFIX"))')"
INCS="$($PY -m pybind11 --includes)"
mkdir -p "$OUT"
TARGET="$OUT/Cvortrace$SUFFIX"
NEWEST_SRC="$(ls -t "$REF"/src/*.cpp "$REF"/include/*.hpp | head -1)"
if [ -f "$TARGET" ] && [ "$TARGET" -nt "$NEWEST_SRC" ] && [ "$TARGET" -nt "$0" ]; then
  exit 0
fi
g++ -O3 -std=c++17 -fPIC -shared -fopenmp -I "$REF/include" $INCS \
    "$REF"/src/*.cpp -o "$TARGET.tmp"
mv "$TARGET.tmp" "$TARGET"
echo "built $TARGET"
