#!/usr/bin/env bash
# Builds the reference's own gpulite GPU path (HaoZeke/linkcell v0.3.3,
# src/gpu/knearest.cpp + src/gpu/capi.cpp) straight from the reference
# sources, with g++ only. Output goes to oracle/_ref/ (git-ignored; it
# stays inside the tree, so copies of the tree carry it). The library
# dlopens libcuda / libcudart / libnvrtc at run time and JIT-compiles its
# kernels, so it needs no CUDA SDK at build time. Used only as a measured
# baseline and cross-check (never linked into the product).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
# the reference checkout: LINKCELL_REFERENCE, else beside the repository
REF="${LINKCELL_REFERENCE:-$HERE/../../reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF/src/gpu/knearest.cpp" ]; then
  echo "reference sources not found at $REF; skipping gpulite build" >&2
  exit 0
fi
mkdir -p "$OUT"
${CXX:-g++} -std=c++17 -O2 -fPIC -shared -DLINKCELL_HAS_GPULITE=1 \
  -I"$REF/include" -I"$REF/third_party/gpulite" -I"$REF/src/gpu" \
  "$REF/src/gpu/knearest.cpp" "$REF/src/gpu/capi.cpp" \
  -ldl -o "$OUT/libref_gpulite.so"
echo "built $OUT/libref_gpulite.so"
