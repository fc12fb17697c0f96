#!/usr/bin/env bash
# Builds the reference's own rigid-path kernels for the CPU into
# oracle/_ref/libdynref.so (test infrastructure; git-ignored output).
#
# The reference sources are read from $DYNAMAP_REFERENCE (default
# /root/reference, as in oracle/refsrc.py) and
# compiled unmodified except for the CUDA launch syntax, which a C++
# compiler cannot parse: each `K<<<grid, block>>>(` becomes
# `DYNREF_LAUNCH(K)(` (see shim/cuda_runtime.h), and for buildNLSKernel's
# hard-coded photometric weight, which becomes a settable value (below).  The rewritten copies live
# only under oracle/_ref/src and are never committed.  Eigen, OpenCV, the
# CUDA runtime and the CUDA math libraries gnSolver.h includes are replaced
# by the small headers in shim/.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${DYNAMAP_REFERENCE:-/root/reference}"
OUT="$HERE/../_ref"
INC="$REF/include"
if [ ! -d "$INC" ]; then
  echo "reference tree not found at $REF; nothing to build" >&2
  exit 0
fi
mkdir -p "$OUT/src"
SRCS=(geometry/tsdf/tsdf.cu dataStructure/hashTable/hashTable.cu dataStructure/heap/heap.cu
      image/sensor/rgbdImage.cu image/pyramid/pyramid.cu image/conv2D/conv2D.cu
      image/kernel2D/kernel2D.cu solver/gnSolver/gnSolver.cu
      geometry/mesh/meshExtractor/meshExtractor.cu geometry/mesh/mesh.cu
      geometry/mesh/meshSTD.cu)
OBJS=()
INCS=(-I"$HERE/shim" -I"$INC" -I"$INC/dataStructure" -I"$INC/dataStructure/heap"
      -I"$INC/dataStructure/hashTable" -I"$INC/image" -I"$INC/image/sensor"
      -I"$INC/geometry" -I"$INC/geometry/tsdf" -I"$INC/geometry/mesh"
      -I"$INC/geometry/mesh/meshExtractor" -I"$INC/math" -I"$INC/utils"
      -I"$INC/builder" -I"$INC/solver" -I"$INC/solver/gnSolver")
CXXFLAGS=(-O2 -std=c++17 -fPIC -ffp-contract=off -fno-fast-math -w -pthread)
for s in "${SRCS[@]}"; do
  base="$(echo "$s" | tr '/' '_')"
  gen="$OUT/src/${base%.cu}.cpp"
  sed -E 's/\b([A-Za-z_][A-Za-z0-9_]*)[[:space:]]*<<<[^>]*>>>[[:space:]]*\(/DYNREF_LAUNCH(\1)(/g' \
    "$INC/$s" > "$gen"
  if [ "$s" = solver/gnSolver/gnSolver.cu ]; then
    # The one substitution beyond the launch syntax: buildNLSKernel's
    # hard-coded photometric weight (gnSolver.cu:180,
    # `float color_weight = 0.0f;`) reads dynref::color_weight() instead
    # (shim/cuda_runtime.h, default 0), so the colour term can be pinned at
    # a nonzero weight.  The build stops if the declaration is not found
    # exactly once.
    n="$(grep -c 'float color_weight = 0\.0f;' "$gen" || true)"
    if [ "$n" != 1 ]; then
      echo "gnSolver.cu: expected one 'float color_weight = 0.0f;', found $n" >&2
      exit 1
    fi
    sed -i -E 's/float color_weight = 0\.0f;/float color_weight = ::dynref::color_weight();/' "$gen"
  fi
  obj="$OUT/src/${base%.cu}.o"
  g++ "${CXXFLAGS[@]}" "${INCS[@]}" -I"$(dirname "$INC/$s")" -c "$gen" -o "$obj"
  OBJS+=("$obj")
done
g++ "${CXXFLAGS[@]}" "${INCS[@]}" -c "$HERE/driver.cpp" -o "$OUT/src/driver.o"
g++ -shared -pthread -o "$OUT/libdynref.so" "${OBJS[@]}" "$OUT/src/driver.o"
echo "built $OUT/libdynref.so"
