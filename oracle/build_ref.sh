#!/usr/bin/env bash
# Builds the reference oracle into oracle/_ref/ — TEST INFRASTRUCTURE ONLY.
#
#   oracle/_ref/libbbrt_ref.so      the reference's headers + oracle/ref_harness.cpp
#   oracle/_ref/triangle_intersect  the reference's own unit test, built as is
#
# The reference (manuelarturosantana/BillardBallRayTracing3D) is header-only
# C++17.  Its MKL and MPI includes are satisfied by oracle/shim/ (a naive
# row-major cblas_dgemm and an empty mpi.h).  Its trace constants are
# `static constexpr` members (include/ScatObjects/SurfacePatch.hpp:117,121,122);
# to run a workload's coarse-grid size and Newton tolerance they are turned
# into `static inline` members in a throw-away copy of the headers made under
# oracle/_ref/src, which is deleted again once the library is built.
#
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]
#   REFERENCE_ROOT defaults to $BBRT_REFERENCE_ROOT, else to a directory named
#   `reference` beside this repository's root.
set -euo pipefail
here="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
ref="${1:-${BBRT_REFERENCE_ROOT:-$(dirname "$(dirname "$here")")/reference}}"
out="$here/_ref"
if [ ! -d "$ref/include" ]; then
    echo "build_ref: no reference at $ref; nothing built" >&2
    exit 0
fi
mkdir -p "$out"
src="$out/src"
rm -rf "$src"
mkdir -p "$src"
cp -r "$ref/include" "$src/include"
sed -i -E 's/static constexpr (int|double) (kCoarseGridSize|kNewtonMaxIters|kNewtonTol)/static inline \1 \2/' \
    "$src/include/ScatObjects/SurfacePatch.hpp"
if [ "$(grep -c 'static inline' "$src/include/ScatObjects/SurfacePatch.hpp")" != "3" ]; then
    echo "build_ref: constant patch did not apply" >&2
    rm -rf "$src"
    exit 1
fi
g++ -O3 -std=c++17 -fopenmp -fPIC -shared \
    -I"$here/shim" -I"$src/include" \
    "$here/ref_harness.cpp" -o "$out/libbbrt_ref.so.tmp"
mv "$out/libbbrt_ref.so.tmp" "$out/libbbrt_ref.so"
rm -rf "$src"
# The reference's unit test, from its sources where they lie.
g++ -O2 -std=c++17 "$ref/tests/Triangle_Intersect.cpp" -o "$out/triangle_intersect"
echo "build_ref: built $out/libbbrt_ref.so and $out/triangle_intersect"
