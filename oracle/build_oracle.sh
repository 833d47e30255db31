#!/usr/bin/env bash
# Builds the oracle port (oracle/bbrt_oracle.cpp) into oracle/liboracle.so.
# TEST INFRASTRUCTURE ONLY: the product never loads this library.
# -ffp-contract=off keeps every product and sum rounded separately, as in the
# reference's default x86-64 build.
set -euo pipefail
here="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
g++ -O2 -std=c++17 -fopenmp -fPIC -shared -ffp-contract=off \
    "$here/bbrt_oracle.cpp" -o "$here/liboracle.so.tmp"
mv "$here/liboracle.so.tmp" "$here/liboracle.so"
echo "build_oracle: built $here/liboracle.so"
