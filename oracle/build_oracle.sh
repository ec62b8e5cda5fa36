#!/usr/bin/env bash
# Test infrastructure: builds the CPU oracle (oracle/ve_oracle.cpp) into
# oracle/liboracle.so with the pinned floating-point policy (no contraction,
# IEEE division/sqrt, no fast-math).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
g++ -std=c++17 -O2 -ffp-contract=off -fno-fast-math -fPIC -shared -pthread -Wall -Wno-unused-function \
    "$HERE/ve_oracle.cpp" "$HERE/terrain_oracle.cpp" -o "$HERE/liboracle.so"
echo "build_oracle: wrote $HERE/liboracle.so"
