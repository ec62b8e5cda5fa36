#!/usr/bin/env bash
# Test infrastructure: compiles the reference's OWN octree code in place
# (src/octree_cpu.cpp, src/renderer/octree.cpp) together with the
# project-written shims (oracle/ref_shim) and bridge (oracle/ref_bridge.cpp)
# into oracle/_ref/libveref.so.  Nothing from the reference is copied; output
# goes only to oracle/_ref/ (git-ignored).  Skips quietly when the reference
# tree is absent (it is not present on the GPU boxes, which use the prebuilt
# library).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
# the reference tree: $VE_REFERENCE_ROOT, else BASELINE.json's reference_path
REF="${VE_REFERENCE_ROOT:-}"
if [ -z "$REF" ] && [ -f "$HERE/../BASELINE.json" ]; then
    REF="$(python3 -c 'import json,sys; print(json.load(open(sys.argv[1])).get("reference_path", ""))' "$HERE/../BASELINE.json" 2>/dev/null || true)"
fi
OUT="$HERE/_ref"
if [ ! -f "$REF/src/octree_cpu.cpp" ]; then
    echo "build_ref: reference sources not found at $REF; skipping" >&2
    exit 0
fi
mkdir -p "$OUT"
g++ -std=c++20 -O2 -ffp-contract=off -fPIC -shared -w \
    -I "$HERE/ref_shim" -I "$REF/src" -I "$REF/src/renderer" \
    "$REF/src/octree_cpu.cpp" "$REF/src/renderer/octree.cpp" "$HERE/ref_bridge.cpp" \
    -o "$OUT/libveref.so"
echo "build_ref: wrote $OUT/libveref.so"
