#!/usr/bin/env bash
# Builds the reference's own text front-end (sysparse.cpp + codegen.cpp, compiled as-is
# from the read-only reference tree) into oracle/_ref/ref_codegen. Test infrastructure:
# it only regenerates the golden fixtures in tests/golden/. Needs the reference tree;
# exits 0 without building when it is absent (machines without the reference tree use the prebuilt files).
set -euo pipefail
REF="${UCB_REFERENCE_DIR:-/root/reference/U-CUDA}"
HERE="$(cd "$(dirname "$0")" && pwd)"
if [ ! -f "$REF/codegen.cpp" ]; then
  echo "reference tree not found at $REF; skipping oracle/_ref" >&2
  exit 0
fi
mkdir -p "$HERE/_ref"
g++ -O2 -std=c++17 -I"$REF" "$HERE/ref_codegen_main.cpp" "$REF/codegen.cpp" "$REF/sysparse.cpp" \
    -o "$HERE/_ref/ref_codegen"
echo "built $HERE/_ref/ref_codegen"
