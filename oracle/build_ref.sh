#!/usr/bin/env bash
# Builds, from the reference's own sources where they lie (read-only; nothing is copied),
# into oracle/_ref/:
#   * ref_codegen: the reference's text front-end (sysparse.cpp + codegen.cpp, compiled
#     as-is), which regenerates the golden fixtures in tests/golden/;
#   * refk_*.cubin + refk_manifest.json: the reference's NVRTC integrator kernels,
#     unchanged (oracle/build_ref_kernels.py), which the GPU parity tests launch through
#     oracle/_ref/libucb_refharness.so.
# Test infrastructure. Usage: build_ref.sh <path to the reference's U-CUDA directory>
# (or UCB_REFERENCE_DIR). Exits 0 without building when no reference tree is given or
# found: machines without it use the prebuilt files.
set -euo pipefail
REF="${1:-${UCB_REFERENCE_DIR:-}}"
HERE="$(cd "$(dirname "$0")" && pwd)"
if [ -z "$REF" ] || [ ! -f "$REF/codegen.cpp" ]; then
  echo "reference tree not given or not found (${REF:-unset}); skipping oracle/_ref" >&2
  exit 0
fi
mkdir -p "$HERE/_ref"
g++ -O2 -std=c++17 -I"$REF" "$HERE/ref_codegen_main.cpp" "$REF/codegen.cpp" "$REF/sysparse.cpp" \
    -o "$HERE/_ref/ref_codegen"
echo "built $HERE/_ref/ref_codegen"
# The reference's CSV writers (data_export.cpp, compiled as-is) behind a small driver. Its
# GUI-bound analysis_session.h is replaced by oracle/ref_stubs/analysis_session.h: -I- makes
# quoted includes skip the including file's own directory, so the stub directory is searched
# first (the C++ library's parallel-STL headers then need their own directory on the path).
PSTL="$(dirname "$(find /usr/include/c++ -name execution_defs.h 2>/dev/null | head -1)")"
CUDA_HOME="${CUDA_HOME:-/usr/local/cuda}"
g++ -O1 -std=c++17 -I"$HERE/ref_stubs" -I- -I"$REF" -I"$CUDA_HOME/include" ${PSTL:+-I"$PSTL"} \
    "$HERE/ref_csv_main.cpp" "$REF/data_export.cpp" -o "$HERE/_ref/ref_csv" 2>&1 | grep -v "obsolete option" || true
test -x "$HERE/_ref/ref_csv" && echo "built $HERE/_ref/ref_csv"
python "$HERE/build_ref_kernels.py" "$REF" "$HERE/_ref"
