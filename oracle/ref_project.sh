#!/usr/bin/env bash
# Builds the projection harness over the reference's own emdata::project3d: the reference's
# emdata.cpp and utils.cpp compiled where they lie (read-only, unmodified) with
# ref_project_main.cpp and ref_hdf_stubs.cpp (HDF5 readers that MRC inputs never reach), into
# oracle/_ref/ref_project (TEST INFRASTRUCTURE ONLY: golden projections).  Host C++ only.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${GISSPA_REFERENCE:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF/src/EMReader/emdata.cpp" ]; then
  echo "reference sources not present at $REF; nothing to build"
  exit 0
fi
mkdir -p "$OUT/shim"
cat > "$OUT/shim/hdf5.h" <<'H'
#pragma once
typedef long long hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
H
g++ -std=c++17 -O2 -w -I"$OUT/shim" -I"$REF/include" -I"$REF/include/EMReader" -I"$REF/include/utils" \
  "$REF/src/EMReader/emdata.cpp" "$REF/src/utils/utils.cpp" "$HERE/ref_project_main.cpp" \
  "$HERE/ref_hdf_stubs.cpp" -o "$OUT/ref_project"
echo "built $OUT/ref_project"
