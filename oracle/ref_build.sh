#!/usr/bin/env bash
# Compiles the reference search path from the GisSPA_v2.0 sources where they lie
# (read-only, unmodified) into oracle/_ref/gisspa_ref, for generating golden pick
# lists on a GPU machine (TEST INFRASTRUCTURE ONLY).  HDF5 is never reached with
# MRC inputs: a two-typedef hdf5.h lets the reader headers compile, and
# ref_emdata_min.cpp replaces the HDF5-dependent reader (emdata.cpp).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${GISSPA_REFERENCE:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF/src/norm.cu" ]; then
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
nvcc -gencode arch=compute_100a,code=sm_100a -std=c++17 -O3 -Xcompiler -fopenmp -w \
  -I"$OUT/shim" -I"$REF/include" -I"$REF/include/EMReader" -I"$REF/include/utils" \
  "$REF/src/main.cu" "$REF/src/norm.cu" "$REF/src/nonorm.cu" "$REF/src/kernels.cu" "$REF/src/fft.cu" \
  "$REF/src/helper.cu" "$REF/src/EMReader/DataReader2.cpp" "$REF/src/utils/image.cpp" \
  "$REF/src/utils/templates.cpp" "$REF/src/utils/tileimages.cpp" "$REF/src/utils/utils.cpp" \
  "$HERE/ref_emdata_min.cpp" -o "$OUT/gisspa_ref" -lcufft -lgomp
echo "built $OUT/gisspa_ref"
