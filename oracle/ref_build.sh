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
NV=(nvcc -gencode arch=compute_100a,code=sm_100a -std=c++17 -Xcompiler -fopenmp -w
    -I"$OUT/shim" -I"$REF/include" -I"$REF/include/EMReader" -I"$REF/include/utils")
REST=("$REF/src/main.cu" "$REF/src/norm.cu" "$REF/src/nonorm.cu" "$REF/src/fft.cu"
      "$REF/src/helper.cu" "$REF/src/EMReader/DataReader2.cpp" "$REF/src/utils/image.cpp"
      "$REF/src/utils/templates.cpp" "$REF/src/utils/tileimages.cpp" "$REF/src/utils/utils.cpp"
      "$HERE/ref_emdata_min.cpp")
"${NV[@]}" -O3 "${REST[@]}" "$REF/src/kernels.cu" -o "$OUT/gisspa_ref" -lcufft -lgomp
echo "built $OUT/gisspa_ref"
# Test-only variant: the same sources and flags, except that kernels.cu is compiled with
# device debug code generation (-G: no optimisation, every shared-memory access issued as
# written and in order).  The warp-synchronous reduction tails of compute_sum_sqr and
# compute_area_sum_ofSQR (kernels.cu:362-375, 423-436: no volatile, no __syncwarp) then read
# what their neighbours wrote, so this build gives those sums their intended values; its pick
# lists tell how much of the reference's norm_type=1 score spread those tails cause.
mkdir -p "$OUT/sync_obj"
"${NV[@]}" -G -c "$REF/src/kernels.cu" -o "$OUT/sync_obj/kernels.o"
"${NV[@]}" -O3 "${REST[@]}" "$OUT/sync_obj/kernels.o" -o "$OUT/gisspa_ref_sync" -lcufft -lgomp
echo "built $OUT/gisspa_ref_sync"
