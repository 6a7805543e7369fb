#!/bin/bash
# Builds the reference's own GPU pair kernel and invariance code, unmodified, from the
# sources where they lie, into oracle/_ref/libref_bia.so (test and baseline
# infrastructure; git-ignored).  Exports the reference's find_dxyuv_kernel_ and
# invariance_gpu_ (bia/find_dXYUV_kernel.cu:526-561, bia/invariance.cu:50-110).
# Only METHOD = 1 (ALG) of the kernel is ever called: its RKF mode reaches a
# __syncthreads() inside divergent code (bia/bia-rkf.cu:102).
#
#   bash oracle/build_ref.sh <reference checkout>      (or BIA_REFERENCE_DIR=<checkout>)
set -e
REF=${1:-${BIA_REFERENCE_DIR:-}}
if [ -z "$REF" ]; then
  echo "usage: build_ref.sh <reference checkout> (or set BIA_REFERENCE_DIR); skipping"
  exit 0
fi
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
mkdir -p "$OUT"
if [ ! -f "$REF/bia/find_dXYUV_kernel.cu" ]; then
  echo "reference sources not found under $REF; skipping"
  exit 0
fi
NVCC=${NVCC:-nvcc}
$NVCC -gencode arch=compute_100a,code=sm_100a -O3 -Xcompiler -fPIC -shared -w \
      -I"$REF/bia" "$REF/bia/find_dXYUV_kernel.cu" "$REF/bia/invariance.cu" \
      -o "$OUT/libref_bia.so"
echo "built $OUT/libref_bia.so"
