#!/usr/bin/env bash
# Builds the reference's own CUDA kernels for the commitment path, straight from the
# reference sources, into oracle/_ref/libvortex_ref.so. Test infrastructure only: the
# GPU parity tests use it to pin the CPU oracle against the reference's kernels, and
# tests/golden/gen_ref_golden.py uses it to produce the committed golden vectors.
# Needs the path of the reference checkout, as the first argument or in REF_ROOT;
# without it (or on a machine without the checkout) the prebuilt library is kept.
#     oracle/build_ref.sh <reference checkout>
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF_ROOT="${1:-${REF_ROOT:-}}"
OUT="$HERE/_ref"
if [ -z "$REF_ROOT" ] || [ ! -d "$REF_ROOT/cuda" ]; then
  echo "reference sources not given or not found (REF_ROOT='$REF_ROOT'); keeping prebuilt $OUT" >&2
  exit 0
fi
mkdir -p "$OUT"
SRCS="circle_ntt.cu circle_ntt_stwo.cu twiddles.cu batch_inverse.cu blake2s.cu merkle_leaves_lifted.cu
      fri.cu constraint.cu quotient.cu bit_reverse_wide.cu fields.cu gather.cu barycentric_eval.cu
      accumulate_lift.cu pack_leaves.cu"
OBJS=""
for s in $SRCS; do
  o="$OUT/${s%.cu}.o"
  nvcc -O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -c "$REF_ROOT/cuda/$s" -o "$o"
  OBJS="$OBJS $o"
done
nvcc -shared -cudart static -gencode arch=compute_100a,code=sm_100a $OBJS -o "$OUT/libvortex_ref.so"
rm -f $OBJS
echo "built $OUT/libvortex_ref.so"
