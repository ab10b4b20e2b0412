#!/usr/bin/env bash
# Builds the reference's own CUDA kernels for the commitment path, straight from the
# reference sources, into oracle/_ref/libvortex_ref.so. Test infrastructure only: the
# GPU parity tests use it to pin the CPU oracle against the reference's kernels, and
# tests/golden/gen_ref_golden.py uses it to produce the committed golden vectors.
# Needs the reference checkout (REF_ROOT, default /root/reference); on a machine without
# it the prebuilt library is used as is.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF_ROOT="${REF_ROOT:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -d "$REF_ROOT/cuda" ]; then
  echo "reference sources not found at $REF_ROOT; keeping prebuilt $OUT" >&2
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
