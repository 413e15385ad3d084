#!/bin/bash
# Builds the reference program (fudan-ppi/Eirene, read-only at REF) from its own
# sources into oracle/_ref/stm_test, for use as the oracle's cross-check only.
# Recipe: nvcc for every .cu (with CUB from the CUDA toolkit pre-included, since
# src/input-helper.h:10 defines offset_t as a macro that breaks CUB's headers),
# g++ for every .cpp, link with cudart.  Nothing is copied into this repository.
set -euo pipefail
# REF: the reference checkout (the directory holding src/); its default is
# where this build environment mounts it
REF=${REF:-/root/reference}
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
if [ ! -d "$REF/src" ]; then echo "reference sources not found at $REF (set REF to the reference checkout)" >&2; exit 2; fi
mkdir -p "$OUT/obj"
objs=()
for f in "$REF"/src/gpu-stm-tree-v*/*.cu; do
  [ -s "$f" ] || continue                      # the *-test.cu files are empty
  o="$OUT/obj/$(basename "$(dirname "$f")")_$(basename "$f" .cu).o"
  "$NVCC" -std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a -include cub/cub.cuh \
      -I"$REF/src" -w -c "$f" -o "$o"
  objs+=("$o")
done
for f in "$REF"/src/*.cpp "$REF"/src/gpu-stm-tree-v*/*.cpp; do
  o="$OUT/obj/$(basename "$(dirname "$f")")_$(basename "$f" .cpp).o"
  g++ -std=c++14 -O3 -w -I"$REF/src" -I/usr/local/cuda/include -c "$f" -o "$o"
  objs+=("$o")
done
"$NVCC" -gencode arch=compute_100a,code=sm_100a -o "$OUT/stm_test" "${objs[@]}" -lcudart
echo "built $OUT/stm_test"
