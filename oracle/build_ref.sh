#!/usr/bin/env bash
# Builds the MG-alphaGCD reference from its own sources (read in place, never
# copied) into oracle/_ref/ref_harness, with the single-PE shim headers in
# oracle/ref_shim/ standing in for NVSHMEM and MPI.  Test infrastructure only:
# the harness produces the golden vectors under tests/golden/.
#
# Usage: oracle/build_ref.sh [reference_root]
#   reference_root: the argument, else $MG_REFERENCE_ROOT, else /root/reference
# Flags follow the reference's CMakeLists.txt (-O3, -Xcompiler -fopenmp,
# separable compilation, -DTIMING, -D_FORCE_INLINES), with sm_100a as target.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${MG_REFERENCE_ROOT:-/root/reference}}"
OUT="$HERE/_ref"
if [ ! -d "$REF/src" ]; then
  echo "build_ref: no reference tree at $REF (skipped)" >&2
  exit 0
fi
mkdir -p "$OUT/obj"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
FLAGS=(-std=c++17 -O3 -Xptxas -O3 -Xcompiler -O3 -Xcompiler -fopenmp -rdc=true
       -gencode arch=compute_100a,code=sm_100a -DTIMING -D_FORCE_INLINES
       -ccbin /usr/bin/g++ -w
       -I "$HERE/ref_shim" -I "$REF/include" -I "$REF/include/mmio")
SRCS=(src/common.cu src/graph/host_graph.cpp src/graph/gpu_graph.cu src/mmio/mmio_wrapper.cu
      src/bin/BIN.cu src/partition/edge_partition.cu src/louvain/louvain.cu src/louvain/louvain_gl.cu
      src/louvain/louvain_baseline.cu src/coarsen_graph/coarsen_graph_mg.cu)
OBJS=()
pids=()
for s in "${SRCS[@]}"; do
  o="$OUT/obj/$(echo "$s" | tr '/' '_').o"
  OBJS+=("$o")
  if [ ! -f "$o" ] || [ "$REF/$s" -nt "$o" ] || [ "$HERE/ref_shim/nvshmem.h" -nt "$o" ]; then
    "$NVCC" "${FLAGS[@]}" -x cu -c "$REF/$s" -o "$o" &
    pids+=($!)
  fi
done
for p in "${pids[@]}"; do wait "$p"; done
"$NVCC" "${FLAGS[@]}" -x cu -c "$HERE/ref_harness.cu" -o "$OUT/obj/ref_harness.o"
"$NVCC" "${FLAGS[@]}" "${OBJS[@]}" "$OUT/obj/ref_harness.o" -o "$OUT/ref_harness" -lgomp
echo "build_ref: $OUT/ref_harness"
