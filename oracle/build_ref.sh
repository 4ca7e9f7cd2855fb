#!/usr/bin/env bash
# Builds the reference ssc-raft CUDA library (parallel-beam FBP / EM / Radon /
# lowpass / flat-dark / BST / rotation-axis / tEMFQ path only) from its own sources, for sm_100a, into oracle/_ref/.
#
# The reference is compiled where it lies (read-only tree); nothing is copied
# into this repository.  Flags follow the reference CMakeLists.txt:8-17
# (fast-math, fmad on, C++17) with the architecture replaced by sm_100a.
# Two include-path workarounds are needed with CUDA 12.9:
#   * nvToolsExt.h moved under nvtx3 (used by cuda/src/.../conebeam radon.cu;
#     harmless for the files below),
#   * common/types.hpp is force-included so the NUM_THREADS macro is defined
#     before CUB headers see it.
# The output library is test infrastructure (the checker), never the product.
set -euo pipefail
REF=${RAFT_REFERENCE_DIR:-/root/reference}
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
OBJ="$OUT/obj"
if [ ! -d "$REF/cuda/src" ]; then
  echo "reference sources not found at $REF; skipping oracle/_ref build" >&2
  exit 0
fi
mkdir -p "$OBJ"
SRCS=(
  cuda/src/common/opt.cu
  cuda/src/common/padding.cu
  cuda/src/common/config.cu
  cuda/src/pipelines/process.cu
  cuda/src/processing/filters/filters.cu
  cuda/src/processing/filters/low_pass.cu
  cuda/src/processing/background_correction.cu
  cuda/src/processing/rotation_axis.cu
  cuda/src/geometries/parallel/reconstruction_methods/parameters.cu
  cuda/src/geometries/parallel/reconstruction_methods/fbp.cu
  cuda/src/geometries/parallel/reconstruction_methods/bst.cu
  cuda/src/geometries/parallel/reconstruction_methods/em_rt.cu
  cuda/src/geometries/parallel/reconstruction_methods/kernels/em_RT_kernel.cu
  cuda/src/geometries/parallel/reconstruction_methods/em_frequency.cu
  cuda/src/geometries/parallel/forward_methods/radon_rt.cu
  cuda/src/geometries/parallel/forward_methods/radon_fst.cu
  cuda/src/geometries/parallel/forward_methods/kernels/radon_fst_kernel.cu
)
FLAGS=(-std=c++17 -O3 -use_fast_math --expt-extended-lambda -Xcompiler -fPIC
       -gencode arch=compute_100a,code=sm_100a
       -I "$REF/cuda/inc" -I "$REF/cuda/inc/common" -I "$REF/cuda/inc/common10"
       -I /usr/local/cuda/include/nvtx3 -include common/types.hpp)
pids=()
objs=()
for s in "${SRCS[@]}"; do
  o="$OBJ/$(echo "$s" | tr '/' '_' ).o"
  objs+=("$o")
  if [ ! -f "$o" ] || [ "$REF/$s" -nt "$o" ]; then
    nvcc "${FLAGS[@]}" -c "$REF/$s" -o "$o" &
    pids+=($!)
  fi
done
for p in "${pids[@]}"; do wait "$p"; done
nvcc -shared -gencode arch=compute_100a,code=sm_100a "${objs[@]}" -lcufft -lcublas -o "$OUT/libraft_ref.so"
echo "built $OUT/libraft_ref.so"
