#!/usr/bin/env bash
# Builds the reference's OWN implementation from its sources:
#   oracle/_ref/libkf_ref.so       its host (CPU) path - the oracle's checker
#                                  and the timed CPU baseline;
#   oracle/_ref/libkf_ref_cuda.so  the same plus its CUDA path
#                                  (src/kinectfusion/cuda/*.cu, sm_100a) - the
#                                  reference's GPU pipeline, timed on the same
#                                  GPU as a comparison row;
#   oracle/_ref/libkf_ref_b200.so  its host code with the device seams of
#                                  kinectfusion_b200/glue/b200_backend.cpp over
#                                  this library (the drop-in build).
#
# TEST INFRASTRUCTURE ONLY.  Compiles the reference's translation units where
# they lie, read-only, under $KF_REFERENCE (default /root/reference) -
# nothing is copied into this repository - against this project's Eigen
# stand-in (oracle/ref_shim/Eigen), plus this project's driver
# (oracle/ref_driver.cpp).  The reference's own build system (CMake + CPM
# fetching Eigen, Ceres, fmt, spdlog, ...) is not run; the flags follow its
# release preset (-O3 -DNDEBUG, C++23 host / C++20 CUDA,
# --expt-relaxed-constexpr, src/kinectfusion/CMakeLists.txt:43-52), with
# -ffp-contract=off on the host (an x86-64 build without -march flags has no
# FMA to contract into) and the B200's sm_100a for the device code.
# Outputs go to oracle/_ref/ only (git-ignored; they travel to the GPU box
# with the rest of the tree).  Each library is rebuilt only when one of its
# inputs is newer.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${KF_REFERENCE:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -d "$REF/src/kinectfusion" ]; then
  echo "reference sources not found at $REF; oracle/_ref not built" >&2
  exit 0
fi
mkdir -p "$OUT"
CXX="${CXX:-/usr/bin/g++}"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
TUS=(depth_processing tsdf_integration raycasting marching_cubes icp_optimizer comparison pipeline pipeline_set volume)
CUS=(block_rep depth_processing device_pipeline device_volume icp_correspondence occupancy raycasting tsdf_integration)
HOST_FLAGS=(-std=c++23 -O3 -DNDEBUG -fPIC -ffp-contract=off -fno-fast-math -w -I"$HERE/ref_shim" -I"$REF/include")
INPUTS=("$HERE/ref_driver.cpp" "$HERE/ref_build.sh" "$HERE"/ref_shim/Eigen/* "$HERE/../include/kf_b200.h"
        "$REF"/include/kinectfusion/*.hpp "$REF"/include/kinectfusion/*/*.h* "$REF"/src/kinectfusion/*.cpp
        "$REF"/src/kinectfusion/cuda/*)

stale() {  # stale <target>: true when the target is missing or older than an input
  [ -f "$1" ] || return 0
  for f in "${INPUTS[@]}"; do [ "$f" -nt "$1" ] && return 0; done
  return 1
}

build_host() {
  local obj="$OUT/obj_host"
  mkdir -p "$obj"
  local pids=()
  for tu in "${TUS[@]}"; do
    "$CXX" "${HOST_FLAGS[@]}" -c "$REF/src/kinectfusion/$tu.cpp" -o "$obj/$tu.o" & pids+=($!)
  done
  "$CXX" "${HOST_FLAGS[@]}" -c "$HERE/ref_driver.cpp" -o "$obj/ref_driver.o" & pids+=($!)
  for p in "${pids[@]}"; do wait "$p"; done
  "$CXX" -shared -o "$OUT/libkf_ref.so.tmp" "$obj"/*.o
  mv "$OUT/libkf_ref.so.tmp" "$OUT/libkf_ref.so"
  rm -rf "$obj"
}

build_cuda() {
  local obj="$OUT/obj_cuda"
  mkdir -p "$obj"
  local cuda_flags=(-std=c++20 -O3 -DNDEBUG --expt-relaxed-constexpr -gencode arch=compute_100a,code=sm_100a
                    -Xcompiler -fPIC -Xcompiler -ffp-contract=off -ccbin "$CXX" -w -DKINECTFUSION_HAS_CUDA
                    -I"$HERE/ref_shim" -I"$REF/include" -I"$REF/src/kinectfusion/cuda")
  local pids=()
  for tu in "${TUS[@]}"; do
    "$CXX" "${HOST_FLAGS[@]}" -DKINECTFUSION_HAS_CUDA -I/usr/local/cuda/include \
      -c "$REF/src/kinectfusion/$tu.cpp" -o "$obj/$tu.o" & pids+=($!)
  done
  "$CXX" "${HOST_FLAGS[@]}" -DKINECTFUSION_HAS_CUDA -DKF_REF_CUDA -I/usr/local/cuda/include \
    -c "$HERE/ref_driver.cpp" -o "$obj/ref_driver.o" & pids+=($!)
  for cu in "${CUS[@]}"; do
    "$NVCC" "${cuda_flags[@]}" -c "$REF/src/kinectfusion/cuda/$cu.cu" -o "$obj/cuda_$cu.o" & pids+=($!)
  done
  for p in "${pids[@]}"; do wait "$p"; done
  "$NVCC" -shared -ccbin "$CXX" -gencode arch=compute_100a,code=sm_100a -o "$OUT/libkf_ref_cuda.so.tmp" "$obj"/*.o
  mv "$OUT/libkf_ref_cuda.so.tmp" "$OUT/libkf_ref_cuda.so"
  rm -rf "$obj"
}

# The reference's own host code with its device seams taken by this
# project's glue (kinectfusion_b200/glue/b200_backend.cpp) over
# kinectfusion_b200/libkf_b200.so: the reference's loop running on this
# library, as a maintainer's drop-in build would.
build_glue() {
  local obj="$OUT/obj_glue"
  mkdir -p "$obj"
  local pids=()
  for tu in "${TUS[@]}"; do
    "$CXX" "${HOST_FLAGS[@]}" -DKINECTFUSION_HAS_CUDA -I/usr/local/cuda/include \
      -c "$REF/src/kinectfusion/$tu.cpp" -o "$obj/$tu.o" & pids+=($!)
  done
  "$CXX" "${HOST_FLAGS[@]}" -DKINECTFUSION_HAS_CUDA -DKF_REF_CUDA -I/usr/local/cuda/include \
    -c "$HERE/ref_driver.cpp" -o "$obj/ref_driver.o" & pids+=($!)
  "$CXX" "${HOST_FLAGS[@]}" -DKINECTFUSION_HAS_CUDA -I"$HERE/../include" \
    -c "$HERE/../kinectfusion_b200/glue/b200_backend.cpp" -o "$obj/b200_backend.o" & pids+=($!)
  for p in "${pids[@]}"; do wait "$p"; done
  "$CXX" -shared -o "$OUT/libkf_ref_b200.so.tmp" "$obj"/*.o -L"$HERE/../kinectfusion_b200" -lkf_b200 \
    -Wl,-rpath,'$ORIGIN/../../kinectfusion_b200' -L/usr/local/cuda/lib64 -lcudart -Wl,-rpath,/usr/local/cuda/lib64
  mv "$OUT/libkf_ref_b200.so.tmp" "$OUT/libkf_ref_b200.so"
  rm -rf "$obj"
}

if stale "$OUT/libkf_ref.so"; then build_host; fi
if [ -x "$NVCC" ] && stale "$OUT/libkf_ref_cuda.so"; then build_cuda; fi
INPUTS+=("$HERE/../kinectfusion_b200/glue/b200_backend.cpp" "$HERE/../kinectfusion_b200/libkf_b200.so")
if [ -f "$HERE/../kinectfusion_b200/libkf_b200.so" ] && stale "$OUT/libkf_ref_b200.so"; then build_glue; fi
echo "$OUT/libkf_ref.so"
