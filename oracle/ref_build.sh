#!/usr/bin/env bash
# Builds the reference's OWN host implementation as oracle/_ref/libkf_ref.so.
#
# TEST INFRASTRUCTURE ONLY (the checker of the CPU oracle).  Compiles the
# reference's CPU translation units where they lie, read-only, under
# $KF_REFERENCE (default /root/reference) - nothing is copied into this
# repository - with g++ -std=c++23, without KINECTFUSION_HAS_CUDA (so the
# CPU stubs of the device seams are used), against this project's Eigen
# stand-in (oracle/ref_shim/Eigen), plus this project's driver
# (oracle/ref_driver.cpp).  The reference's own build system (CMake + CPM
# fetching Eigen, Ceres, fmt, spdlog, ...) is not run.
#
# Flags: -O2 -ffp-contract=off (no FMA contraction, as an x86-64 build of
# the reference without -march flags evaluates its float expressions), no
# fast-math.  Output goes to oracle/_ref/ only (git-ignored; it travels to
# the GPU box with the rest of the tree).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${KF_REFERENCE:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -d "$REF/src/kinectfusion" ]; then
  echo "reference sources not found at $REF; oracle/_ref not built" >&2
  exit 0
fi
mkdir -p "$OUT/obj"
CXX="${CXX:-/usr/bin/g++}"
FLAGS=(-std=c++23 -O2 -fPIC -ffp-contract=off -fno-fast-math -w -I"$HERE/ref_shim" -I"$REF/include")
TUS=(depth_processing tsdf_integration raycasting marching_cubes icp_optimizer comparison pipeline pipeline_set volume)
pids=()
for tu in "${TUS[@]}"; do
  "$CXX" "${FLAGS[@]}" -c "$REF/src/kinectfusion/$tu.cpp" -o "$OUT/obj/$tu.o" &
  pids+=($!)
done
"$CXX" "${FLAGS[@]}" -c "$HERE/ref_driver.cpp" -o "$OUT/obj/ref_driver.o" &
pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
"$CXX" -shared -o "$OUT/libkf_ref.so.tmp" "$OUT"/obj/*.o
mv "$OUT/libkf_ref.so.tmp" "$OUT/libkf_ref.so"
rm -rf "$OUT/obj"
echo "$OUT/libkf_ref.so"
