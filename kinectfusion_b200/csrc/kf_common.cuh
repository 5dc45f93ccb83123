// kf_common.cuh - shared device types and math for the sm_100a kernels.
//
// The library is compiled with --fmad=false, -prec-div=true and
// -prec-sqrt=true, so every float expression below rounds each multiply and
// add separately, in the same order as the reference's host C++ (the parity
// oracle).  Citations are file:line in maximsolodukhin/KinectFusion.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/kf_b200.h"

namespace kf {

constexpr float kNaN = __builtin_nanf("");

struct f3 {
  float x, y, z;
};

__host__ __device__ __forceinline__ f3 make(float x, float y, float z) { return f3{x, y, z}; }
__host__ __device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ __forceinline__ f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
// vector.hpp:140-143: (x*x' + y*y') + z*z'
__host__ __device__ __forceinline__ float dot(f3 a, f3 b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }
__host__ __device__ __forceinline__ f3 cross(f3 a, f3 b) {
  return {(a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x)};
}
__device__ __forceinline__ float norm(f3 a) { return sqrtf(dot(a, a)); }
// Host branch of normalized (vector.hpp:164-175): sqrt then three divides.
__device__ __forceinline__ f3 normalized(f3 a) {
  const float length = norm(a);
  return length > 0.0f ? a / length : f3{0.0f, 0.0f, 0.0f};
}
__device__ __forceinline__ bool finite3(f3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
__device__ __forceinline__ f3 nan3() { return {kNaN, kNaN, kNaN}; }

__device__ __forceinline__ f3 load3(const float* p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ f3 ldg3(const float* p) { return {__ldg(p), __ldg(p + 1), __ldg(p + 2)}; }
__device__ __forceinline__ void store3(float* p, f3 a) {
  p[0] = a.x;
  p[1] = a.y;
  p[2] = a.z;
}

// RigidTransform (vector.hpp:209-236) held by value in kernel parameters.
struct Rigid {
  f3 rx, ry, rz, t;
};
__host__ __device__ __forceinline__ Rigid rigid_from(const kf_rigid& r) {
  return Rigid{{r.r[0], r.r[1], r.r[2]}, {r.r[3], r.r[4], r.r[5]}, {r.r[6], r.r[7], r.r[8]},
               {r.t[0], r.t[1], r.t[2]}};
}
__host__ __device__ __forceinline__ f3 rotate(const Rigid& T, f3 p) {
  return {dot(T.rx, p), dot(T.ry, p), dot(T.rz, p)};
}
__host__ __device__ __forceinline__ f3 apply(const Rigid& T, f3 p) { return rotate(T, p) + T.t; }

struct Intr {
  float fx, fy, cx, cy;
};
__host__ __device__ __forceinline__ Intr intr_from(const kf_intrinsics& k) { return {k.fx, k.fy, k.cx, k.cy}; }
// CameraIntrinsics::project (rgbd.hpp:40-44)
__device__ __forceinline__ void project(const Intr& k, f3 p, float& px, float& py) {
  px = ((k.fx * p.x) / p.z) + k.cx;
  py = ((k.fy * p.y) / p.z) + k.cy;
}
// CameraIntrinsics::back_project (rgbd.hpp:52-56)
__device__ __forceinline__ f3 back_project(const Intr& k, float px, float py, float depth) {
  return {((px - k.cx) * depth) / k.fx, ((py - k.cy) * depth) / k.fy, depth};
}

// depth_in_range (rgbd.hpp:122-133)
__device__ __forceinline__ bool depth_in_range(uint16_t raw, float scale, float lo, float hi, float& m) {
  if (raw == 0) return false;
  m = static_cast<float>(raw) / scale;
  return !(m < lo || m > hi);
}

__device__ __forceinline__ float clampf(float v, float lo, float hi) {
  if (v < lo) return lo;
  if (hi < v) return hi;
  return v;
}

// ---- voxel codecs (volume.hpp:25-146) -------------------------------------
constexpr float kQScale = 32767.0f;
constexpr float kQInvScale = 1.0f / 32767.0f;
constexpr float kWScale = 256.0f;
constexpr float kWInvScale = 1.0f / 256.0f;
constexpr float kWMax = 65535.0f / 256.0f;

__device__ __forceinline__ uint16_t bf16_encode(float t) {
  const uint32_t bits = __float_as_uint(clampf(t, -1.0f, 1.0f));
  return static_cast<uint16_t>((bits + 0x7FFFu + ((bits >> 16) & 1u)) >> 16);
}
__device__ __forceinline__ float bf16_decode(uint16_t raw) { return __uint_as_float(static_cast<uint32_t>(raw) << 16); }
__device__ __forceinline__ uint16_t qweight_encode(float w) {
  return static_cast<uint16_t>(clampf(w, 0.0f, kWMax) * kWScale);
}
__device__ __forceinline__ float qweight_decode(uint32_t raw16) { return static_cast<float>(raw16) * kWInvScale; }
__device__ __forceinline__ int16_t qtsdf_encode(float t) {
  return static_cast<int16_t>(clampf(t, -1.0f, 1.0f) * kQScale);
}
__device__ __forceinline__ float qtsdf_decode(int16_t raw) { return static_cast<float>(raw) * kQInvScale; }

// Storage of the three geometric voxels: Voxel (2 x f32, 8 B), QuantizedVoxel
// and Bf16Voxel (u16 distance | u16 weight << 16, 4 B).
template <int Kind>
struct VoxelTraits;

template <>
struct VoxelTraits<KF_VOXEL_FLOAT> {
  using Raw = float2;
  static constexpr int kBytes = 8;
  __device__ __forceinline__ static float tsdf(Raw r) { return r.x; }
  __device__ __forceinline__ static float weight(Raw r) { return r.y; }
  __device__ __forceinline__ static bool observed(Raw r) { return r.y > 0.0f; }
  __device__ __forceinline__ static bool finite(Raw r) { return isfinite(r.x); }
  __device__ __forceinline__ static Raw encode(float t, float w) { return make_float2(t, w); }
  __host__ __device__ static Raw unobserved() { return make_float2(1.0f, 0.0f); }
};

template <>
struct VoxelTraits<KF_VOXEL_QUANTIZED> {
  using Raw = uint32_t;
  static constexpr int kBytes = 4;
  __device__ __forceinline__ static float tsdf(Raw r) { return qtsdf_decode(static_cast<int16_t>(r & 0xFFFFu)); }
  __device__ __forceinline__ static float weight(Raw r) { return qweight_decode(r >> 16); }
  __device__ __forceinline__ static bool observed(Raw r) { return (r >> 16) != 0u; }
  __device__ __forceinline__ static bool finite(Raw) { return true; }
  __device__ __forceinline__ static Raw encode(float t, float w) {
    return static_cast<uint32_t>(static_cast<uint16_t>(qtsdf_encode(t))) |
           (static_cast<uint32_t>(qweight_encode(w)) << 16);
  }
  __host__ __device__ static Raw unobserved() { return 32767u; }
};

template <>
struct VoxelTraits<KF_VOXEL_BF16> {
  using Raw = uint32_t;
  static constexpr int kBytes = 4;
  __device__ __forceinline__ static float tsdf(Raw r) { return bf16_decode(static_cast<uint16_t>(r & 0xFFFFu)); }
  __device__ __forceinline__ static float weight(Raw r) { return qweight_decode(r >> 16); }
  __device__ __forceinline__ static bool observed(Raw r) { return (r >> 16) != 0u; }
  __device__ __forceinline__ static bool finite(Raw) { return true; }
  __device__ __forceinline__ static Raw encode(float t, float w) {
    return static_cast<uint32_t>(bf16_encode(t)) | (static_cast<uint32_t>(qweight_encode(w)) << 16);
  }
  __host__ __device__ static Raw unobserved() { return 0x3F80u; }
};

// Device view of one volume (VolumeView / SparseVolumeView, volume.hpp:291-356,
// block_rep.hpp:26-110).  Sparse volumes resolve blocks through the block table.
struct VolumeDev {
  void* voxels;
  float4* colors;       // nullptr when the color facet is off
  // sparse storage: the voxel-block hash (block_table_lookup); nullptr for
  // dense storage
  const unsigned long long* table;
  uint32_t table_mask;  // entries - 1 (entries a power of two)
  uint32_t rx, ry, rz;
  uint32_t bx, by, bz;  // block extent
  float voxel_size;
  float inv_voxel_size; // 1.0f / voxel_size, as TrilinearSampler (volume_sampler.hpp:172)
  f3 origin;
  float truncation;
};

constexpr uint32_t kUnallocated = 0xFFFFFFFFu;

// The voxel-block hash of sparse storage (the reference's BlockRep maps
// blocks to pool slots through a dense grid of block slots,
// block_rep.hpp:26-110; here an open-addressing table whose size follows the
// pool, not the domain).  Entry = (block << 32) | slot, kEmptyEntry when
// free; linear probing from the block's hash.  Entries are only ever added
// (by the allocation pass, atomicCAS on an empty entry) and the table has at
// least twice as many entries as the pool has slots, so a probe sequence
// always reaches the block's entry or an empty one; every loop is bounded by
// the table size all the same.
constexpr unsigned long long kEmptyEntry = ~0ull;

__host__ __device__ __forceinline__ uint32_t block_hash(uint32_t block) {
  // murmur3's 32-bit finaliser: neighbouring blocks land far apart
  uint32_t h = block;
  h ^= h >> 16;
  h *= 0x85EBCA6Bu;
  h ^= h >> 13;
  h *= 0xC2B2AE35u;
  h ^= h >> 16;
  return h;
}

// Slot of `block`, or kUnallocated.  For kernels that only read the table.
__device__ __forceinline__ uint32_t block_table_lookup(const unsigned long long* __restrict__ table, uint32_t mask,
                                                       uint32_t block) {
  uint32_t h = block_hash(block) & mask;
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const unsigned long long e = __ldg(table + h);
    if (e == kEmptyEntry) return kUnallocated;
    if (static_cast<uint32_t>(e >> 32) == block) return static_cast<uint32_t>(e);
    h = (h + 1u) & mask;
  }
  return kUnallocated;
}

// Voxel storage is bricked: 8x8x8 bricks of 512 contiguous voxels, voxel
// (x, y, z) at brick slot * 512 + ((z & 7) * 8 + (y & 7)) * 8 + (x & 7) (the
// intra-block order of BlockGrid::intra_of_voxel, grid.hpp:54-69).  Dense
// volumes place brick b (x-major block index) at slot b; sparse volumes look
// the slot up in the block table.  A trilinear stencil or an 8-voxel walk along any
// axis stays inside one or two 4 KB bricks, where the reference's
// x-fastest layout puts z-neighbours a whole slice (2 MB at 512^3) apart.
__device__ __forceinline__ uint32_t brick_offset(uint32_t x, uint32_t y, uint32_t z) {
  return ((z & 7u) * 8u + (y & 7u)) * 8u + (x & 7u);
}

// Storage index of an in-bounds voxel, or -1 when its block is not allocated.
__device__ __forceinline__ long long storage_index(const VolumeDev& v, uint32_t x, uint32_t y, uint32_t z) {
  const uint32_t block = ((z >> 3) * v.by + (y >> 3)) * v.bx + (x >> 3);
  if (v.table == nullptr) {
    return static_cast<long long>(block) * 512 + brick_offset(x, y, z);
  }
  const uint32_t slot = block_table_lookup(v.table, v.table_mask, block);
  if (slot == kUnallocated) return -1;
  return static_cast<long long>(slot) * 512 + brick_offset(x, y, z);
}

// VolumeGeometry::cell_center (volume.hpp:276-283)
__device__ __forceinline__ f3 cell_center(const VolumeDev& v, uint32_t x, uint32_t y, uint32_t z) {
  const f3 c = make(static_cast<float>(x) + 0.5f, static_cast<float>(y) + 0.5f, static_cast<float>(z) + 0.5f) *
               v.voxel_size;
  return v.origin + c;
}

// pixel_from_color (rgbd.hpp:88-98)
__device__ __forceinline__ uint32_t pixel_from_color(f3 c) {
  const uint32_t r = static_cast<uint32_t>(clampf(c.x, 0.0f, 255.0f));
  const uint32_t g = static_cast<uint32_t>(clampf(c.y, 0.0f, 255.0f));
  const uint32_t b = static_cast<uint32_t>(clampf(c.z, 0.0f, 255.0f));
  return r | (g << 8) | (b << 16) | (0xFFu << 24);
}
// color_from_pixel (rgbd.hpp:102-107)
__device__ __forceinline__ f3 color_from_pixel(uint32_t p) {
  return make(static_cast<float>(p & 0xFFu), static_cast<float>((p >> 8) & 0xFFu),
              static_cast<float>((p >> 16) & 0xFFu));
}

inline unsigned ceil_div(unsigned a, unsigned b) { return (a + b - 1) / b; }

}  // namespace kf
