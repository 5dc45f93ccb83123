// kf_sampler.cuh - the trilinear sampler of the raycast and the mesher
// (TrilinearSampler, volume_sampler.hpp:116-255; trilinear.hpp:85-269).
//
// Arithmetic is the host expression order (the library builds with
// --fmad=false, -prec-div=true, -prec-sqrt=true), so a sample is
// bit-identical to the CPU sampler of the same volume.
#pragma once

#include "kf_common.cuh"

namespace kf {

template <int Kind>
struct Sampler {
  using VT = VoxelTraits<Kind>;
  using Raw = typename VT::Raw;
  VolumeDev v;

  __device__ __forceinline__ f3 grid_of(f3 p) const { return (p - v.origin) * v.inv_voxel_size; }

  __device__ __forceinline__ bool contains(f3 g) const {
    return g.x >= 0.0f && g.y >= 0.0f && g.z >= 0.0f && g.x < static_cast<float>(v.rx) &&
           g.y < static_cast<float>(v.ry) && g.z < static_cast<float>(v.rz);
  }

  // Corner pointer (clipped), nullptr when outside or unallocated.
  __device__ __forceinline__ const Raw* corner(int x, int y, int z) const {
    if (x < 0 || y < 0 || z < 0 || x >= static_cast<int>(v.rx) || y >= static_cast<int>(v.ry) ||
        z >= static_cast<int>(v.rz)) {
      return nullptr;
    }
    const long long i = storage_index(v, static_cast<uint32_t>(x), static_cast<uint32_t>(y), static_cast<uint32_t>(z));
    if (i < 0) return nullptr;
    return reinterpret_cast<const Raw*>(v.voxels) + i;
  }

  __device__ __forceinline__ static float axis_weight(float f, int o) { return o == 0 ? 1.0f - f : f; }

  // TrilinearSampler::tsdf + trilinear::blend_tsdf
  __device__ bool tsdf(f3 point, int policy, float& out) const {
    const f3 g = grid_of(point);
    if (!contains(g)) return false;
    const f3 gg = make(g.x - 0.5f, g.y - 0.5f, g.z - 0.5f);
    const f3 fl = make(floorf(gg.x), floorf(gg.y), floorf(gg.z));
    const int bx = static_cast<int>(fl.x), by = static_cast<int>(fl.y), bz = static_cast<int>(fl.z);
    const f3 fr = gg - fl;
    float acc = 0.0f, ws = 0.0f;
    int valid = 0;
    if (bx >= 0 && by >= 0 && bz >= 0 && (bx & 7) != 7 && (by & 7) != 7 && (bz & 7) != 7 &&
        bx + 1 < static_cast<int>(v.rx) && by + 1 < static_cast<int>(v.ry) && bz + 1 < static_cast<int>(v.rz)) {
      // All eight corners in one brick: one storage lookup (sparse storage:
      // one block-table probe; an unallocated block has no corner), fixed
      // offsets from the base voxel, loads issued together, blended in the
      // reference corner order.
      const long long base =
          storage_index(v, static_cast<uint32_t>(bx), static_cast<uint32_t>(by), static_cast<uint32_t>(bz));
      const Raw* b = reinterpret_cast<const Raw*>(v.voxels) + (base < 0 ? 0 : base);
      Raw r[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) r[c] = base < 0 ? VT::unobserved() : __ldg(b + ((c >> 2) * 64 + ((c >> 1) & 1) * 8 + (c & 1)));
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (!VT::observed(r[c]) || !VT::finite(r[c])) continue;
        const float w = axis_weight(fr.x, c & 1) * axis_weight(fr.y, (c >> 1) & 1) * axis_weight(fr.z, c >> 2);
        acc += w * VT::tsdf(r[c]);
        ws += w;
        ++valid;
      }
    } else {
#pragma unroll
    for (int oz = 0; oz <= 1; ++oz) {
#pragma unroll
      for (int oy = 0; oy <= 1; ++oy) {
#pragma unroll
        for (int ox = 0; ox <= 1; ++ox) {
          const Raw* c = corner(bx + ox, by + oy, bz + oz);
          if (c == nullptr) continue;
          const Raw r = __ldg(c);
          if (!VT::observed(r) || !VT::finite(r)) continue;
          const float w = axis_weight(fr.x, ox) * axis_weight(fr.y, oy) * axis_weight(fr.z, oz);
          acc += w * VT::tsdf(r);
          ws += w;
          ++valid;
        }
      }
    }
    }
    if (policy == KF_CORNERS_REQUIRE_ALL && valid < 8) return false;
    if (ws <= 1.0e-6f) return false;
    const float d = acc / ws;
    if (!isfinite(d)) return false;
    out = d;
    return true;
  }

  // TrilinearSampler::color + trilinear::blend_color
  __device__ bool color(f3 point, f3& out) const {
    if (v.colors == nullptr) return false;  // no colour facet
    const f3 g = grid_of(point);
    if (!contains(g)) return false;
    const f3 gg = make(g.x - 0.5f, g.y - 0.5f, g.z - 0.5f);
    const f3 fl = make(floorf(gg.x), floorf(gg.y), floorf(gg.z));
    const int bx = static_cast<int>(fl.x), by = static_cast<int>(fl.y), bz = static_cast<int>(fl.z);
    const f3 fr = gg - fl;
    f3 acc = make(0.0f, 0.0f, 0.0f);
    float ws = 0.0f;
#pragma unroll
    for (int oz = 0; oz <= 1; ++oz) {
#pragma unroll
      for (int oy = 0; oy <= 1; ++oy) {
#pragma unroll
        for (int ox = 0; ox <= 1; ++ox) {
          const Raw* c = corner(bx + ox, by + oy, bz + oz);
          if (c == nullptr) continue;
          const float4 cv = __ldg(v.colors + (c - reinterpret_cast<const Raw*>(v.voxels)));
          if (cv.w <= 0.0f) continue;
          const float w = axis_weight(fr.x, ox) * axis_weight(fr.y, oy) * axis_weight(fr.z, oz);
          acc = acc + make(cv.x, cv.y, cv.z) * w;
          ws += w;
        }
      }
    }
    if (ws <= 1.0e-6f) return false;
    out = acc / ws;
    return true;
  }

  // trilinear::central_normal (trilinear.hpp:243-266).  The six samples
  // are independent reads of an unchanging volume, so all are taken before
  // any is tested: the result is that of the reference's early-exit order.
  __device__ bool central_normal(f3 p, int policy, f3& out) const {
    const float vs = v.voxel_size;
    float xp = 0.0f, xm = 0.0f, yp = 0.0f, ym = 0.0f, zp = 0.0f, zm = 0.0f;
    const bool ok = tsdf(make(p.x + vs, p.y + 0.0f, p.z + 0.0f), policy, xp) &
                    tsdf(make(p.x - vs, p.y - 0.0f, p.z - 0.0f), policy, xm) &
                    tsdf(make(p.x + 0.0f, p.y + vs, p.z + 0.0f), policy, yp) &
                    tsdf(make(p.x - 0.0f, p.y - vs, p.z - 0.0f), policy, ym) &
                    tsdf(make(p.x + 0.0f, p.y + 0.0f, p.z + vs), policy, zp) &
                    tsdf(make(p.x - 0.0f, p.y - 0.0f, p.z - vs), policy, zm);
    if (!ok) return false;
    const f3 d = make(xp - xm, yp - ym, zp - zm);
    const float length = norm(d);
    if (length <= 0.0f) return false;
    out = d / length;
    return true;
  }

  // TrilinearSampler::cell_normal (volume_sampler.hpp:189-239)
  __device__ bool cell_normal(f3 p, f3& out) const {
    const f3 g = grid_of(p);
    if (!contains(g)) return false;
    const f3 gg = make(g.x - 0.5f, g.y - 0.5f, g.z - 0.5f);
    const f3 fl = make(floorf(gg.x), floorf(gg.y), floorf(gg.z));
    const int bx = static_cast<int>(fl.x), by = static_cast<int>(fl.y), bz = static_cast<int>(fl.z);
    const f3 f = gg - fl;
    float c[2][2][2];
#pragma unroll
    for (int oz = 0; oz <= 1; ++oz) {
#pragma unroll
      for (int oy = 0; oy <= 1; ++oy) {
#pragma unroll
        for (int ox = 0; ox <= 1; ++ox) {
          const Raw* cp = corner(bx + ox, by + oy, bz + oz);
          if (cp == nullptr) return central_normal(p, KF_CORNERS_SKIP_MISSING, out);
          const Raw r = __ldg(cp);
          if (!VT::observed(r) || !VT::finite(r)) return central_normal(p, KF_CORNERS_SKIP_MISSING, out);
          c[oz][oy][ox] = VT::tsdf(r);
        }
      }
    }
    auto lerp = [](float l, float h, float m) { return l + (m * (h - l)); };
    const float gx = lerp(lerp(c[0][0][1] - c[0][0][0], c[0][1][1] - c[0][1][0], f.y),
                          lerp(c[1][0][1] - c[1][0][0], c[1][1][1] - c[1][1][0], f.y), f.z);
    const float gy = lerp(lerp(c[0][1][0] - c[0][0][0], c[0][1][1] - c[0][0][1], f.x),
                          lerp(c[1][1][0] - c[1][0][0], c[1][1][1] - c[1][0][1], f.x), f.z);
    const float gz = lerp(lerp(c[1][0][0] - c[0][0][0], c[1][0][1] - c[0][0][1], f.x),
                          lerp(c[1][1][0] - c[0][1][0], c[1][1][1] - c[0][1][1], f.x), f.y);
    const f3 gr = make(gx, gy, gz);
    const float length = norm(gr);
    if (length <= 0.0f) return false;
    out = gr / length;
    return true;
  }
};

}  // namespace kf
