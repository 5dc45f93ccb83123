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

  // The six points of central_normal, in its order: +x, -x, +y, -y, +z, -z.
  __device__ __forceinline__ static void central_points(f3 p, float vs, f3 (&pt)[6]) {
    pt[0] = make(p.x + vs, p.y + 0.0f, p.z + 0.0f);
    pt[1] = make(p.x - vs, p.y - 0.0f, p.z - 0.0f);
    pt[2] = make(p.x + 0.0f, p.y + vs, p.z + 0.0f);
    pt[3] = make(p.x - 0.0f, p.y - vs, p.z - 0.0f);
    pt[4] = make(p.x + 0.0f, p.y + 0.0f, p.z + vs);
    pt[5] = make(p.x - 0.0f, p.y - 0.0f, p.z - vs);
  }

  // tsdf() at the six points of central_normal in one pass, for the common
  // case: dense storage, each point's stencil base one voxel from the base
  // c of the +y point's x and the +x point's y and z, along the point's own
  // axis (its other two coordinates are the centre's, so they share c's),
  // and every voxel of the plus-shaped neighbourhood (c + {-1..2} along one
  // axis, c + {0, 1} along the others: 32 voxels) inside the volume.  The 32
  // voxels are read once; each point blends its eight corners in the
  // sampler's order with its own weights, so `val` holds the values tsdf()
  // returns and `ok` is true when all six exist.  Returns false (nothing
  // decided) when the case does not apply.
  __device__ __forceinline__ bool central_six(f3 p, int policy, float (&val)[6], bool& ok) const {
    if (v.table != nullptr) return false;
    f3 pt[6];
    central_points(p, v.voxel_size, pt);
    f3 g[6];
    bool inside = true;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      g[k] = grid_of(pt[k]);
      inside = inside && contains(g[k]);
    }
    if (!inside) {  // a point outside the volume has no value
      ok = false;
      return true;
    }
    f3 fr[6];
    int b[6][3];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const f3 gg = make(g[k].x - 0.5f, g[k].y - 0.5f, g[k].z - 0.5f);
      const f3 fl = make(floorf(gg.x), floorf(gg.y), floorf(gg.z));
      b[k][0] = static_cast<int>(fl.x);
      b[k][1] = static_cast<int>(fl.y);
      b[k][2] = static_cast<int>(fl.z);
      fr[k] = gg - fl;
    }
    const int cx = b[2][0], cy = b[0][1], cz = b[0][2];
    const bool pattern = b[0][0] == cx + 1 && b[0][2] == cz && b[1][0] == cx - 1 && b[1][1] == cy &&
                         b[1][2] == cz && b[2][1] == cy + 1 && b[2][2] == cz && b[3][0] == cx &&
                         b[3][1] == cy - 1 && b[3][2] == cz && b[4][0] == cx && b[4][1] == cy &&
                         b[4][2] == cz + 1 && b[5][0] == cx && b[5][1] == cy && b[5][2] == cz - 1;
    if (!pattern || cx < 1 || cy < 1 || cz < 1 || cx + 2 >= static_cast<int>(v.rx) ||
        cy + 2 >= static_cast<int>(v.ry) || cz + 2 >= static_cast<int>(v.rz)) {
      return false;
    }
    // storage_index is separable in dense storage: x, y and z terms
    size_t tx[4], ty[4], tz[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint32_t x = static_cast<uint32_t>(cx - 1 + i), y = static_cast<uint32_t>(cy - 1 + i),
                     z = static_cast<uint32_t>(cz - 1 + i);
      tx[i] = static_cast<size_t>(x >> 3) * 512u + (x & 7u);
      ty[i] = static_cast<size_t>(y >> 3) * v.bx * 512u + (y & 7u) * 8u;
      tz[i] = static_cast<size_t>(z >> 3) * v.by * v.bx * 512u + (z & 7u) * 64u;
    }
    const Raw* __restrict__ vox = reinterpret_cast<const Raw*>(v.voxels);
    // a corner's value, NaN where the sampler skips it (unobserved or not finite)
    auto value = [&](int dx, int dy, int dz) {
      const Raw r = __ldg(vox + (tx[dx + 1] + ty[dy + 1] + tz[dz + 1]));
      return VT::observed(r) && VT::finite(r) ? VT::tsdf(r) : __int_as_float(0x7fffffff);
    };
    float mid[2][2][2], ax[2][2][2], ay[2][2][2], az[2][2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          mid[i][j][k] = value(i, j, k);
          ax[i][j][k] = value(i == 0 ? -1 : 2, j, k);
          ay[i][j][k] = value(j, i == 0 ? -1 : 2, k);
          az[i][j][k] = value(j, k, i == 0 ? -1 : 2);
        }
      }
    }
    auto at = [&](int dx, int dy, int dz) {
      if (dx < 0 || dx > 1) return ax[dx < 0 ? 0 : 1][dy][dz];
      if (dy < 0 || dy > 1) return ay[dy < 0 ? 0 : 1][dx][dz];
      if (dz < 0 || dz > 1) return az[dz < 0 ? 0 : 1][dx][dy];
      return mid[dx][dy][dz];
    };
    const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    ok = true;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      float acc = 0.0f, ws = 0.0f;
      int valid = 0;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const float t = at(off[k][0] + (c & 1), off[k][1] + ((c >> 1) & 1), off[k][2] + (c >> 2));
        if (t != t) continue;
        const float w = axis_weight(fr[k].x, c & 1) * axis_weight(fr[k].y, (c >> 1) & 1) * axis_weight(fr[k].z, c >> 2);
        acc += w * t;
        ws += w;
        ++valid;
      }
      bool good = !(policy == KF_CORNERS_REQUIRE_ALL && valid < 8) && !(ws <= 1.0e-6f);
      const float d = good ? acc / ws : 0.0f;
      good = good && isfinite(d);
      val[k] = d;
      ok = ok && good;
    }
    return true;
  }

  // trilinear::central_normal (trilinear.hpp:243-266).  The six samples
  // are independent reads of an unchanging volume, so all are taken before
  // any is tested: the result is that of the reference's early-exit order.
  __device__ bool central_normal(f3 p, int policy, f3& out) const {
    float s6[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    bool ok = false;
    if (!central_six(p, policy, s6, ok)) {
      f3 pt[6];
      central_points(p, v.voxel_size, pt);
      ok = tsdf(pt[0], policy, s6[0]) & tsdf(pt[1], policy, s6[1]) & tsdf(pt[2], policy, s6[2]) &
           tsdf(pt[3], policy, s6[3]) & tsdf(pt[4], policy, s6[4]) & tsdf(pt[5], policy, s6[5]);
    }
    if (!ok) return false;
    const float xp = s6[0], xm = s6[1], yp = s6[2], ym = s6[3], zp = s6[4], zm = s6[5];
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
