// kf_raycast.cu - per-pixel trilinear ray march (SurfaceRaycast::render_pixel,
// raycasting.hpp:116-245; TrilinearSampler, volume_sampler.hpp:116-255;
// trilinear.hpp:85-269).
//
// One thread per pixel.  Corner gathers go through the read-only data path
// (the volume does not change during a render).  Arithmetic is the host
// expression order, so a render is bit-identical to the CPU raycast of the
// same volume and camera.
//
// Empty-space skip, exact, at two granularities.  A sample whose eight
// corners are all observed with tsdf exactly 1 is exactly 1.0 (the blend
// divides a sum by the identical sum); a sample with no observed corner is
// nullopt.  Neither needs the corner gather:
//  * 8^3 blocks whose 3x3x3 block neighbourhood is entirely free space (or
//    entirely unobserved) are crossed in one go, replaying the march's
//    ray_length additions up to the block exit;
//  * otherwise per-voxel bits (observed / exactly 1) decide single samples.
// The sample positions, and therefore the output, are those of the plain
// march.  Samples before the volume box are replayed the same way, and the
// march ends once the ray has left the box.
#include <cmath>

#include "kf_internal.h"

namespace kf {
namespace {

struct RaycastParams {
  float min_depth, max_depth, step_scale;
  int policy;
  int cell_normals;
  int seed_previous;
};

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
    if (v.grid == nullptr && bx >= 0 && by >= 0 && bz >= 0 && (bx & 7) != 7 && (by & 7) != 7 && (bz & 7) != 7 &&
        bx + 1 < static_cast<int>(v.rx) && by + 1 < static_cast<int>(v.ry) && bz + 1 < static_cast<int>(v.rz)) {
      // Dense, all eight corners in one brick: fixed offsets from the base
      // voxel, loads issued together, blended in the reference corner order.
      const Raw* b = reinterpret_cast<const Raw*>(v.voxels) +
                     storage_index(v, static_cast<uint32_t>(bx), static_cast<uint32_t>(by), static_cast<uint32_t>(bz));
      Raw r[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) r[c] = __ldg(b + ((c >> 2) * 64 + ((c >> 1) & 1) * 8 + (c & 1)));
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

  // trilinear::central_normal (trilinear.hpp:243-266)
  __device__ bool central_normal(f3 p, int policy, f3& out) const {
    const float vs = v.voxel_size;
    float plus, minus;
    if (!tsdf(make(p.x + vs, p.y + 0.0f, p.z + 0.0f), policy, plus)) return false;
    if (!tsdf(make(p.x - vs, p.y - 0.0f, p.z - 0.0f), policy, minus)) return false;
    const float gx = plus - minus;
    if (!tsdf(make(p.x + 0.0f, p.y + vs, p.z + 0.0f), policy, plus)) return false;
    if (!tsdf(make(p.x - 0.0f, p.y - vs, p.z - 0.0f), policy, minus)) return false;
    const float gy = plus - minus;
    if (!tsdf(make(p.x + 0.0f, p.y + 0.0f, p.z + vs), policy, plus)) return false;
    if (!tsdf(make(p.x - 0.0f, p.y - 0.0f, p.z - vs), policy, minus)) return false;
    const float gz = plus - minus;
    const f3 d = make(gx, gy, gz);
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

// Corner masks of the trilinear stencil with base voxel (sx, sy, sz), read
// from the per-voxel skip bits (16 words "tsdf exactly 1" + 16 words
// "observed" per brick).  Bit c of each mask is corner (c & 1, (c >> 1) & 1,
// c >> 2), the sampler's blend order.  A corner outside the volume is missing:
// neither "one" nor "observed".
__device__ __forceinline__ void stencil_masks(const uint32_t* __restrict__ bits, const VolumeDev& v, int sx, int sy,
                                              int sz, uint32_t& observed, uint32_t& one) {
  if (sx >= 0 && sy >= 0 && sz >= 0 && (sx & 7) != 7 && (sy & 7) != 7 && (sz & 7) != 7 &&
      sx + 1 < static_cast<int>(v.rx) && sy + 1 < static_cast<int>(v.ry) && sz + 1 < static_cast<int>(v.rz)) {
    const uint32_t brick = ((static_cast<uint32_t>(sz) >> 3) * v.by + (static_cast<uint32_t>(sy) >> 3)) * v.bx +
                           (static_cast<uint32_t>(sx) >> 3);
    // one z-layer of a brick is 64 bits (two words); the stencil's four
    // corners in a layer sit at bits y*8+x + {0, 1, 8, 9}
    const uint2* b = reinterpret_cast<const uint2*>(bits + static_cast<size_t>(brick) * 32u);
    const uint32_t lz = static_cast<uint32_t>(sz) & 7u;
    const uint32_t shift = (static_cast<uint32_t>(sy) & 7u) * 8u + (static_cast<uint32_t>(sx) & 7u);
    const uint2 n0 = __ldg(b + lz), n1 = __ldg(b + lz + 1u), o0 = __ldg(b + 8u + lz), o1 = __ldg(b + 9u + lz);
    auto quad = [shift](uint2 layer) {
      const uint64_t l = ((static_cast<uint64_t>(layer.y) << 32) | layer.x) >> shift;
      return static_cast<uint32_t>((l & 3u) | ((l >> 6) & 0xCu));
    };
    one = quad(n0) | (quad(n1) << 4);
    observed = quad(o0) | (quad(o1) << 4);
    return;
  }
  one = 0u;
  observed = 0u;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int x = sx + (c & 1), y = sy + ((c >> 1) & 1), z = sz + (c >> 2);
    if (x < 0 || y < 0 || z < 0 || x >= static_cast<int>(v.rx) || y >= static_cast<int>(v.ry) ||
        z >= static_cast<int>(v.rz)) {
      continue;
    }
    const uint32_t brick = ((static_cast<uint32_t>(z) >> 3) * v.by + (static_cast<uint32_t>(y) >> 3)) * v.bx +
                           (static_cast<uint32_t>(x) >> 3);
    const uint32_t idx = brick_offset(static_cast<uint32_t>(x), static_cast<uint32_t>(y), static_cast<uint32_t>(z));
    const uint32_t* w = bits + static_cast<size_t>(brick) * 32u;
    one |= ((__ldg(w + (idx >> 5)) >> (idx & 31u)) & 1u) << c;
    observed |= ((__ldg(w + 16u + (idx >> 5)) >> (idx & 31u)) & 1u) << c;
  }
}

// What the sampler returns for a stencil, decided from its corner masks
// without reading a voxel: 1 = exactly 1.0, 2 = nullopt, 0 = needs the
// gather.  With every observed corner exactly 1, the blend's numerator and
// denominator are the same sum of weights, so the value is 1.0 whenever the
// weight sum passes the sampler's 1e-6 test (the sum is recomputed here from
// the fractional position, in the sampler's order).
__device__ __forceinline__ int stencil_class(uint32_t observed, uint32_t one, int policy, f3 g) {
  if (observed == 0u) return 2;
  if (policy == KF_CORNERS_REQUIRE_ALL && observed != 0xFFu) return 2;
  if (one != observed) return 0;
  if (observed == 0xFFu) return 1;  // the eight weights sum to 1 within rounding
  const f3 gg = make(g.x - 0.5f, g.y - 0.5f, g.z - 0.5f);
  const f3 fr = gg - make(floorf(gg.x), floorf(gg.y), floorf(gg.z));
  float ws = 0.0f;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    if (!((observed >> c) & 1u)) continue;
    const float w = ((c & 1) ? fr.x : 1.0f - fr.x) * (((c >> 1) & 1) ? fr.y : 1.0f - fr.y) *
                    ((c >> 2) ? fr.z : 1.0f - fr.z);
    ws += w;
  }
  return ws <= 1.0e-6f ? 2 : 1;
}

// Ray parameter where the ray leaves block (bxi, byi, bzi).  Approximate:
// samples within rounding distance of the face still lie in the block's
// one-block safety neighbourhood.
__device__ __forceinline__ float block_exit(const VolumeDev& v, f3 o, f3 inv_dir, uint32_t bxi, uint32_t byi,
                                            uint32_t bzi) {
  const float edge = 8.0f * v.voxel_size;
  const f3 lo = v.origin + make(static_cast<float>(bxi), static_cast<float>(byi), static_cast<float>(bzi)) * edge;
  const float tx = ((inv_dir.x >= 0.0f ? lo.x + edge : lo.x) - o.x) * inv_dir.x;
  const float ty = ((inv_dir.y >= 0.0f ? lo.y + edge : lo.y) - o.y) * inv_dir.y;
  const float tz = ((inv_dir.z >= 0.0f ? lo.z + edge : lo.z) - o.z) * inv_dir.z;
  return fminf(tx, fminf(ty, tz));
}

// Ray parameters where the ray enters and leaves the volume box, widened by
// two voxels (FP64: the samples' own rounding stays far inside the margin).
__device__ __forceinline__ void box_range(const VolumeDev& v, f3 o, f3 d, float& t_in, float& t_out) {
  double lo = -1e300, hi = 1e300;
  const double org[3] = {o.x, o.y, o.z}, dir[3] = {d.x, d.y, d.z};
  const double bmin[3] = {v.origin.x, v.origin.y, v.origin.z};
  const double ext[3] = {static_cast<double>(v.rx) * v.voxel_size, static_cast<double>(v.ry) * v.voxel_size,
                         static_cast<double>(v.rz) * v.voxel_size};
  for (int a = 0; a < 3; ++a) {
    if (dir[a] == 0.0) {
      if (org[a] < bmin[a] || org[a] > bmin[a] + ext[a]) {
        lo = 1e300;
        hi = -1e300;
      }
      continue;
    }
    const double t0 = (bmin[a] - org[a]) / dir[a];
    const double t1 = (bmin[a] + ext[a] - org[a]) / dir[a];
    lo = fmax(lo, fmin(t0, t1));
    hi = fmin(hi, fmax(t0, t1));
  }
  const double margin = 2.0 * v.voxel_size;
  t_in = static_cast<float>(lo - margin);
  t_out = static_cast<float>(hi + margin);
  if (!(lo <= hi)) {
    t_in = 1e30f;
    t_out = -1e30f;
  }
}

template <int Kind, bool Color>
__global__ void __launch_bounds__(64)
    raycast_kernel(VolumeDev v, const uint32_t* __restrict__ free_safe, const uint32_t* __restrict__ empty_safe,
                   const uint32_t* __restrict__ voxel_bits,
                   RaycastParams rp, Intr k, uint32_t width,
                   uint32_t height, Rigid pose, const IcpState* __restrict__ state, float* __restrict__ points,
                   float* __restrict__ normals, uint32_t* __restrict__ colors) {
  if (state != nullptr) {
    if (state->failed) return;
    const float* c = state->camera;
    pose = Rigid{{c[0], c[1], c[2]}, {c[3], c[4], c[5]}, {c[6], c[7], c[8]}, {c[9], c[10], c[11]}};
  }
  const uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t row = blockIdx.y * blockDim.y + threadIdx.y;
  if (col >= width || row >= height) return;
  const size_t pix = static_cast<size_t>(row) * width + col;
  const Sampler<Kind> s{v};

  float seed = rp.min_depth;
  if (rp.seed_previous) {
    const f3 previous = load3(points + pix * 3);
    if (finite3(previous) && dot(previous, previous) > 0.0f) {
      const float previous_depth = norm(previous - pose.t);
      const float truncated = previous_depth - (2.0f * v.truncation);
      seed = rp.min_depth < truncated ? truncated : rp.min_depth;
    }
  }
  f3 out_point = nan3(), out_normal = nan3();
  uint32_t out_color = 0;

  const f3 translated = back_project(k, static_cast<float>(col), static_cast<float>(row), 1.0f);
  const f3 direction = rotate(pose, translated);
  const float dn = norm(direction);
  if (dn > 0.0f) {
    const f3 dir = direction / dn;
    // find_zero_crossing (raycasting.hpp:165-211)
    const float base_step = v.voxel_size * rp.step_scale;
    // The step taken after a sample of exactly 1.0 (observed free space).
    const float precomp_one = 1.0f * v.truncation * rp.step_scale;
    const float free_step = base_step < precomp_one ? precomp_one : base_step;
    bool have_prev = false;
    float prev_tsdf = 0.0f;
    f3 prev_point = make(0.0f, 0.0f, 0.0f);
    float ray_length = seed;
    bool found = false;
    f3 surface = make(0.0f, 0.0f, 0.0f);
    // Samples outside the volume box are nullopt: replay the base steps up
    // to the box, and stop once the ray has left it (a box is convex).
    float t_in, t_out;
    box_range(v, pose.t, dir, t_in, t_out);
    const f3 inv_dir = make(dir.x != 0.0f ? 1.0f / dir.x : 1e30f, dir.y != 0.0f ? 1.0f / dir.y : 1e30f,
                            dir.z != 0.0f ? 1.0f / dir.z : 1e30f);
    while (ray_length < t_in && ray_length <= rp.max_depth) ray_length += base_step;
    while (ray_length <= rp.max_depth) {
      if (ray_length > t_out) break;
      const f3 point = pose.t + (dir * ray_length);
      if (voxel_bits != nullptr) {
        // Exact skip (see the file comment): decide the sample from the
        // per-voxel bits of its stencil, and cross whole safe blocks.
        const f3 g = (point - v.origin) * v.inv_voxel_size;
        if (!(g.x >= 0.0f && g.y >= 0.0f && g.z >= 0.0f && g.x < static_cast<float>(v.rx) &&
              g.y < static_cast<float>(v.ry) && g.z < static_cast<float>(v.rz))) {
          have_prev = false;  // outside the grid: nullopt
          ray_length += base_step;
          continue;
        }
        const int sx = static_cast<int>(floorf(g.x - 0.5f)), sy = static_cast<int>(floorf(g.y - 0.5f)),
                  sz = static_cast<int>(floorf(g.z - 0.5f));
        uint32_t observed, one;
        stencil_masks(voxel_bits, v, sx, sy, sz, observed, one);
        const int cls = stencil_class(observed, one, rp.policy, g);
        if (cls != 0) {
          const uint32_t bxi = static_cast<uint32_t>(g.x) >> 3, byi = static_cast<uint32_t>(g.y) >> 3,
                         bzi = static_cast<uint32_t>(g.z) >> 3;
          const uint32_t block = (bzi * v.by + byi) * v.bx + bxi;
          const uint32_t bbit = 1u << (block & 31u);
          const bool block_safe = (__ldg((cls == 1 ? free_safe : empty_safe) + (block >> 5)) & bbit) != 0u;
          const float t_exit = block_safe ? block_exit(v, pose.t, inv_dir, bxi, byi, bzi) : 0.0f;
          if (cls == 1) {
            // Exactly 1.0: leaving a surface from behind ends the march at
            // the first such sample; after it every step is free_step.
            if (have_prev && prev_tsdf < 0.0f) break;
            float last = ray_length;
            do {
              last = ray_length;
              ray_length += free_step;
            } while (ray_length < t_exit && ray_length <= rp.max_depth);
            have_prev = true;
            prev_tsdf = 1.0f;
            prev_point = last == ray_length ? point : pose.t + (dir * last);
          } else {
            have_prev = false;  // nullopt
            do {
              ray_length += base_step;
            } while (ray_length < t_exit && ray_length <= rp.max_depth);
          }
          continue;
        }
      }
      float tsdf;
      if (!s.tsdf(point, rp.policy, tsdf)) {
        have_prev = false;
        ray_length += base_step;
        continue;
      }
      if (have_prev && prev_tsdf > 0.0f && tsdf <= 0.0f) {
        const float gap = prev_tsdf - tsdf;
        const float alpha = gap != 0.0f ? prev_tsdf / gap : 0.0f;
        surface = prev_point + ((point - prev_point) * alpha);
        found = true;
        break;
      }
      if (have_prev && prev_tsdf < 0.0f && tsdf > 0.0f) break;
      have_prev = true;
      prev_tsdf = tsdf;
      prev_point = point;
      const float precomp = tsdf * v.truncation * rp.step_scale;
      const float step = base_step < precomp ? precomp : base_step;
      ray_length += tsdf > 0.0f ? step : base_step;
    }
    if (found) {
      // write_surface_sample (raycasting.hpp:215-245)
      f3 n;
      const bool has_normal = rp.cell_normals ? s.cell_normal(surface, n) : s.central_normal(surface, rp.policy, n);
      if (has_normal) {
        out_point = surface;
        out_normal = n;
        if constexpr (Color) {
          f3 c;
          if (s.color(surface, c)) out_color = pixel_from_color(c);
        } else {
          const f3 view = normalized(pose.t - surface);
          const float d = dot(n, view);
          const float intensity = 255.0f * (0.0f < d ? d : 0.0f);
          out_color = pixel_from_color(make(intensity, intensity, intensity));
        }
      }
    }
  }
  store3(points + pix * 3, out_point);
  store3(normals + pix * 3, out_normal);
  colors[pix] = out_color;
}

template <int Kind, bool Color>
void launch_typed(const Pipeline& p, const kf_raycast_camera& cam, float* points, float* normals,
                  uint32_t* colors, const IcpState* state, cudaStream_t s) {
  RaycastParams rp;
  rp.min_depth = p.config.raycast.min_depth;
  rp.max_depth = p.config.raycast.max_depth;
  rp.step_scale = p.config.raycast.step_scale;
  rp.policy = p.config.raycast.corner_policy;
  rp.cell_normals = p.config.raycast.cell_gradient_normals;
  rp.seed_previous = p.config.raycast.seed_from_previous;
  const uint32_t* free_safe = p.safe_blocks.count ? p.safe_blocks.ptr : nullptr;
  const uint32_t* empty_safe = p.safe_blocks.count ? p.empty_safe.ptr : nullptr;
  const dim3 block(8, 8);
  const dim3 grid(ceil_div(cam.width, 8), ceil_div(cam.height, 8));
  const uint32_t* voxel_bits = p.safe_blocks.count && p.view.grid == nullptr ? p.voxel_bits.ptr : nullptr;
  raycast_kernel<Kind, Color><<<grid, block, 0, s>>>(p.view, free_safe, empty_safe, voxel_bits, rp, intr_from(cam.intrinsics), cam.width,
                                                     cam.height, rigid_from(cam.camera_to_world), state, points,
                                                     normals, colors);
  check(cudaGetLastError(), "raycast_kernel launch");
}

}  // namespace

void launch_raycast(const Pipeline& p, const kf_raycast_camera& cam, float* points, float* normals,
                    uint32_t* colors, const IcpState* state, cudaStream_t s) {
  const bool color = p.config.color == KF_COLOR_FLOAT;
  switch (p.config.voxel) {
    case KF_VOXEL_QUANTIZED:
      color ? launch_typed<KF_VOXEL_QUANTIZED, true>(p, cam, points, normals, colors, state, s)
            : launch_typed<KF_VOXEL_QUANTIZED, false>(p, cam, points, normals, colors, state, s);
      break;
    case KF_VOXEL_BF16:
      color ? launch_typed<KF_VOXEL_BF16, true>(p, cam, points, normals, colors, state, s)
            : launch_typed<KF_VOXEL_BF16, false>(p, cam, points, normals, colors, state, s);
      break;
    default:
      color ? launch_typed<KF_VOXEL_FLOAT, true>(p, cam, points, normals, colors, state, s)
            : launch_typed<KF_VOXEL_FLOAT, false>(p, cam, points, normals, colors, state, s);
      break;
  }
}

}  // namespace kf
