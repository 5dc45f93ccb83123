// kf_raycast.cu - per-pixel trilinear ray march (SurfaceRaycast::render_pixel,
// raycasting.hpp:116-245; TrilinearSampler, volume_sampler.hpp:116-255;
// trilinear.hpp:85-269).
//
// One thread per pixel.  Corner gathers go through the read-only data path
// (the volume does not change during a render).  Arithmetic is the host
// expression order, so a render is bit-identical to the CPU raycast of the
// same volume and camera.
//
// Empty-space skip, exact.  A sample whose eight corners are all observed
// with tsdf exactly 1 is exactly 1.0 (the blend divides a sum by the
// identical sum), and so is one whose observed corners are all exactly 1
// when their weights pass the sampler's 1e-6 test; a sample with no observed
// corner (or, under REQUIRE_ALL, a missing one) is nullopt.  None of these
// needs the corner gather.  The integration pass keeps, per stencil base
// voxel, bits that decide this class where the corners alone settle it, and
// per 8^3 brick whether every stencil based in it is nullopt or exactly 1.0:
//  * a sample in such a brick and of that class crosses the brick in one go,
//    replaying the march's ray_length additions while the samples' bases
//    stay in the brick;
//  * otherwise the per-base bits decide single samples, and the per-voxel
//    bits settle the partially observed ones.
// The sample positions, and therefore the output, are those of the plain
// march.  Samples before the volume box are replayed the same way, and the
// march ends once the ray has left the box.
#include <cmath>

#include "kf_internal.h"
#include "kf_sampler.cuh"

namespace kf {
namespace {

// Rays left in a warp at or below which they march cooperatively, in renders
// that start with lanes to spare (fewer rays than lanes per warp).  Where
// every lane starts with a ray the rays march alone to the end: there the
// cooperative rounds' extra shuffles cost more than their speculation saves
// (640x480 render 0.405 -> 0.388 ms without them, maps identical).
constexpr int kCoopLanes = 8;

struct RaycastParams {
  float min_depth, max_depth, step_scale;
  int policy;
  int cell_normals;
  int seed_previous;
  uint32_t rays_per_warp;  // 32: one lane per ray, 2D CTA tile; 16 or 8: warp tiles below
  int coop_rays;           // kCoopLanes, or 0 when rays_per_warp is 32
};

// Pixel tile of one warp that holds `rays` rays (lanes 0..rays-1; the other
// lanes start done and lend themselves to the live rays' cooperative rounds):
// 16 rays -> 4 x 4 pixels, 8 -> 4 x 2, 4 -> 4 x 1, 2 -> 2 x 1, 1 -> 1 x 1.
// A CTA stacks its warps in y.
__device__ __forceinline__ void warp_tile_pixel(uint32_t rays, uint32_t& col, uint32_t& row, bool& has_ray) {
  const uint32_t tid = threadIdx.y * blockDim.x + threadIdx.x;
  const uint32_t warp = tid >> 5, lane = tid & 31u;
  const uint32_t warps = (blockDim.x * blockDim.y) >> 5;
  const uint32_t tw = rays < 4u ? rays : 4u, th = rays / tw;
  col = blockIdx.x * tw + (lane % tw);
  row = (blockIdx.y * warps + warp) * th + (lane / tw) % th;
  has_ray = lane < rays;
}

// Corner masks of the trilinear stencil with base voxel (sx, sy, sz), read
// from the per-voxel bits (per brick layer z, 16 bytes: 64 bits "tsdf
// exactly 1", 64 bits "observed", bit y*8+x).  Bit c of each mask is corner
// (c & 1, (c >> 1) & 1, c >> 2), the sampler's blend order.  A corner outside
// the volume is missing: neither "one" nor "observed".
__device__ __forceinline__ void stencil_masks(const uint32_t* __restrict__ bits, const VolumeDev& v, int sx, int sy,
                                              int sz, uint32_t& observed, uint32_t& one) {
  if (sx >= 0 && sy >= 0 && sz >= 0 && (sx & 7) != 7 && (sy & 7) != 7 && (sz & 7) != 7 &&
      sx + 1 < static_cast<int>(v.rx) && sy + 1 < static_cast<int>(v.ry) && sz + 1 < static_cast<int>(v.rz)) {
    const uint32_t brick = ((static_cast<uint32_t>(sz) >> 3) * v.by + (static_cast<uint32_t>(sy) >> 3)) * v.bx +
                           (static_cast<uint32_t>(sx) >> 3);
    // the stencil's four corners in a layer sit at bits y*8+x + {0, 1, 8, 9}
    const uint4* b = reinterpret_cast<const uint4*>(bits) + static_cast<size_t>(brick) * 8u;
    const uint32_t lz = static_cast<uint32_t>(sz) & 7u;
    const uint32_t shift = (static_cast<uint32_t>(sy) & 7u) * 8u + (static_cast<uint32_t>(sx) & 7u);
    const uint4 l0 = __ldg(b + lz), l1 = __ldg(b + lz + 1u);
    auto quad = [shift](uint32_t lo, uint32_t hi) {
      const uint64_t l = ((static_cast<uint64_t>(hi) << 32) | lo) >> shift;
      return static_cast<uint32_t>((l & 3u) | ((l >> 6) & 0xCu));
    };
    one = quad(l0.x, l0.y) | (quad(l1.x, l1.y) << 4);
    observed = quad(l0.z, l0.w) | (quad(l1.z, l1.w) << 4);
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
    const size_t word = static_cast<size_t>(brick) * 32u + (static_cast<uint32_t>(z) & 7u) * 4u +
                          ((static_cast<uint32_t>(y) >> 2) & 1u);
    const uint32_t bit = (static_cast<uint32_t>(y) & 3u) * 8u + (static_cast<uint32_t>(x) & 7u);
    one |= ((__ldg(bits + word) >> bit) & 1u) << c;
    observed |= ((__ldg(bits + word + 2u) >> bit) & 1u) << c;
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

// The grid position of a sample is inside the volume (TrilinearSampler's
// bounds test; outside, the sample is nullopt).
__device__ __forceinline__ bool in_grid(const VolumeDev& v, f3 g) {
  return g.x >= 0.0f && g.y >= 0.0f && g.z >= 0.0f && g.x < static_cast<float>(v.rx) &&
         g.y < static_cast<float>(v.ry) && g.z < static_cast<float>(v.rz);
}

// Record of the per-base stencil bits holding the stencil of grid position
// g, the bit of that stencil in the record's 64-bit halves, and the brick
// of the base voxel.  Returns false when the base voxel lies below the
// volume (g < 0.5 on an axis); there is no record then.
struct Slot {
  uint32_t record, bit, bx, by, bz;
};
__device__ __forceinline__ bool stencil_slot(const VolumeDev& v, f3 g, Slot& s) {
  const int sx = static_cast<int>(floorf(g.x - 0.5f)), sy = static_cast<int>(floorf(g.y - 0.5f)),
            sz = static_cast<int>(floorf(g.z - 0.5f));
  if (sx < 0 || sy < 0 || sz < 0) return false;
  const uint32_t ux = static_cast<uint32_t>(sx), uy = static_cast<uint32_t>(sy), uz = static_cast<uint32_t>(sz);
  s.bx = ux >> 3;
  s.by = uy >> 3;
  s.bz = uz >> 3;
  s.record = ((s.bz * v.by + s.by) * v.bx + s.bx) * 8u + (uz & 7u);
  s.bit = (uy & 7u) * 8u + (ux & 7u);
  return true;
}

// Class of a stencil from its record: 1 = exactly 1.0, 2 = nullopt, 0 = not
// decided by the stencil bits, the corner weights may decide (every observed
// corner is exactly 1), 3 = not decided, only the gather decides (an observed
// corner holds another value).
__device__ __forceinline__ int record_class(uint4 r, uint32_t bit) {
  const uint32_t undecided = bit < 32u ? r.x >> bit : r.y >> (bit - 32u);
  const uint32_t one = bit < 32u ? r.z >> bit : r.w >> (bit - 32u);
  if (undecided & 1u) return (one & 1u) ? 0 : 3;
  return (one & 1u) ? 1 : 2;
}

// Ray parameter up to which the samples' stencil bases stay in a box of
// bricks: the box of `size` voxels per axis whose lowest voxel is (lox, loy,
// loz); a sample's grid position keeps its base in the box while it stays in
// the box shifted by half a voxel, [lo + 0.5, lo + size + 0.5) per axis,
// clipped to the volume when `clip` is set.  The ray is taken as g0 + gdir *
// t in grid units; `margin` (voxels) shrinks the box by more than the
// rounding that separates this line from the march's own sample positions,
// so every sample before the returned parameter has its base in the box.
__device__ __forceinline__ float box_exit(const VolumeDev& v, f3 g0, f3 inv_gdir, uint32_t lox, uint32_t loy,
                                          uint32_t loz, uint32_t size, bool clip, float margin) {
  auto axis = [margin, clip, size](float g, float inv, uint32_t lo_voxel, uint32_t extent) {
    const float lo = static_cast<float>(lo_voxel) + 0.5f + margin;
    float hi = static_cast<float>(lo_voxel + size) + 0.5f - margin;
    if (clip) hi = fminf(hi, static_cast<float>(extent) - margin);
    return ((inv >= 0.0f ? hi : lo) - g) * inv;
  };
  return fminf(axis(g0.x, inv_gdir.x, lox, v.rx), fminf(axis(g0.y, inv_gdir.y, loy, v.ry),
                                                          axis(g0.z, inv_gdir.z, loz, v.rz)));
}

// A march sample: nullopt, a value, or past the march's end.
enum : int { kNull = 0, kValue = 1, kEnd = 2 };
// What a sample does to the march: nothing, a zero crossing, the end.
enum : int { kNone = 0, kFound = 1, kStop = 2 };

// The sample at `point` (find_zero_crossing's volume.tsdf, raycasting.hpp:
// 176-205): kNull or kValue with its value in `tsdf`.  With the skip
// structures, a sample the stencil bits decide needs no corner gather, and
// `jump` gets its brick (bit 31 | x | y << 10 | z << 20) when every stencil
// of that brick has the sample's class, with `radius` the radius in bricks
// of the cube around it whose bricks all have that class.
template <int Kind>
__device__ __forceinline__ int march_sample(const Sampler<Kind>& s, const VolumeDev& v,
                                            const uint32_t* __restrict__ voxel_bits,
                                            const uint4* __restrict__ stencil_bits,
                                            const uint8_t* __restrict__ brick_class,
                                            const uint8_t* __restrict__ brick_radius,
                                            const uint8_t* __restrict__ null_bricks, int policy, f3 point,
                                            float& tsdf, uint32_t& jump, uint32_t& radius) {
  jump = 0u;
  radius = 0u;
  if (null_bricks != nullptr) {
    // sparse storage: a stencil based in a block whose 2x2x2 block
    // neighbourhood is unallocated has no observed corner
    const f3 g = (point - v.origin) * v.inv_voxel_size;
    if (!in_grid(v, g)) return kNull;
    const int sx = static_cast<int>(floorf(g.x - 0.5f)), sy = static_cast<int>(floorf(g.y - 0.5f)),
              sz = static_cast<int>(floorf(g.z - 0.5f));
    if (sx >= 0 && sy >= 0 && sz >= 0) {
      const uint32_t bx = static_cast<uint32_t>(sx) >> 3, by = static_cast<uint32_t>(sy) >> 3,
                     bz = static_cast<uint32_t>(sz) >> 3;
      if (__ldg(null_bricks + (static_cast<size_t>(bz) * v.by + by) * v.bx + bx)) {
        if (bx < 1024u && by < 1024u && bz < 1024u) jump = 0x80000000u | bx | (by << 10) | (bz << 20);
        return kNull;
      }
    }
    return s.tsdf(point, policy, tsdf) ? kValue : kNull;
  }
  if (voxel_bits != nullptr) {
    const f3 g = (point - v.origin) * v.inv_voxel_size;
    if (!in_grid(v, g)) return kNull;
    Slot slot;
    int cls = 0, summary = 0;
    uint32_t cube = 0u;
    if (stencil_slot(v, g, slot)) {
      const uint4 rec = __ldg(stencil_bits + slot.record);
      summary = __ldg(brick_class + (slot.record >> 3));
      if (brick_radius != nullptr) cube = __ldg(brick_radius + (slot.record >> 3));
      cls = record_class(rec, slot.bit);
    }
    if (cls == 0) {
      uint32_t observed, one;
      stencil_masks(voxel_bits, v, static_cast<int>(floorf(g.x - 0.5f)), static_cast<int>(floorf(g.y - 0.5f)),
                    static_cast<int>(floorf(g.z - 0.5f)), observed, one);
      cls = stencil_class(observed, one, policy, g);
    } else if (cls == 3) {
      cls = 0;  // the masks would only confirm it: straight to the gather
    }
    if (cls != 0) {
      if (summary == (cls == 1 ? 2 : 1) && slot.bx < 1024u && slot.by < 1024u && slot.bz < 1024u) {
        jump = 0x80000000u | slot.bx | (slot.by << 10) | (slot.bz << 20);
        radius = cube;
      }
      if (cls == 2) return kNull;
      tsdf = 1.0f;
      return kValue;
    }
  }
  return s.tsdf(point, policy, tsdf) ? kValue : kNull;
}

// find_zero_crossing's tests of a sample against the previous one
// (raycasting.hpp:186-203): a crossing from positive to non-positive gives
// the interpolated surface; a rise from negative to positive ends the march.
__device__ __forceinline__ int sample_event(int kind, float tsdf, f3 point, bool p_have, float p_tsdf, f3 p_point,
                                            f3& surf) {
  if (kind == kEnd) return kStop;
  if (kind == kValue && p_have) {
    if (p_tsdf > 0.0f && tsdf <= 0.0f) {
      const float gap = p_tsdf - tsdf;
      const float alpha = gap != 0.0f ? p_tsdf / gap : 0.0f;
      surf = p_point + ((point - p_point) * alpha);
      return kFound;
    }
    if (p_tsdf < 0.0f && tsdf > 0.0f) return kStop;
  }
  return kNone;
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

template <int Kind>
__global__ void __launch_bounds__(64)
    raycast_kernel(VolumeDev v, const uint32_t* __restrict__ voxel_bits, const uint4* __restrict__ stencil_bits,
                   const uint8_t* __restrict__ brick_class, const uint8_t* __restrict__ brick_radius,
                   const uint8_t* __restrict__ null_bricks,
                   RaycastParams rp, Intr k, uint32_t width,
                   uint32_t height, Rigid pose, const IcpState* __restrict__ state, float* __restrict__ points) {
  if (state != nullptr) {
    if (state->failed) return;
    const float* c = state->camera;
    pose = Rigid{{c[0], c[1], c[2]}, {c[3], c[4], c[5]}, {c[6], c[7], c[8]}, {c[9], c[10], c[11]}};
  }
  // Every lane of a warp takes part in the march's rounds (lanes without a
  // ray are done from the start), so that the warp reconverges at each
  // sample instead of running its lanes' divergent marches one after
  // another.
  uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t row = blockIdx.y * blockDim.y + threadIdx.y;
  bool has_ray = true;
  if (rp.rays_per_warp < 32u) warp_tile_pixel(rp.rays_per_warp, col, row, has_ray);
  const bool in_image = has_ray && col < width && row < height;
  const size_t pix = in_image ? static_cast<size_t>(row) * width + col : 0;
  const Sampler<Kind> s{v};

  float seed = rp.min_depth;
  if (rp.seed_previous && in_image) {
    const f3 previous = load3(points + pix * 3);
    if (finite3(previous) && dot(previous, previous) > 0.0f) {
      const float previous_depth = norm(previous - pose.t);
      const float truncated = previous_depth - (2.0f * v.truncation);
      seed = rp.min_depth < truncated ? truncated : rp.min_depth;
    }
  }

  const f3 translated = back_project(k, static_cast<float>(col), static_cast<float>(row), 1.0f);
  const f3 direction = rotate(pose, translated);
  const float dn = norm(direction);
  bool done = !(in_image && dn > 0.0f);
  const f3 dir = done ? make(0.0f, 0.0f, 1.0f) : direction / dn;
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
  // The ray in grid units for brick exits, and the margin that covers the
  // rounding of the samples' own positions (grows with the coordinates).
  const f3 g0 = (pose.t - v.origin) * v.inv_voxel_size;
  const f3 gdir = dir * v.inv_voxel_size;
  const f3 inv_gdir = make(gdir.x != 0.0f ? 1.0f / gdir.x : 1e30f, gdir.y != 0.0f ? 1.0f / gdir.y : 1e30f,
                           gdir.z != 0.0f ? 1.0f / gdir.z : 1e30f);
  const float reach = fmaxf(fabsf(g0.x), fmaxf(fabsf(g0.y), fabsf(g0.z))) +
                      fmaxf(fabsf(gdir.x), fmaxf(fabsf(gdir.y), fabsf(gdir.z))) * fmaxf(fabsf(t_out), 1.0f) +
                      static_cast<float>(max(v.rx, max(v.ry, v.rz)));
  const float margin = (1.0f / 64.0f) + reach * 4.0e-6f;
  if (!done) {
    while (ray_length < t_in && ray_length <= rp.max_depth) ray_length += base_step;
  }
  float spec = free_step;  // the step the ray's last sample implies
  // The step after a sample (find_zero_crossing's advance, raycasting.hpp:
  // 204-209): nullopt and non-positive values take the base step.
  auto step_after = [&](int kind, float tsdf) {
    if (kind == kValue && tsdf > 0.0f) {
      const float precomp = tsdf * v.truncation * rp.step_scale;
      return base_step < precomp ? precomp : base_step;
    }
    return base_step;
  };
  // Take a sample (known kind and event) into the march state; a decided
  // sample whose brick holds only its class also takes every following
  // sample up to the exit of the cube of bricks of that class around it.
  auto apply = [&](int event, int kind, float tsdf, f3 point, float r, uint32_t jump, uint32_t radius, f3 surf) {
    if (event == kFound) {
      found = true;
      surface = surf;
      done = true;
      return;
    }
    if (event == kStop) {
      done = true;
      return;
    }
    const float step = step_after(kind, tsdf);
    float last = r, next = r + step;
    if (jump != 0u) {
      const uint32_t bxi = jump & 1023u, byi = (jump >> 10) & 1023u, bzi = (jump >> 20) & 1023u;
      const float t_exit = box_exit(v, g0, inv_gdir, 8u * (bxi - radius), 8u * (byi - radius), 8u * (bzi - radius),
                                    8u * (2u * radius + 1u), kind == kValue, margin);
      while (next < t_exit && next <= rp.max_depth && !(next > t_out)) {
        last = next;
        next += step;
      }
    }
    have_prev = kind == kValue;
    prev_tsdf = tsdf;
    prev_point = last == r ? point : pose.t + (dir * last);
    ray_length = next;
    spec = step;
  };

  const unsigned lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31u;
  unsigned live;
  while ((live = __ballot_sync(0xFFFFFFFFu, !done)) != 0u) {
    const int n = __popc(live);
    if (n > rp.coop_rays) {
      // every live lane takes the next sample of its own ray
      if (!done) {
        const float r = ray_length;
        int kind = kEnd;
        float tsdf = 0.0f;
        uint32_t jump = 0u, radius = 0u;
        f3 point = make(0.0f, 0.0f, 0.0f);
        if (r <= rp.max_depth && !(r > t_out)) {
          point = pose.t + (dir * r);
          kind = march_sample(s, v, voxel_bits, stencil_bits, brick_class, brick_radius, null_bricks, rp.policy,
                              point, tsdf, jump, radius);
        }
        f3 surf = make(0.0f, 0.0f, 0.0f);
        const int event = sample_event(kind, tsdf, point, have_prev, prev_tsdf, prev_point, surf);
        apply(event, kind, tsdf, point, r, jump, radius, surf);
      }
      continue;
    }
    // Few rays left: each live ray gets a segment of G lanes, lane `off` of
    // which takes the sample `off` steps ahead, assuming every step until
    // then equals the ray's last one.  The samples up to the first one that
    // ends the march or takes another step are exactly the march's next
    // samples; the ray takes them all in this round.
    const int lg = n > 8 ? 1 : (n > 4 ? 2 : (n > 2 ? 3 : (n > 1 ? 4 : 5)));
    const unsigned G = 1u << lg;
    const unsigned seg = lane >> lg, off = lane & (G - 1u);
    const bool active = seg < static_cast<unsigned>(n);
    unsigned owner = lane;
    if (active) {
      unsigned m = live;
      for (unsigned i = 0; i < seg; ++i) m &= m - 1u;
      owner = static_cast<unsigned>(__ffs(m) - 1);
    }
    const float o_r = __shfl_sync(0xFFFFFFFFu, ray_length, owner);
    const float o_s = __shfl_sync(0xFFFFFFFFu, spec, owner);
    const float o_tout = __shfl_sync(0xFFFFFFFFu, t_out, owner);
    const f3 o_dir = make(__shfl_sync(0xFFFFFFFFu, dir.x, owner), __shfl_sync(0xFFFFFFFFu, dir.y, owner),
                          __shfl_sync(0xFFFFFFFFu, dir.z, owner));
    const bool o_hp = __shfl_sync(0xFFFFFFFFu, have_prev ? 1 : 0, owner) != 0;
    const float o_pt = __shfl_sync(0xFFFFFFFFu, prev_tsdf, owner);
    const f3 o_pp = make(__shfl_sync(0xFFFFFFFFu, prev_point.x, owner),
                         __shfl_sync(0xFFFFFFFFu, prev_point.y, owner),
                         __shfl_sync(0xFFFFFFFFu, prev_point.z, owner));
    float r = o_r;
    for (unsigned i = 0; i < off; ++i) r += o_s;
    int kind = kEnd;
    float tsdf = 0.0f;
    uint32_t jump = 0u, radius = 0u;
    f3 point = make(0.0f, 0.0f, 0.0f);
    if (active && r <= rp.max_depth && !(r > o_tout)) {
      point = pose.t + (o_dir * r);
      kind = march_sample(s, v, voxel_bits, stencil_bits, brick_class, brick_radius, null_bricks, rp.policy, point,
                          tsdf, jump, radius);
    }
    // the state before this sample: the previous lane's sample, or the ray's
    const int up_kind = __shfl_up_sync(0xFFFFFFFFu, kind, 1);
    const float up_tsdf = __shfl_up_sync(0xFFFFFFFFu, tsdf, 1);
    const f3 up_point = make(__shfl_up_sync(0xFFFFFFFFu, point.x, 1), __shfl_up_sync(0xFFFFFFFFu, point.y, 1),
                             __shfl_up_sync(0xFFFFFFFFu, point.z, 1));
    f3 surf = make(0.0f, 0.0f, 0.0f);
    const int event = off == 0 ? sample_event(kind, tsdf, point, o_hp, o_pt, o_pp, surf)
                               : sample_event(kind, tsdf, point, up_kind == kValue, up_tsdf, up_point, surf);
    const bool stop = !active || event != kNone || !(step_after(kind, tsdf) == o_s);
    const unsigned stops = __ballot_sync(0xFFFFFFFFu, stop);
    // each live lane reads the last sample its segment took
    unsigned src = lane;
    if (!done) {
      const unsigned base = static_cast<unsigned>(__popc(live & ((1u << lane) - 1u))) << lg;
      const unsigned mine = (stops >> base) & (G == 32u ? 0xFFFFFFFFu : ((1u << G) - 1u));
      src = base + (mine != 0u ? static_cast<unsigned>(__ffs(mine) - 1) : G - 1u);
    }
    const int m_event = __shfl_sync(0xFFFFFFFFu, event, src);
    const int m_kind = __shfl_sync(0xFFFFFFFFu, kind, src);
    const float m_r = __shfl_sync(0xFFFFFFFFu, r, src);
    const float m_tsdf = __shfl_sync(0xFFFFFFFFu, tsdf, src);
    const uint32_t m_jump = __shfl_sync(0xFFFFFFFFu, jump, src);
    const uint32_t m_radius = __shfl_sync(0xFFFFFFFFu, radius, src);
    const f3 m_point = make(__shfl_sync(0xFFFFFFFFu, point.x, src), __shfl_sync(0xFFFFFFFFu, point.y, src),
                            __shfl_sync(0xFFFFFFFFu, point.z, src));
    const f3 m_surf = make(__shfl_sync(0xFFFFFFFFu, surf.x, src), __shfl_sync(0xFFFFFFFFu, surf.y, src),
                           __shfl_sync(0xFFFFFFFFu, surf.z, src));
    if (!done) apply(m_event, m_kind, m_tsdf, m_point, m_r, m_jump, m_radius, m_surf);
  }
  if (in_image) store3(points + pix * 3, found ? surface : nan3());
}

// write_surface_sample (raycasting.hpp:215-245) for every pixel whose march
// found a zero crossing (its point is finite): the normal, then the colour
// or the shading; without a normal the pixel has no surface.
template <int Kind, bool Color>
__global__ void __launch_bounds__(128, 6)
    surface_kernel(VolumeDev v, RaycastParams rp, uint32_t width, uint32_t height, Rigid pose,
                   const IcpState* __restrict__ state, float* __restrict__ points, float* __restrict__ normals,
                   uint32_t* __restrict__ colors) {
  if (state != nullptr) {
    if (state->failed) return;
    if constexpr (!Color) {  // the shading needs the camera position
      const float* c = state->camera;
      pose = Rigid{{c[0], c[1], c[2]}, {c[3], c[4], c[5]}, {c[6], c[7], c[8]}, {c[9], c[10], c[11]}};
    }
  }
  const uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t row = blockIdx.y * blockDim.y + threadIdx.y;
  if (col >= width || row >= height) return;
  const size_t pix = static_cast<size_t>(row) * width + col;
  const Sampler<Kind> s{v};
  const f3 surface = load3(points + pix * 3);
  f3 out_point = nan3(), out_normal = nan3();
  uint32_t out_color = 0;
  if (finite3(surface)) {
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
  store3(points + pix * 3, out_point);
  store3(normals + pix * 3, out_normal);
  colors[pix] = out_color;
}

// ---- band march (BandSkip, empty_space_skip.hpp:19-153, 196-287) ----------
// The reference's approximate skip: the ray jumps to the entry of the next
// block of the dilated band bitmap (blocks holding an observed voxel with
// tsdf < 1 - 1/64, grown by one block).  Its output differs from the plain
// march by design; these kernels reproduce the reference's band march
// operation for operation, so they match the oracle's band march bit for bit.
struct BandDev {
  const uint32_t* words;  // dilated bits, z-major: ((x * by) + y) * bz + z
  uint32_t bx, by, bz;
};

constexpr float kBandEpsilon = 1.0f / 64.0f;  // occupancy.hpp:148
constexpr float kMarchInfinity = 1.0e30f;     // BlockMarch::kInfinity

// compat::min / compat::max (cuda_compat.hpp:75-86)
__device__ __forceinline__ float cmin(float lhs, float rhs) { return rhs < lhs ? rhs : lhs; }
__device__ __forceinline__ float cmax(float lhs, float rhs) { return lhs < rhs ? rhs : lhs; }

__device__ __forceinline__ bool band_test(const BandDev& b, uint32_t x, uint32_t y, uint32_t z) {
  const uint64_t i = (static_cast<uint64_t>(x) * b.by + y) * b.bz + z;
  return ((__ldg(b.words + (i >> 5)) >> (i & 31u)) & 1u) != 0u;
}

__device__ __forceinline__ float axis_exit(float origin, float direction, float low, float high) {
  return ((direction >= 0.0f ? high : low) - origin) / direction;
}

// BlockMarch over one ray (empty_space_skip.hpp:19-153)
struct BlockMarchDev {
  const VolumeDev& v;
  float block_size;
  f3 o, d;

  __device__ float block_exit(uint32_t x, uint32_t y, uint32_t z) const {
    const float lx = v.origin.x + (static_cast<float>(x) * block_size);
    const float ly = v.origin.y + (static_cast<float>(y) * block_size);
    const float lz = v.origin.z + (static_cast<float>(z) * block_size);
    const float hx = lx + (1.0f * block_size), hy = ly + (1.0f * block_size), hz = lz + (1.0f * block_size);
    return cmin(axis_exit(o.x, d.x, lx, hx), cmin(axis_exit(o.y, d.y, ly, hy), axis_exit(o.z, d.z, lz, hz)));
  }
  __device__ float column_exit(uint32_t x, uint32_t y) const {
    const float lx = v.origin.x + (static_cast<float>(x) * block_size);
    const float ly = v.origin.y + (static_cast<float>(y) * block_size);
    float exit = kMarchInfinity;
    if (d.x != 0.0f) exit = cmin(exit, axis_exit(o.x, d.x, lx, lx + block_size));
    if (d.y != 0.0f) exit = cmin(exit, axis_exit(o.y, d.y, ly, ly + block_size));
    return exit;
  }
  __device__ float z_entry(uint64_t z) const {
    const float side = d.z >= 0.0f ? 0.0f : 1.0f;
    const float plane = v.origin.z + ((static_cast<float>(z) + side) * block_size);
    return (plane - o.z) / d.z;
  }
  __device__ static void slab(float origin, float direction, float low, float high, float& entry, float& exit) {
    if (direction == 0.0f) {
      if (origin < low || origin > high) entry = kMarchInfinity;
      return;
    }
    const float t_low = (low - origin) / direction;
    const float t_high = (high - origin) / direction;
    entry = cmax(entry, cmin(t_low, t_high));
    exit = cmin(exit, cmax(t_low, t_high));
  }
  __device__ float volume_entry() const {
    float entry = 0.0f, exit = kMarchInfinity;
    slab(o.x, d.x, v.origin.x, v.origin.x + (static_cast<float>(v.rx) * v.voxel_size), entry, exit);
    slab(o.y, d.y, v.origin.y, v.origin.y + (static_cast<float>(v.ry) * v.voxel_size), entry, exit);
    slab(o.z, d.z, v.origin.z, v.origin.z + (static_cast<float>(v.rz) * v.voxel_size), entry, exit);
    return entry <= exit ? entry : kMarchInfinity;
  }
};

// BandSkip::word_scan_z (empty_space_skip.hpp:266-284)
__device__ float band_word_scan_z(const BandDev& b, const BlockMarchDev& m, uint32_t x, uint32_t y, uint32_t z) {
  const uint64_t index = (static_cast<uint64_t>(x) * b.by + y) * b.bz + z;
  const uint32_t word = __ldg(b.words + (index >> 5));
  const uint32_t offset = static_cast<uint32_t>(index & 31u);
  const bool forward = m.d.z >= 0.0f;
  int found;
  if (forward) {
    const uint32_t masked = word & ~((1u << offset) - 1u);  // find_set_at_or_after
    found = masked == 0u ? -1 : __ffs(static_cast<int>(masked)) - 1;
  } else {
    const uint32_t masked = word & (offset >= 31u ? ~0u : ((1u << (offset + 1u)) - 1u));  // at_or_before
    found = masked == 0u ? -1 : 31 - __clz(static_cast<int>(masked));
  }
  uint64_t target_z;
  if (found >= 0) {
    target_z = z + static_cast<uint64_t>(found) - offset;
  } else {
    target_z = forward ? z + (32u - offset) : z - (offset < z ? offset : z);
  }
  return cmin(m.z_entry(target_z), m.column_exit(x, y));
}

// BandSkip::advance (empty_space_skip.hpp:225-262)
__device__ float band_advance(const BandDev& b, const VolumeDev& v, f3 o, f3 d, float ray_length, float base_step,
                              float max_depth) {
  const BlockMarchDev m{v, 8.0f * v.voxel_size, o, d};
  const float nudge = 0.25f * v.voxel_size;
  const bool z_major = fabsf(d.z) >= fabsf(d.x) && fabsf(d.z) >= fabsf(d.y) && (b.bz % 32u) == 0u;
  while (ray_length <= max_depth) {
    const f3 point = o + (d * ray_length);
    const float gx = (point.x - v.origin.x) / v.voxel_size;
    const float gy = (point.y - v.origin.y) / v.voxel_size;
    const float gz = (point.z - v.origin.z) / v.voxel_size;
    if (!(gx >= 0.0f && gy >= 0.0f && gz >= 0.0f && gx < static_cast<float>(v.rx) &&
          gy < static_cast<float>(v.ry) && gz < static_cast<float>(v.rz))) {
      const float entry = m.volume_entry();
      if (entry >= kMarchInfinity || entry > max_depth) return max_depth + base_step;
      ray_length = cmax(ray_length + base_step, entry + nudge);
      continue;
    }
    const uint32_t x = static_cast<uint32_t>(gx) / 8u, y = static_cast<uint32_t>(gy) / 8u,
                   z = static_cast<uint32_t>(gz) / 8u;
    if (band_test(b, x, y, z)) return ray_length;
    float target = kMarchInfinity;
    if (z_major) target = band_word_scan_z(b, m, x, y, z);
    if (target >= kMarchInfinity) target = m.block_exit(x, y, z);
    ray_length = cmax(ray_length + base_step, target + nudge);
  }
  return ray_length;
}

// find_zero_crossing with BandSkip (raycasting.hpp:165-211): one thread per
// pixel; writes the crossing (NaN for none) for surface_kernel.
template <int Kind>
__global__ void __launch_bounds__(64)
    band_march_kernel(VolumeDev v, BandDev band, RaycastParams rp, Intr k, uint32_t width, uint32_t height,
                      Rigid pose, const IcpState* __restrict__ state, float* __restrict__ points) {
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
  const f3 translated = back_project(k, static_cast<float>(col), static_cast<float>(row), 1.0f);
  const f3 direction = rotate(pose, translated);
  const float dn = norm(direction);
  bool found = false;
  f3 surface = make(0.0f, 0.0f, 0.0f);
  if (dn > 0.0f) {
    const f3 dir = direction / dn;
    const float base_step = v.voxel_size * rp.step_scale;
    bool have_prev = false;
    float prev_tsdf = 0.0f;
    f3 prev_point = make(0.0f, 0.0f, 0.0f);
    float ray_length = seed;
    while (ray_length <= rp.max_depth) {
      const float advanced = band_advance(band, v, pose.t, dir, ray_length, base_step, rp.max_depth);
      if (advanced != ray_length) {
        have_prev = false;  // the skipped samples were all nullopt
        ray_length = advanced;
        if (ray_length > rp.max_depth) break;
      }
      const f3 point = pose.t + (dir * ray_length);
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
  }
  store3(points + pix * 3, found ? surface : nan3());
}

// BlockBitmapOps::rebuild with BandFilter (occupancy.hpp:105-121, 150-171):
// warp w computes raw word w (32 blocks in z-major order), reading each
// block's 512 contiguous voxels; blocks past the extent read as clear.
template <int Kind>
__global__ void __launch_bounds__(256) band_raw_kernel(VolumeDev v, uint32_t* __restrict__ raw, uint32_t words) {
  using VT = VoxelTraits<Kind>;
  using Raw = typename VT::Raw;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t first = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t stride = (gridDim.x * blockDim.x) >> 5;
  const uint64_t total = static_cast<uint64_t>(v.bx) * v.by * v.bz;
  const Raw* vox = static_cast<const Raw*>(v.voxels);
  for (uint32_t w = first; w < words; w += stride) {
    uint32_t word = 0;
    for (uint32_t j = 0; j < 32u; ++j) {
      const uint64_t i = static_cast<uint64_t>(w) * 32u + j;
      if (i >= total) break;  // warp-uniform
      const uint32_t z = static_cast<uint32_t>(i % v.bz);
      const uint32_t y = static_cast<uint32_t>((i / v.bz) % v.by);
      const uint32_t x = static_cast<uint32_t>(i / (static_cast<uint64_t>(v.bz) * v.by));
      const Raw* brick = vox + ((static_cast<size_t>(z) * v.by + y) * v.bx + x) * 512u;
      bool any = false;
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const Raw r = brick[lane + 32u * q];
        any |= VT::observed(r) && VT::tsdf(r) < (1.0f - kBandEpsilon);
      }
      if (__any_sync(0xFFFFFFFFu, any)) word |= 1u << j;
    }
    if (lane == 0) raw[w] = word;
  }
}

// BlockBitmapOps::dilate (occupancy.hpp:69-103): bit i is set when a block
// of its clipped 3^3 neighbourhood is in the raw band.  One thread per bit,
// one warp per word.
__global__ void __launch_bounds__(256) band_dilate_kernel(const uint32_t* __restrict__ raw, uint32_t* __restrict__ map,
                                                          uint32_t bx, uint32_t by, uint32_t bz, uint32_t words) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t total = static_cast<uint64_t>(bx) * by * bz;
  bool hit = false;
  if (i < total) {
    const int z = static_cast<int>(i % bz), y = static_cast<int>((i / bz) % by);
    const int x = static_cast<int>(i / (static_cast<uint64_t>(bz) * by));
    for (int oz = -1; oz <= 1 && !hit; ++oz) {
      for (int oy = -1; oy <= 1 && !hit; ++oy) {
        for (int ox = -1; ox <= 1 && !hit; ++ox) {
          const int nx = x + ox, ny = y + oy, nz = z + oz;
          if (nx < 0 || ny < 0 || nz < 0 || nx >= static_cast<int>(bx) || ny >= static_cast<int>(by) ||
              nz >= static_cast<int>(bz)) {
            continue;
          }
          const uint64_t n = (static_cast<uint64_t>(nx) * by + ny) * bz + nz;
          hit = ((__ldg(raw + (n >> 5)) >> (n & 31u)) & 1u) != 0u;
        }
      }
    }
  }
  const uint32_t word = __ballot_sync(0xFFFFFFFFu, hit);
  if ((threadIdx.x & 31u) == 0 && (i >> 5) < words) map[i >> 5] = word;
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
  const uint64_t rays = static_cast<uint64_t>(cam.width) * cam.height;
  const uint32_t lanes = p.raycast_lanes[rays <= 20000u ? 0 : (rays <= 80000u ? 1 : 2)];
  rp.rays_per_warp = p.config.raycast_backend == KF_RAYCAST_BAND_MARCH ? 32u : 32u / lanes;
  rp.coop_rays = rp.rays_per_warp < 32u ? kCoopLanes : 0;
  dim3 block(p.raycast_block_x, p.raycast_block_y);
  dim3 grid(ceil_div(cam.width, block.x), ceil_div(cam.height, block.y));
  if (rp.rays_per_warp < 32u) {
    // two warps per CTA, each a tw x th pixel tile (warp_tile_pixel)
    const uint32_t tw = rp.rays_per_warp < 4u ? rp.rays_per_warp : 4u, th = rp.rays_per_warp / tw;
    block = dim3(64, 1);
    grid = dim3(ceil_div(cam.width, tw), ceil_div(cam.height, 2u * th));
  }
  // the skip structures exist once a full-sweep integration prepared them
  const uint32_t* voxel_bits = p.brick_class.count && p.view.table == nullptr ? p.voxel_bits.ptr : nullptr;
  const uint4* stencil_bits = reinterpret_cast<const uint4*>(p.stencil_bits.ptr);
  const Rigid pose = rigid_from(cam.camera_to_world);
  if (p.config.raycast_backend == KF_RAYCAST_BAND_MARCH) {
    const BandDev band{p.band_map.ptr, p.view.bx, p.view.by, p.view.bz};
    band_march_kernel<Kind><<<grid, block, 0, s>>>(p.view, band, rp, intr_from(cam.intrinsics), cam.width,
                                                   cam.height, pose, state, points);
    check(cudaGetLastError(), "band_march_kernel launch");
  } else {
    const uint8_t* null_bricks = p.view.table != nullptr ? p.null_bricks.ptr : nullptr;
    const uint8_t* brick_radius = voxel_bits != nullptr && p.brick_radius.count ? p.brick_radius.ptr : nullptr;
    raycast_kernel<Kind><<<grid, block, 0, s>>>(p.view, voxel_bits, stencil_bits, p.brick_class.ptr, brick_radius,
                                                null_bricks, rp,
                                                intr_from(cam.intrinsics), cam.width, cam.height, pose, state,
                                                points);
    check(cudaGetLastError(), "raycast_kernel launch");
  }
  const dim3 sblock(32, 4);
  const dim3 sgrid(ceil_div(cam.width, 32), ceil_div(cam.height, 4));
  surface_kernel<Kind, Color><<<sgrid, sblock, 0, s>>>(p.view, rp, cam.width, cam.height, pose, state, points,
                                                       normals, colors);
  check(cudaGetLastError(), "surface_kernel launch");
}

}  // namespace

void launch_band_rebuild(Pipeline& p, cudaStream_t s) {
  if (p.band_map.count == 0) return;
  const uint32_t words = static_cast<uint32_t>(p.band_map.count);
  const unsigned grid = std::min<unsigned>(148u * 8u, ceil_div(words * 32u, 256u));
  switch (p.config.voxel) {
    case KF_VOXEL_QUANTIZED:
      band_raw_kernel<KF_VOXEL_QUANTIZED><<<grid, 256, 0, s>>>(p.view, p.band_raw.ptr, words);
      break;
    case KF_VOXEL_BF16:
      band_raw_kernel<KF_VOXEL_BF16><<<grid, 256, 0, s>>>(p.view, p.band_raw.ptr, words);
      break;
    default:
      band_raw_kernel<KF_VOXEL_FLOAT><<<grid, 256, 0, s>>>(p.view, p.band_raw.ptr, words);
      break;
  }
  check(cudaGetLastError(), "band_raw_kernel launch");
  band_dilate_kernel<<<ceil_div(words * 32u, 256u), 256, 0, s>>>(p.band_raw.ptr, p.band_map.ptr, p.view.bx,
                                                                  p.view.by, p.view.bz, words);
  check(cudaGetLastError(), "band_dilate_kernel launch");
}

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
