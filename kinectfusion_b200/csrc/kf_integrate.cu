// kf_integrate.cu - projective TSDF integration into a dense volume
// (IntegrationContext::observe/fuse + ClassicTsdf/AngleWeightedTsdf,
// tsdf_integration.hpp:127-342; reference device sweep tsdf_integration.cu:61-107).
//
// The reference sweeps every (x, y) column of the volume and tests every voxel
// of a column that projects into the image.  Almost all of that work is in
// voxels that cannot fuse: behind the measured surface or outside the image.
// Here the full sweep runs in three steps, with the same result:
//
//  1. pixel table: one float4 per depth pixel - depth in metres (NaN when
//     unusable), |K^-1 [u v 1]|, the rule's observation weight, RGBA8 colour.
//     These are the per-pixel parts of observe(), the same float expressions
//     evaluated once per pixel instead of once per voxel.
//  2. block culling: a max-depth pyramid over 8x8 pixel tiles, then one
//     thread per 8^3 block bounds the block's projection and camera depth.
//     A block is dropped only when no voxel of it can fuse: it lies behind
//     the camera, projects outside the image (1.5-pixel margin), or is
//     farther than (max depth of its footprint + truncation) * (1 + 2/f)
//     (a fused voxel has |p|/lambda <= depth + truncation, and |p|/lambda >=
//     p.z * (1 - 0.71/f) since the pixel ray is rounded by half a pixel).
//  3. listed-block integration: one CTA per surviving block, every voxel
//     runs the exact host observe/fuse; the CTA also maintains the raycast's
//     skip bits (per voxel: observed / exactly 1; per block: free / observed).
//
// Voxels are bricked (kf_common.cuh): a CTA's block is 512 contiguous
// voxels and a warp reads and writes 32 consecutive ones (256 B for float).
#include <algorithm>
#include <cmath>

#include "kf_internal.h"

namespace kf {
namespace {

struct IntegParams {
  float max_weight;
  int projective_distance;
  int distance_scaled_truncation;
  float truncation_distance_scale;
  int has_color;
};

constexpr int kTile = 8;          // pixels per depth tile edge
constexpr int kBlockThreads = 128;

// Per-pixel part of IntegrationContext::observe and the rule weight
// (tsdf_integration.hpp:196-212, 329-342).
__global__ void pixel_table_kernel(const uint16_t* __restrict__ depth, const uint32_t* __restrict__ color,
                                   const float* __restrict__ normals, uint32_t width, uint32_t height,
                                   Intr k, float depth_scale, float min_depth, float max_depth,
                                   float observation_weight, int angle_weighted,
                                   float4* __restrict__ table) {
  const uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t row = blockIdx.y * blockDim.y + threadIdx.y;
  if (col >= width || row >= height) return;
  const size_t pix = static_cast<size_t>(row) * width + col;
  float sd;
  bool valid = depth_in_range(depth[pix], depth_scale, min_depth, max_depth, sd);
  const f3 ray = back_project(k, static_cast<float>(col), static_cast<float>(row), 1.0f);
  const float lambda = norm(ray);
  if (!finite3(ray) || lambda == 0.0f) valid = false;
  float weight = observation_weight;
  if (valid && angle_weighted && normals != nullptr) {
    const f3 n = load3(normals + pix * 3);
    if (finite3(n)) {
      const f3 view = -normalized(ray);
      const float d = dot(normalized(n), view);
      const float cos_theta = 0.0f < d ? d : 0.0f;
      weight *= cos_theta / sd;
    }
  }
  const uint32_t c = color != nullptr ? color[pix] : 0u;
  table[pix] = make_float4(valid ? sd : kNaN, lambda, weight, __uint_as_float(c));
}

// Level 0 of the depth-tile pyramid: the largest usable depth of each 8x8
// pixel tile (0 when the tile has none).
__global__ void tile_max_kernel(const float4* __restrict__ table, uint32_t width, uint32_t height,
                                uint32_t tiles_x, uint32_t tiles_y, float* __restrict__ out) {
  const uint32_t tx = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t ty = blockIdx.y * blockDim.y + threadIdx.y;
  if (tx >= tiles_x || ty >= tiles_y) return;
  float m = 0.0f;
  for (uint32_t y = ty * kTile; y < min((ty + 1) * kTile, height); ++y) {
    for (uint32_t x = tx * kTile; x < min((tx + 1) * kTile, width); ++x) {
      const float d = __ldg(&table[static_cast<size_t>(y) * width + x].x);
      if (d > m) m = d;  // NaN compares false
    }
  }
  out[ty * tiles_x + tx] = m;
}

struct TileLevels {
  uint32_t count;
  uint32_t w[12], h[12], off[12];
};

// Coarser levels by 2x2 max, one CTA (the pyramid is a few thousand values).
__global__ void tile_pyramid_kernel(float* __restrict__ tiles, TileLevels lv) {
  for (uint32_t l = 1; l < lv.count; ++l) {
    const float* src = tiles + lv.off[l - 1];
    float* dst = tiles + lv.off[l];
    const uint32_t n = lv.w[l] * lv.h[l];
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
      const uint32_t x = i % lv.w[l], y = i / lv.w[l];
      float m = 0.0f;
      for (uint32_t dy = 0; dy < 2; ++dy) {
        for (uint32_t dx = 0; dx < 2; ++dx) {
          const uint32_t sx = x * 2 + dx, sy = y * 2 + dy;
          if (sx < lv.w[l - 1] && sy < lv.h[l - 1]) m = fmaxf(m, src[sy * lv.w[l - 1] + sx]);
        }
      }
      dst[i] = m;
    }
    __syncthreads();
  }
}

struct CullParams {
  float trunc_base, trunc_scale;
  int distance_scaled;
  float slack;  // 1 / (1 - 2/f)
  uint32_t width, height;
};

// Step 2: one thread per 8^3 block; survivors are appended to `list`.
__global__ void cull_blocks_kernel(VolumeDev v, Rigid T, Intr k, const float* __restrict__ tiles, TileLevels lv,
                                   CullParams cp, const IcpState* __restrict__ state, uint32_t* __restrict__ list,
                                   unsigned* __restrict__ count) {
  if (state != nullptr) {
    if (state->failed) return;
    const float* w = state->world_to_camera;
    T = Rigid{{w[0], w[1], w[2]}, {w[3], w[4], w[5]}, {w[6], w[7], w[8]}, {w[9], w[10], w[11]}};
  }
  const uint32_t block = blockIdx.x * blockDim.x + threadIdx.x;
  bool keep = false;
  if (block < v.bx * v.by * v.bz) {
    const uint32_t bxi = block % v.bx, byi = (block / v.bx) % v.by, bzi = block / (v.bx * v.by);
    const float x0 = static_cast<float>(bxi * 8) + 0.5f, x1 = static_cast<float>(min(bxi * 8 + 8, v.rx) - 1) + 0.5f;
    const float y0 = static_cast<float>(byi * 8) + 0.5f, y1 = static_cast<float>(min(byi * 8 + 8, v.ry) - 1) + 0.5f;
    const float z0 = static_cast<float>(bzi * 8) + 0.5f, z1 = static_cast<float>(min(bzi * 8 + 8, v.rz) - 1) + 0.5f;
    float zmin = 1e30f, zmax = -1e30f, umin = 1e30f, umax = -1e30f, vmin = 1e30f, vmax = -1e30f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const f3 w = v.origin + make(c & 1 ? x1 : x0, c & 2 ? y1 : y0, c & 4 ? z1 : z0) * v.voxel_size;
      const f3 p = apply(T, w);
      zmin = fminf(zmin, p.z);
      zmax = fmaxf(zmax, p.z);
      if (p.z > 1e-4f) {
        const float u = (k.fx * p.x) / p.z + k.cx, vv = (k.fy * p.y) / p.z + k.cy;
        umin = fminf(umin, u);
        umax = fmaxf(umax, u);
        vmin = fminf(vmin, vv);
        vmax = fmaxf(vmax, vv);
      }
    }
    const float fw = static_cast<float>(cp.width), fh = static_cast<float>(cp.height);
    if (zmax > 0.0f) {
      if (zmin <= 1e-4f) {
        keep = true;  // straddles the camera plane: the projection is unbounded
      } else if (umax >= -2.0f && vmax >= -2.0f && umin <= fw + 1.0f && vmin <= fh + 1.0f) {
        const int u0 = max(0, static_cast<int>(floorf(umin - 1.5f)));
        const int u1 = min(static_cast<int>(cp.width) - 1, static_cast<int>(ceilf(umax + 1.5f)));
        const int v0 = max(0, static_cast<int>(floorf(vmin - 1.5f)));
        const int v1 = min(static_cast<int>(cp.height) - 1, static_cast<int>(ceilf(vmax + 1.5f)));
        if (u0 <= u1 && v0 <= v1) {
          // the finest level whose tiles cover the rectangle with at most
          // 4x4 texels (any level's tiles over the rectangle bound every pixel
          // in it; finer ones bound it tighter)
          int tx0 = u0 / kTile, tx1 = u1 / kTile, ty0 = v0 / kTile, ty1 = v1 / kTile;
          uint32_t l = 0;
          while (l + 1 < lv.count && (tx1 - tx0 > 3 || ty1 - ty0 > 3)) {
            tx0 >>= 1;
            tx1 >>= 1;
            ty0 >>= 1;
            ty1 >>= 1;
            ++l;
          }
          float maxd = 0.0f;
          for (int ty = ty0; ty <= ty1; ++ty)
            for (int tx = tx0; tx <= tx1; ++tx) maxd = fmaxf(maxd, __ldg(tiles + lv.off[l] + ty * lv.w[l] + tx));
          if (maxd > 0.0f) {
            const float trunc = cp.distance_scaled ? cp.trunc_base + cp.trunc_scale * maxd : cp.trunc_base;
            keep = zmin <= (maxd + trunc) * cp.slack + 1e-3f;
          }
        }
      }
    }
  }
  // warp-aggregated append
  const unsigned ballot = __ballot_sync(0xFFFFFFFFu, keep);
  if (ballot == 0) return;
  const int lane = threadIdx.x & 31;
  unsigned base = 0;
  if (lane == __ffs(ballot) - 1) base = atomicAdd(count, static_cast<unsigned>(__popc(ballot)));
  base = __shfl_sync(0xFFFFFFFFu, base, __ffs(ballot) - 1);
  if (keep) list[base + __popc(ballot & ((1u << lane) - 1u))] = block;
}

// The pixel lround(project(K, p)) of a camera point, as observe() picks it
// (tsdf_integration.hpp:196-205), decided without the projection's two IEEE
// divisions where that cannot change the answer: 1 = in the image at
// (rx, ry), -1 = no pixel (behind the camera or outside the image), 0 = too
// close to a rounding boundary (k + 0.5) to tell - the caller then runs the
// exact quotient.  The estimate uses __fdividef (at most 2 ulp): below 2048
// in magnitude it is within 1.3e-3 pixel of the exact value, so a margin of
// 4e-3 pixel decides exactly; beyond that the point is outside any image
// this path accepts (width and height up to 2048; wider images always take
// the exact path).  Rounding to nearest even equals lround away from the
// half-way points.
__device__ __forceinline__ int pixel_estimate(const Intr& k, f3 p, uint32_t width, uint32_t height, uint32_t& rx,
                                              uint32_t& ry) {
  if (!(p.z > 0.0f)) return -1;
  if (!(p.z >= 1e-6f) || width > 2048u || height > 2048u) return 0;
  const float ax = __fdividef(k.fx * p.x, p.z) + k.cx;
  const float ay = __fdividef(k.fy * p.y, p.z) + k.cy;
  if (!(fabsf(ax) < 2048.0f && fabsf(ay) < 2048.0f)) return -1;
  const float nx = rintf(ax), ny = rintf(ay);
  if (fabsf(ax - nx) > 0.5f - 4e-3f || fabsf(ay - ny) > 0.5f - 4e-3f) return 0;
  const int ix = __float2int_rn(nx), iy = __float2int_rn(ny);
  if (static_cast<uint32_t>(ix) >= width || static_cast<uint32_t>(iy) >= height) return -1;
  rx = static_cast<uint32_t>(ix);
  ry = static_cast<uint32_t>(iy);
  return 1;
}

// Where the projective sdf = d - |p| / lambda falls: -1 certainly below
// -truncation (no update), +1 certainly at or above +truncation (the update
// writes tsdf exactly 1), 0 undecided (the exact expression runs).  |p| and
// the quotient are estimated with rsqrtf and __fdividef (relative error below
// 1e-6 together); the margin is 1e-4 m plus 1e-6 of the distance, far above
// that error.
__device__ __forceinline__ int sdf_region(f3 p, float d, float lambda, float truncation) {
  const float s2 = dot(p, p);
  if (!(s2 > 1e-30f) || !(lambda >= 1.0f)) return 0;
  const float dist = __fdividef(s2 * rsqrtf(s2), lambda);
  const float est = d - dist;
  const float margin = 1e-4f + 1e-6f * dist;
  if (est < -truncation - margin) return -1;
  if (est > truncation + margin) return 1;
  return 0;
}

// Step 3: one CTA per listed block, four voxels (along z) per thread.
template <int Kind, bool Color>
__global__ void __launch_bounds__(kBlockThreads, 10)
    integrate_blocks_kernel(VolumeDev v, const float4* __restrict__ table, uint32_t width, uint32_t height, Intr k,
                            Rigid T, IntegParams ip, const IcpState* __restrict__ state,
                            const uint32_t* __restrict__ list, const unsigned* __restrict__ count,
                            uint32_t* __restrict__ voxel_bits, uint32_t* __restrict__ dirty_bits,
                            unsigned long long* __restrict__ counters) {
  using VT = VoxelTraits<Kind>;
  using Raw = typename VT::Raw;
  if (state != nullptr) {
    if (state->failed) return;
    const float* w = state->world_to_camera;
    T = Rigid{{w[0], w[1], w[2]}, {w[3], w[4], w[5]}, {w[6], w[7], w[8]}, {w[9], w[10], w[11]}};
  }
  Raw* __restrict__ voxels = reinterpret_cast<Raw*>(v.voxels);
  const unsigned n = *count;
  // Per block, two passes over its 512 voxels (thread t: x = t & 7,
  // y = (t >> 3) & 7, z = 4 (t >> 6) + i, i < 4):
  //  A. every voxel: camera point, pixel, table entry, and the sdf's region
  //     from an error-bounded estimate (sdf_region).  Voxels certainly behind
  //     the band are done; voxels certainly in front of it whose stored tsdf
  //     is exactly 1 fuse to exactly 1 without a division.  Everything else
  //     (including voxels whose pixel sits at a rounding boundary of the
  //     estimate) goes to the block's queue in shared memory.
  //  B. the queue, densely, one voxel per thread: the exact sdf and the
  //     exact weighted average.
  // Both passes set the voxel's bits in shared masks (bit v of the 512-bit
  // masks, v = z * 64 + y * 8 + x), which the raycast's skip bits take
  // afterwards.  The work per voxel is the host expression either way, so
  // the stored bits are the same; the queue only keeps a warp's lanes busy
  // with the voxels that need the long exact path.
  __shared__ uint32_t s_fused[16], s_one[16];
  __shared__ unsigned s_queued;
  __shared__ uint16_t s_queue_voxel[512];
  __shared__ float4 s_queue_table[512];
  const uint32_t lx = threadIdx.x & 7u, ly = (threadIdx.x >> 3) & 7u, lz = (threadIdx.x >> 6) * 4u;
  unsigned updates = 0, color_updates = 0;
  for (unsigned item = blockIdx.x; item < n; item += gridDim.x) {
    const uint32_t block = list[item];
    // sparse volumes: listed blocks are allocated (SparseVolumeView::find_voxel)
    const uint32_t slot = v.table != nullptr ? block_table_lookup(v.table, v.table_mask, block) : block;
    const uint32_t bxi = block % v.bx, byi = (block / v.bx) % v.by, bzi = block / (v.bx * v.by);
    if (threadIdx.x < 16) {
      s_fused[threadIdx.x] = 0u;
      s_one[threadIdx.x] = 0u;
    }
    if (threadIdx.x == 0) s_queued = 0u;
    __syncthreads();
    Raw* __restrict__ brick = voxels + static_cast<size_t>(slot) * 512;
    // ---- pass A ------------------------------------------------------------
    {
      const uint32_t x = bxi * 8 + lx, y = byi * 8 + ly;
      f3 cp[4];
      float4 tb[4];
      uint32_t seen = 0;     // bit i: voxel i projects into the image
      uint32_t unknown = 0;  // bit i: voxel i's pixel needs the exact quotient
      // IntegrationContext::observe's pixel and table entry
      // (tsdf_integration.hpp:183-205), the four gathers in flight together
#pragma unroll
      for (uint32_t i = 0; i < 4; ++i) {
        const uint32_t z = bzi * 8 + lz + i;
        tb[i] = make_float4(kNaN, 0.0f, 0.0f, 0.0f);
        cp[i] = make(0.0f, 0.0f, 0.0f);
        if (x < v.rx && y < v.ry && z < v.rz) {
          cp[i] = apply(T, cell_center(v, x, y, z));
          uint32_t rx = 0, ry = 0;
          const int pe = pixel_estimate(k, cp[i], width, height, rx, ry);
          if (pe > 0) {
            tb[i] = __ldg(table + (static_cast<size_t>(ry) * width + rx));
            seen |= 1u << i;
          } else if (pe == 0) {
            unknown |= 1u << i;
          }
        }
      }
      // the sdf's region (tsdf_integration.hpp:206-224): -1 no update, 1 in
      // front of the band (tsdf exactly 1), 0 needs the exact sdf
      int region[4];
#pragma unroll
      for (uint32_t i = 0; i < 4; ++i) {
        region[i] = -1;
        if (!((seen >> i) & 1u)) continue;
        const float sd = tb[i].x;
        if (isnan(sd) || !(tb[i].z > 0.0f)) continue;
        const float truncation =
            ip.distance_scaled_truncation ? v.truncation + (ip.truncation_distance_scale * sd) : v.truncation;
        if (ip.projective_distance) {
          region[i] = sdf_region(cp[i], sd, tb[i].y, truncation);
        } else {
          const float d = sd - cp[i].z;  // exact already
          region[i] = d < -truncation ? -1 : (d >= truncation ? 1 : 0);
        }
      }
      Raw old[4];
#pragma unroll
      for (uint32_t i = 0; i < 4; ++i) {
        if (region[i] > 0) old[i] = brick[(lz + i) * 64u + ly * 8u + lx];
      }
#pragma unroll
      for (uint32_t i = 0; i < 4; ++i) {
        const uint32_t vi = (lz + i) * 64u + ly * 8u + lx;
        if ((unknown >> i) & 1u) {
          const unsigned q = atomicAdd(&s_queued, 1u);
          s_queue_voxel[q] = static_cast<uint16_t>(vi | 0x4000u);
          continue;
        }
        if (region[i] < 0) continue;
        if (region[i] > 0 && VT::tsdf(old[i]) == 1.0f) {
          // sdf >= truncation: clamp(sdf / truncation) is exactly 1, and
          // (1 * w0 + 1 * ow) / (w0 + ow) is exactly 1 (BasicVoxel::fused,
          // volume.hpp:137-146); no colour update (sdf > truncation / 2)
          const float sum_w = VT::weight(old[i]) + tb[i].z;
          const Raw fused = VT::encode(1.0f, ip.max_weight < sum_w ? ip.max_weight : sum_w);
          brick[vi] = fused;
          ++updates;
          atomicOr(&s_fused[vi >> 5], 1u << (vi & 31u));
          if (VT::tsdf(fused) == 1.0f) atomicOr(&s_one[vi >> 5], 1u << (vi & 31u));
        } else {
          const unsigned q = atomicAdd(&s_queued, 1u);
          s_queue_voxel[q] = static_cast<uint16_t>(vi | (region[i] > 0 ? 0x8000u : 0u));
          s_queue_table[q] = tb[i];
        }
      }
    }
    __syncthreads();
    // ---- pass B: the queued voxels, exact ----------------------------------
    const unsigned queued = s_queued;
    for (unsigned q = threadIdx.x; q < queued; q += kBlockThreads) {
      const uint32_t tag = s_queue_voxel[q];
      const uint32_t vi = tag & 0x1FFu;
      const bool front = (tag & 0x8000u) != 0u;
      const uint32_t x = bxi * 8 + (vi & 7u), y = byi * 8 + ((vi >> 3) & 7u), z = bzi * 8 + (vi >> 6);
      const f3 cp = apply(T, cell_center(v, x, y, z));
      float4 tb;
      if (tag & 0x4000u) {
        // the exact pixel (tsdf_integration.hpp:196-205) and its table entry
        float px, py;
        project(k, cp, px, py);
        const long rx = lroundf(px), ry = lroundf(py);
        if (!(rx >= 0 && ry >= 0 && rx < static_cast<long>(width) && ry < static_cast<long>(height))) continue;
        tb = __ldg(table + (static_cast<size_t>(ry) * width + static_cast<size_t>(rx)));
        if (isnan(tb.x) || !(tb.z > 0.0f)) continue;
      } else {
        tb = s_queue_table[q];
      }
      const float sd = tb.x, ow = tb.z;
      const float truncation =
          ip.distance_scaled_truncation ? v.truncation + (ip.truncation_distance_scale * sd) : v.truncation;
      float tsdf = 1.0f, sdf = 0.0f;
      if (!front) {
        sdf = ip.projective_distance ? sd - (norm(cp) / tb.y) : sd - cp.z;
        if (sdf < -truncation) continue;
        tsdf = clampf(sdf / truncation, -1.0f, 1.0f);
      }
      // ClassicTsdf / AngleWeightedTsdf::update -> BasicVoxel::fused
      // (tsdf_integration.hpp:287-342, volume.hpp:137-146)
      const Raw old = brick[vi];
      const float t0 = VT::tsdf(old);
      const float w0 = VT::weight(old);
      const float sum_w = w0 + ow;
      const float avg = ((t0 * w0) + (tsdf * ow)) / sum_w;
      const Raw fused = VT::encode(avg, ip.max_weight < sum_w ? ip.max_weight : sum_w);
      brick[vi] = fused;
      ++updates;
      atomicOr(&s_fused[vi >> 5], 1u << (vi & 31u));
      if (VT::tsdf(fused) == 1.0f) atomicOr(&s_one[vi >> 5], 1u << (vi & 31u));
      if constexpr (Color) {
        if (ip.has_color && !front && sdf <= truncation * 0.5f) {
          // ColorVoxel::fused (volume.hpp:160-170)
          ++color_updates;
          float4* __restrict__ cbrick = v.colors + static_cast<size_t>(slot) * 512;
          const float4 cv = cbrick[vi];
          const f3 c = color_from_pixel(__float_as_uint(tb.w));
          const f3 avgc = ((make(cv.x, cv.y, cv.z) * cv.w) + (c * ow)) / (cv.w + ow);
          const float cw = cv.w + ow;
          cbrick[vi] = make_float4(avgc.x, avgc.y, avgc.z, ip.max_weight < cw ? ip.max_weight : cw);
        }
      }
    }
    __syncthreads();
    // ---- skip bits of the raycast ---------------------------------------
    // Per voxel: `one` (observed with tsdf exactly 1) and `observed`.  A
    // brick layer z is 16 bytes: words 4z, 4z+1 hold `one`, 4z+2, 4z+3 hold
    // `observed`, bit (y & 3) * 8 + x of word (y >> 2) - mask word w of the
    // shared masks is layer w >> 1, half w & 1.  The voxels fused this frame
    // take their new bits, the others keep theirs.
    if (voxel_bits != nullptr) {
      uint32_t* bits = voxel_bits + static_cast<size_t>(block) * 32u;
      uint32_t changed = 0u;
      if (threadIdx.x < 16) {
        const uint32_t fused = s_fused[threadIdx.x];
        if (fused != 0u) {
          const uint32_t w = 4u * (threadIdx.x >> 1) + (threadIdx.x & 1u);
          const uint32_t old_one = __ldcg(bits + w), old_obs = __ldcg(bits + w + 2u);
          const uint32_t one = (old_one & ~fused) | (s_one[threadIdx.x] & fused);
          const uint32_t obs = old_obs | fused;
          if (one != old_one || obs != old_obs) {
            bits[w] = one;
            bits[w + 2u] = obs;
            changed = 1u;
          }
        }
      }
      if (__syncthreads_or(changed != 0u) && threadIdx.x == 0) {
        atomicOr(dirty_bits + (block >> 5), 1u << (block & 31u));
      }
    } else {
      __syncthreads();  // the masks and the queue are reused by the next block
    }
  }
  const unsigned total = __reduce_add_sync(0xFFFFFFFFu, updates);
  const unsigned total_color = __reduce_add_sync(0xFFFFFFFFu, color_updates);
  if ((threadIdx.x & 31u) == 0 && counters != nullptr) {
    if (total) atomicAdd(counters, static_cast<unsigned long long>(total));
    if (total_color) atomicAdd(counters + 1, static_cast<unsigned long long>(total_color));
  }
}

// Stencil bits of one brick layer from the per-voxel bits of the brick and
// its +x, +y, +z neighbours (missing neighbours: no voxel observed).  Bit
// y*8+x of the result describes the trilinear stencil whose base corner is
// voxel (x, y, z) of the brick, i.e. corners (x..x+1, y..y+1, z..z+1).  Only
// bricks whose stencils reach a brick changed this frame are rewritten.
__device__ __forceinline__ uint64_t lo64(uint4 l) { return (static_cast<uint64_t>(l.y) << 32) | l.x; }
__device__ __forceinline__ uint64_t hi64(uint4 l) { return (static_cast<uint64_t>(l.w) << 32) | l.z; }
// value at (x+1, y) for every (x, y); column x = 7 from the +x neighbour's column 0
__device__ __forceinline__ uint64_t next_x(uint64_t a, uint64_t ax) {
  return ((a >> 1) & 0x7F7F7F7F7F7F7F7Full) | ((ax & 0x0101010101010101ull) << 7);
}
// value at (x, y+1); row y = 7 from the +y neighbour's row 0
__device__ __forceinline__ uint64_t next_y(uint64_t a, uint64_t ay) { return (a >> 8) | (ay << 56); }

__global__ void stencil_bits_kernel(const uint4* __restrict__ voxel_bits, uint4* __restrict__ stencil_bits,
                                    uint8_t* __restrict__ brick_class, const uint32_t* __restrict__ dirty,
                                    uint32_t bx, uint32_t by, uint32_t bz, int require_all,
                                    const IcpState* __restrict__ state) {
  if (state != nullptr && state->failed) return;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t brick = t >> 3, z = t & 7u;
  const uint32_t x0 = brick % bx, y0 = (brick / bx) % by, z0 = brick / (bx * by);
  // the brick's eight lanes (one per layer) each test one of the eight
  // bricks its stencils reach (itself and its +x, +y, +z neighbours); the
  // brick is rewritten when any of them changed
  bool changed = false;
  if (brick < bx * by * bz) {
    const uint32_t nx = x0 + (z & 1u), ny = y0 + ((z >> 1) & 1u), nz = z0 + (z >> 2);
    if (nx < bx && ny < by && nz < bz) {
      const uint32_t nb = (nz * by + ny) * bx + nx;
      changed = ((__ldg(dirty + (nb >> 5)) >> (nb & 31u)) & 1u) != 0u;
    }
  }
  const bool work = ((__ballot_sync(0xFFFFFFFFu, changed) >> ((threadIdx.x & 31u) & ~7u)) & 0xFFu) != 0u;
  uint64_t undecided = 0u, one = 0u;
  if (work) {
    uint64_t any_obs = 0u, all_obs = ~0ull, no_bad = ~0ull;
#pragma unroll
    for (uint32_t dz = 0; dz < 2; ++dz) {
      const uint32_t lz = z + dz, nz = z0 + (lz >> 3);
      uint4 q[4];  // (x, y), (x+1, y), (x, y+1), (x+1, y+1) bricks, this layer
#pragma unroll
      for (uint32_t c = 0; c < 4; ++c) {
        const uint32_t nx = x0 + (c & 1u), ny = y0 + (c >> 1);
        q[c] = nx < bx && ny < by && nz < bz
                   ? __ldg(voxel_bits + static_cast<size_t>((nz * by + ny) * bx + nx) * 8u + (lz & 7u))
                   : make_uint4(0u, 0u, 0u, 0u);
      }
      // observed
      const uint64_t o = hi64(q[0]), ox = hi64(q[1]), oy = hi64(q[2]), oxy = hi64(q[3]);
      const uint64_t o1 = next_x(o, ox), o2 = next_y(o, oy), o3 = next_y(o1, next_x(oy, oxy));
      any_obs |= o | o1 | o2 | o3;
      all_obs &= o & o1 & o2 & o3;
      // observed implies exactly 1
      const uint64_t b = lo64(q[0]) | ~o, bxn = lo64(q[1]) | ~ox, byn = lo64(q[2]) | ~oy, bxy = lo64(q[3]) | ~oxy;
      const uint64_t b1 = next_x(b, bxn), b2 = next_y(b, byn), b3 = next_y(b1, next_x(byn, bxy));
      no_bad &= b & b1 & b2 & b3;
    }
    one = all_obs & no_bad;
    // REQUIRE_ALL: a missing corner gives nullopt; otherwise only a stencil
    // without any observed corner does
    const uint64_t decided = require_all ? (~all_obs | no_bad) : (~any_obs | one);
    undecided = ~decided;
    // An undecided stencil keeps its "one" bit when every observed corner is
    // exactly 1 (the corner weights decide between 1.0 and nullopt); without
    // it, an observed corner holds another value and only the gather decides.
    const uint64_t weigh = undecided & no_bad;
    stencil_bits[static_cast<size_t>(brick) * 8u + z] =
        make_uint4(static_cast<uint32_t>(undecided), static_cast<uint32_t>(undecided >> 32),
                   static_cast<uint32_t>(one | weigh), static_cast<uint32_t>((one | weigh) >> 32));
  }
  // brick summary from its eight layers (eight consecutive lanes)
  const uint32_t all_null = __ballot_sync(0xFFFFFFFFu, undecided == 0u && one == 0u);
  const uint32_t all_one = __ballot_sync(0xFFFFFFFFu, one == ~0ull);
  if (work && z == 0) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n8 = (all_null >> lane) & 0xFFu, o8 = (all_one >> lane) & 0xFFu;
    brick_class[brick] = static_cast<uint8_t>(n8 == 0xFFu ? 1u : (o8 == 0xFFu ? 2u : 0u));
  }
}

// Per brick of class 1 or 2: the largest r <= kBrickRadiusCap such that
// every brick within Chebyshev distance r (in bricks) has the same class;
// bricks past the brick grid count as different, so the cube stays inside
// it.  Mixed bricks get 0.  The raycast crosses such a cube in one go, as it
// crosses a single brick of that class.  Three separable passes, one per
// axis: `lower` (the previous pass's radius: the run along x, then the
// square in x and y) bounds the radius at every brick of the new axis'
// segment; the x pass has none.
constexpr uint32_t kBrickRadiusCap = 7;
__global__ void brick_radius_kernel(const uint8_t* __restrict__ brick_class, const uint8_t* __restrict__ lower,
                                    uint8_t* __restrict__ out, uint32_t bx, uint32_t by, uint32_t bz, int axis,
                                    const IcpState* __restrict__ state) {
  if (state != nullptr && state->failed) return;  // no integration this frame: the classes stand
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= bx * by * bz) return;
  const uint32_t c = brick_class[b];
  if (c != 1u && c != 2u) {
    out[b] = 0;
    return;
  }
  const uint32_t coord = axis == 0 ? b % bx : (axis == 1 ? (b / bx) % by : b / (bx * by));
  const uint32_t extent = axis == 0 ? bx : (axis == 1 ? by : bz);
  const size_t stride = axis == 0 ? 1u : (axis == 1 ? bx : static_cast<size_t>(bx) * by);
  // r = the first k that fails, less one: both neighbours at distance k
  // inside the grid and of class c, and (later passes) k within the bound
  // of every brick passed so far.  Every distance's loads are independent
  // of the others' outcome, so all are issued before the scan.
  uint32_t m = lower != nullptr ? lower[b] : kBrickRadiusCap;
  uint32_t r = 0;
  bool run = true;
#pragma unroll
  for (uint32_t k = 1; k <= kBrickRadiusCap; ++k) {
    const bool in = coord >= k && coord + k < extent;
    const size_t lo = in ? b - k * stride : b, hi = in ? b + k * stride : b;
    const uint32_t cl = brick_class[lo], ch = brick_class[hi];
    const uint32_t ml = lower != nullptr ? lower[lo] : kBrickRadiusCap;
    const uint32_t mh = lower != nullptr ? lower[hi] : kBrickRadiusCap;
    run = run && k <= m && in && cl == c && ch == c;
    if (run) m = min(m, min(ml, mh));
    run = run && !(m < k);
    if (run) r = k;
  }
  out[b] = static_cast<uint8_t>(r);
}

// ---- band integration (BandIntegrationSweep<kDevice>, tsdf_integration.cu:
// 240-291; TruncationBandWalk::visit_pixel, tsdf_integration.hpp:384-426) ----
// One thread per pixel walks its truncation band [d - band, d + band] along
// the pixel ray at half-block steps and marks every block a sample falls in
// (consecutive samples in one block mark it once).  The pixel table holds the
// depth that depth_in_range accepted (NaN otherwise; with finite, non-zero
// focal lengths the table's other NaN cause, an unusable ray, cannot occur).
__global__ void band_mark_kernel(const float4* __restrict__ table, uint32_t width, uint32_t height, Intr k,
                                 Rigid T, float trunc_base, float trunc_scale, int distance_scaled,
                                 VolumeDev v, const IcpState* __restrict__ state, uint32_t* __restrict__ bits) {
  if (state != nullptr) {
    if (state->failed) return;
    const float* w = state->world_to_camera;
    T = Rigid{{w[0], w[1], w[2]}, {w[3], w[4], w[5]}, {w[6], w[7], w[8]}, {w[9], w[10], w[11]}};
  }
  const uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t row = blockIdx.y * blockDim.y + threadIdx.y;
  if (col >= width || row >= height) return;
  const float measured = __ldg(&table[static_cast<size_t>(row) * width + col].x);
  if (isnan(measured)) return;
  // camera_to_world = inverse(world_to_camera) (vector.hpp:219-229)
  const f3 c0 = make(T.rx.x, T.ry.x, T.rz.x), c1 = make(T.rx.y, T.ry.y, T.rz.y), c2 = make(T.rx.z, T.ry.z, T.rz.z);
  const Rigid inv{c0, c1, c2, -make(dot(c0, T.t), dot(c1, T.t), dot(c2, T.t))};
  const float band = distance_scaled ? trunc_base + (trunc_scale * measured) : trunc_base;
  const float step = 0.5f * 8.0f * v.voxel_size;  // TruncationBandWalk::half_block_step
  const float inv_voxel = 1.0f / v.voxel_size;
  const int samples = static_cast<int>((2.0f * band) / step) + 1;
  uint32_t previous = 0xFFFFFFFFu;
  for (int i = 0; i <= samples; ++i) {
    const float depth = (measured - band) + (static_cast<float>(i) * step);
    const f3 world = apply(inv, back_project(k, static_cast<float>(col), static_cast<float>(row), depth));
    const f3 g = (world - v.origin) * inv_voxel;
    if (!(g.x >= 0.0f && g.y >= 0.0f && g.z >= 0.0f && g.x < static_cast<float>(v.rx) &&
          g.y < static_cast<float>(v.ry) && g.z < static_cast<float>(v.rz))) {
      continue;
    }
    const uint32_t block = ((static_cast<uint32_t>(g.z) >> 3) * v.by + (static_cast<uint32_t>(g.y) >> 3)) * v.bx +
                           (static_cast<uint32_t>(g.x) >> 3);
    if (block == previous) continue;
    previous = block;
    // lanes hitting the same word merge their bits into one atomic
    const uint32_t word = block >> 5, bit = 1u << (block & 31u);
    const unsigned peers = __match_any_sync(__activemask(), word);
    const uint32_t merged = __reduce_or_sync(peers, bit);
    if ((threadIdx.x + threadIdx.y * blockDim.x) % 32u == static_cast<unsigned>(__ffs(peers) - 1)) {
      atomicOr(bits + word, merged);
    }
  }
}

// Marked blocks into the work list (order does not matter: each listed block
// is fused once, independently of the others).
__global__ void band_compact_kernel(const uint32_t* __restrict__ bits, uint32_t words, uint32_t* __restrict__ list,
                                    unsigned* __restrict__ count, const IcpState* __restrict__ state) {
  if (state != nullptr && state->failed) return;
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= words) return;
  uint32_t word = bits[w];
  if (word == 0u) return;
  const unsigned base = atomicAdd(count, static_cast<unsigned>(__popc(word)));
  unsigned n = 0;
  while (word != 0u) {
    const uint32_t b = static_cast<uint32_t>(__ffs(word) - 1);
    word &= word - 1u;
    list[base + n++] = w * 32u + b;
  }
}

// ---- sparse allocation (BlockRep<kDevice>::integrate, block_rep.cu:100-152) ----
// The reference allocates marked blocks first come, first served (atomicAdd
// on the slot counter, block_rep.cu:18-41) into a dense grid of block slots.
// Here slots go to the newly marked blocks in block-index order (a scan over
// the marked words), so the allocation is deterministic, and each new block
// is inserted into the voxel-block hash with atomicCAS; as in the reference
// every attempt counts, a block past the capacity stays unallocated and its
// updates are dropped.
constexpr int kAllocWords = 1024;  // words per CTA of the allocation scan

// Marked blocks not allocated yet, and their count per word.
__global__ void sparse_new_kernel(const uint32_t* __restrict__ marked, const unsigned long long* __restrict__ table,
                                  uint32_t table_mask, uint32_t words, uint32_t* __restrict__ new_bits,
                                  uint32_t* __restrict__ counts, const IcpState* __restrict__ state) {
  if (state != nullptr && state->failed) return;
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= words) return;
  uint32_t m = marked[w], fresh = 0u;
  while (m != 0u) {
    const uint32_t b = static_cast<uint32_t>(__ffs(m) - 1);
    m &= m - 1u;
    if (block_table_lookup(table, table_mask, w * 32u + b) == kUnallocated) fresh |= 1u << b;
  }
  new_bits[w] = fresh;
  counts[w] = static_cast<uint32_t>(__popc(fresh));
}

// Exclusive scan of the counts within CTAs of kAllocWords words; CTA totals
// to `totals`.
__global__ void __launch_bounds__(kAllocWords)
    sparse_scan_local_kernel(uint32_t* __restrict__ counts, uint32_t words, uint32_t* __restrict__ totals,
                             const IcpState* __restrict__ state) {
  if (state != nullptr && state->failed) return;
  __shared__ uint32_t s_warp[kAllocWords / 32];
  const uint32_t w = blockIdx.x * kAllocWords + threadIdx.x;
  const uint32_t value = w < words ? counts[w] : 0u;
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t incl = value;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t up = __shfl_up_sync(0xFFFFFFFFu, incl, off);
    if (lane >= static_cast<unsigned>(off)) incl += up;
  }
  if (lane == 31u) s_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const uint32_t t = s_warp[lane];
    uint32_t x = t;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t up = __shfl_up_sync(0xFFFFFFFFu, x, off);
      if (lane >= static_cast<unsigned>(off)) x += up;
    }
    s_warp[lane] = x - t;  // exclusive warp offsets
    if (lane == 31u) totals[blockIdx.x] = x;
  }
  __syncthreads();
  if (w < words) counts[w] = s_warp[warp] + incl - value;  // exclusive prefix within the CTA
}

// One CTA: exclusive scan of the CTA totals, this frame's first slot, and
// the attempt counter moved past this frame's new blocks.
__global__ void __launch_bounds__(1024)
    sparse_scan_top_kernel(uint32_t* __restrict__ totals, uint32_t ctas, unsigned long long* __restrict__ allocated,
                           const IcpState* __restrict__ state) {
  if (state != nullptr && state->failed) return;
  __shared__ uint32_t s_warp[32];
  __shared__ unsigned long long s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  for (uint32_t first = 0; first < ctas; first += 1024) {
    const uint32_t i = first + threadIdx.x;
    const uint32_t value = i < ctas ? totals[i] : 0u;
    uint32_t incl = value;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t up = __shfl_up_sync(0xFFFFFFFFu, incl, off);
      if (lane >= static_cast<unsigned>(off)) incl += up;
    }
    if (lane == 31u) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const uint32_t t = s_warp[lane];
      uint32_t x = t;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const uint32_t up = __shfl_up_sync(0xFFFFFFFFu, x, off);
        if (lane >= static_cast<unsigned>(off)) x += up;
      }
      s_warp[lane] = x - t;
    }
    __syncthreads();
    const unsigned long long carry = s_carry;
    if (i < ctas) totals[i] = static_cast<uint32_t>(carry + s_warp[warp] + incl - value);
    __syncthreads();
    if (threadIdx.x == 1023) s_carry = carry + s_warp[31] + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    allocated[1] = allocated[0];
    allocated[0] += s_carry;
  }
}

// Slots for the new blocks of each word, then the frame's work list: every
// marked block that holds a slot.
__global__ void sparse_assign_kernel(const uint32_t* __restrict__ marked, const uint32_t* __restrict__ new_bits,
                                     const uint32_t* __restrict__ prefix, const uint32_t* __restrict__ cta_prefix,
                                     uint32_t words, const unsigned long long* __restrict__ allocated,
                                     unsigned long long capacity, unsigned long long* __restrict__ table,
                                     uint32_t table_mask, uint32_t* __restrict__ slot_block, uint32_t* __restrict__ list,
                                     unsigned* __restrict__ count, uint8_t* __restrict__ null_bricks, uint32_t bx,
                                     uint32_t by, uint32_t bz, const IcpState* __restrict__ state) {
  if (state != nullptr && state->failed) return;
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= words) return;
  const uint32_t fresh_bits = new_bits[w];
  uint32_t fresh = fresh_bits, granted = 0u;
  unsigned long long slot = allocated[1] + cta_prefix[w / kAllocWords] + prefix[w];
  while (fresh != 0u) {
    const uint32_t b = static_cast<uint32_t>(__ffs(fresh) - 1);
    fresh &= fresh - 1u;
    if (slot < capacity) {
      const uint32_t block = w * 32u + b;
      // insert (block, slot): the first empty entry of the block's probe
      // sequence (the table is at most half full)
      const unsigned long long entry = (static_cast<unsigned long long>(block) << 32) | slot;
      uint32_t h = block_hash(block) & table_mask;
      for (uint32_t probe = 0; probe <= table_mask; ++probe) {
        const unsigned long long prev = atomicCAS(table + h, kEmptyEntry, entry);
        if (prev == kEmptyEntry || prev == entry) break;
        h = (h + 1u) & table_mask;
      }
      granted |= 1u << b;
      slot_block[slot] = block;
      // the stencils that can reach this block are no longer all nullopt
      const int x = static_cast<int>(block % bx), y = static_cast<int>((block / bx) % by),
                z = static_cast<int>(block / (bx * by));
      for (int d = 0; d < 8; ++d) {
        const int nx = x - (d & 1), ny = y - ((d >> 1) & 1), nz = z - (d >> 2);
        if (nx >= 0 && ny >= 0 && nz >= 0) {
          null_bricks[(static_cast<size_t>(nz) * by + static_cast<uint32_t>(ny)) * bx + static_cast<uint32_t>(nx)] = 0;
        }
      }
    }
    ++slot;
  }
  // the marked blocks allocated before this frame, and the new ones granted a slot
  uint32_t usable = (marked[w] & ~fresh_bits) | granted;
  if (usable == 0u) return;
  const unsigned base = atomicAdd(count, static_cast<unsigned>(__popc(usable)));
  unsigned n = 0;
  while (usable != 0u) {
    const uint32_t b = static_cast<uint32_t>(__ffs(usable) - 1);
    usable &= usable - 1u;
    list[base + n++] = w * 32u + b;
  }
}

template <int Kind>
__global__ void fill_kernel(void* voxels, float4* colors, size_t count) {
  using VT = VoxelTraits<Kind>;
  auto* out = reinterpret_cast<typename VT::Raw*>(voxels);
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride) {
    out[i] = VT::unobserved();
    if (colors != nullptr) colors[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
}

template <int Kind>
__global__ void count_observed_kernel(const void* voxels, size_t count, unsigned long long* result) {
  using VT = VoxelTraits<Kind>;
  const auto* in = reinterpret_cast<const typename VT::Raw*>(voxels);
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  unsigned long long local = 0;
  for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride) {
    local += VT::weight(in[i]) > 0.0f ? 1u : 0u;
  }
  for (int off = 16; off > 0; off >>= 1) local += __shfl_xor_sync(0xFFFFFFFFu, local, off);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(result, local);
}

TileLevels tile_levels_of(const Pipeline& p) {
  TileLevels lv;
  lv.count = p.tile_levels;
  for (uint32_t l = 0; l < 12; ++l) {
    lv.w[l] = p.tile_w[l];
    lv.h[l] = p.tile_h[l];
    lv.off[l] = p.tile_off[l];
  }
  return lv;
}

template <int Kind, bool Color>
void launch_blocks_typed(Pipeline& p, const float4* table, uint32_t width, uint32_t height, Intr k, Rigid T,
                         const IntegParams& ip, const IcpState* state, cudaStream_t s) {
  if (state == nullptr && p.kernel_start != nullptr) check(cudaEventRecord(p.kernel_start, s), "event record");
  integrate_blocks_kernel<Kind, Color><<<p.integrate_ctas, kBlockThreads, 0, s>>>(
      p.view, table, width, height, k, T, ip, state, p.block_list.ptr, p.block_count.ptr,
      p.voxel_bits.count ? p.voxel_bits.ptr : nullptr, p.brick_dirty.ptr, p.counters.ptr);
  check(cudaGetLastError(), "integrate_blocks_kernel launch");
  if (state == nullptr && p.kernel_stop != nullptr) check(cudaEventRecord(p.kernel_stop, s), "event record");
}

}  // namespace

void prepare_blocks(Pipeline& p, uint32_t width, uint32_t height, cudaStream_t s) {
  const uint32_t blocks = p.view.bx * p.view.by * p.view.bz;
  const size_t words = (blocks + 31) / 32;
  if (p.brick_dirty.count != words) {
    p.block_list.resize(blocks);
    p.block_count.resize(1);
    p.brick_dirty.resize(words);
    p.band_bits.resize(words);
    if (p.view.table == nullptr) {
      // the raycast's skip structures (dense storage only)
      p.voxel_bits.resize(static_cast<size_t>(blocks) * 32u);
      p.stencil_bits.resize(static_cast<size_t>(blocks) * 32u);
      p.brick_class.resize(blocks);
      p.brick_radius.resize(blocks);
      p.radius_scratch.resize(2 * static_cast<size_t>(blocks));
    } else {
      p.new_bits.resize(words);
      p.word_prefix.resize(words);
      p.cta_prefix.resize(ceil_div(static_cast<unsigned>(words), 1024u));
    }
    reset_blocks(p, s);
  }
  // depth-tile pyramid geometry for this frame size
  uint32_t w = ceil_div(width, kTile), h = ceil_div(height, kTile), off = 0, l = 0;
  if (p.tile_levels == 0 || p.tile_w[0] != w || p.tile_h[0] != h) {
    while (true) {
      p.tile_w[l] = w;
      p.tile_h[l] = h;
      p.tile_off[l] = off;
      off += w * h;
      ++l;
      if ((w == 1 && h == 1) || l == 12) break;
      w = (w + 1) / 2;
      h = (h + 1) / 2;
    }
    p.tile_levels = l;
    p.depth_tiles.resize(off);
  }
}

void reset_blocks(Pipeline& p, cudaStream_t s) {
  if (p.brick_dirty.count == 0) return;
  check(cudaMemsetAsync(p.brick_dirty.ptr, 0, p.brick_dirty.bytes(), s), "skip bits reset");
  if (p.voxel_bits.count == 0) return;
  // nothing observed: every stencil is decided nullopt
  check(cudaMemsetAsync(p.voxel_bits.ptr, 0, p.voxel_bits.bytes(), s), "skip bits reset");
  check(cudaMemsetAsync(p.stencil_bits.ptr, 0, p.stencil_bits.bytes(), s), "skip bits reset");
  check(cudaMemsetAsync(p.brick_class.ptr, 1, p.brick_class.bytes(), s), "skip bits reset");
  check(cudaMemsetAsync(p.brick_radius.ptr, 0, p.brick_radius.bytes(), s), "skip bits reset");
}

void reset_sparse(Pipeline& p, cudaStream_t s) {
  if (p.block_table.count == 0) return;
  check(cudaMemsetAsync(p.block_table.ptr, 0xFF, p.block_table.bytes(), s), "block table reset");  // kEmptyEntry
  check(cudaMemsetAsync(p.null_bricks.ptr, 1, p.null_bricks.bytes(), s), "sparse null bricks reset");
  check(cudaMemsetAsync(p.allocated.ptr, 0, p.allocated.bytes(), s), "sparse counter reset");
}

void launch_pixel_table(const uint16_t* depth, const uint32_t* color, const float* normals, uint32_t width,
                        uint32_t height, Intr k, const kf_integration_options& o, int rule, float4* table,
                        cudaStream_t s) {
  const dim3 block(32, 8);
  const dim3 grid(ceil_div(width, 32), ceil_div(height, 8));
  pixel_table_kernel<<<grid, block, 0, s>>>(depth, color, normals, width, height, k, o.depth_scale, o.min_depth,
                                            o.max_depth, o.observation_weight, rule == KF_RULE_ANGLE_WEIGHTED,
                                            table);
  check(cudaGetLastError(), "pixel_table_kernel launch");
}

void launch_integrate_inputs(Pipeline& p, const float4* table, uint32_t width, uint32_t height, cudaStream_t s) {
  prepare_blocks(p, width, height, s);
  if (p.config.integration.mode == KF_INTEGRATION_BAND) return;
  // depth-tile pyramid
  const TileLevels lv = tile_levels_of(p);
  tile_max_kernel<<<dim3(ceil_div(lv.w[0], 16), ceil_div(lv.h[0], 16)), dim3(16, 16), 0, s>>>(
      table, width, height, lv.w[0], lv.h[0], p.depth_tiles.ptr);
  check(cudaGetLastError(), "tile_max_kernel launch");
  tile_pyramid_kernel<<<1, 1024, 0, s>>>(p.depth_tiles.ptr, lv);
  check(cudaGetLastError(), "tile_pyramid_kernel launch");
}

void launch_integrate(Pipeline& p, const float4* table, uint32_t width, uint32_t height, Intr k, Rigid T,
                      int has_color, const IcpState* state, cudaStream_t s, bool inputs_ready) {
  prepare_blocks(p, width, height, s);
  const kf_integration_options& o = p.config.integration;
  const uint32_t blocks = p.view.bx * p.view.by * p.view.bz;
  check(cudaMemsetAsync(p.block_count.ptr, 0, sizeof(unsigned), s), "block count clear");
  check(cudaMemsetAsync(p.brick_dirty.ptr, 0, p.brick_dirty.bytes(), s), "dirty bits clear");
  if (o.mode == KF_INTEGRATION_BAND) {
    // blocks the pixels' truncation bands cross
    check(cudaMemsetAsync(p.band_bits.ptr, 0, p.band_bits.bytes(), s), "band bits clear");
    band_mark_kernel<<<dim3(ceil_div(width, 16), ceil_div(height, 16)), dim3(16, 16), 0, s>>>(
        table, width, height, k, T, p.view.truncation, o.truncation_distance_scale, o.distance_scaled_truncation,
        p.view, state, p.band_bits.ptr);
    check(cudaGetLastError(), "band_mark_kernel launch");
    const uint32_t words = static_cast<uint32_t>(p.band_bits.count);
    if (p.view.table != nullptr) {
      // sparse: allocate the newly marked blocks, list the allocated ones
      const uint32_t ctas = ceil_div(words, static_cast<uint32_t>(kAllocWords));
      sparse_new_kernel<<<ceil_div(words, 256), 256, 0, s>>>(p.band_bits.ptr, p.block_table.ptr, p.view.table_mask,
                                                             words, p.new_bits.ptr, p.word_prefix.ptr, state);
      check(cudaGetLastError(), "sparse_new_kernel launch");
      sparse_scan_local_kernel<<<ctas, kAllocWords, 0, s>>>(p.word_prefix.ptr, words, p.cta_prefix.ptr, state);
      check(cudaGetLastError(), "sparse_scan_local_kernel launch");
      sparse_scan_top_kernel<<<1, 1024, 0, s>>>(p.cta_prefix.ptr, ctas, p.allocated.ptr, state);
      check(cudaGetLastError(), "sparse_scan_top_kernel launch");
      sparse_assign_kernel<<<ceil_div(words, 256), 256, 0, s>>>(
          p.band_bits.ptr, p.new_bits.ptr, p.word_prefix.ptr, p.cta_prefix.ptr, words, p.allocated.ptr,
          p.sparse_capacity, p.block_table.ptr, p.view.table_mask, p.slot_block.ptr, p.block_list.ptr,
          p.block_count.ptr, p.null_bricks.ptr,
          p.view.bx, p.view.by, p.view.bz, state);
      check(cudaGetLastError(), "sparse_assign_kernel launch");
    } else {
      band_compact_kernel<<<ceil_div(words, 256), 256, 0, s>>>(p.band_bits.ptr, words, p.block_list.ptr,
                                                               p.block_count.ptr, state);
      check(cudaGetLastError(), "band_compact_kernel launch");
    }
  } else {
    if (!inputs_ready) launch_integrate_inputs(p, table, width, height, s);
    const TileLevels lv = tile_levels_of(p);
    // block culling
    CullParams cp;
    cp.trunc_base = p.view.truncation;
    cp.trunc_scale = o.truncation_distance_scale;
    cp.distance_scaled = o.distance_scaled_truncation;
    cp.slack = 1.0f / (1.0f - 2.0f / fminf(k.fx, k.fy));
    cp.width = width;
    cp.height = height;
    cull_blocks_kernel<<<ceil_div(blocks, 256), 256, 0, s>>>(p.view, T, k, p.depth_tiles.ptr, lv, cp, state,
                                                             p.block_list.ptr, p.block_count.ptr);
    check(cudaGetLastError(), "cull_blocks_kernel launch");
  }
  // listed blocks
  IntegParams ip;
  ip.max_weight = o.max_weight;
  ip.projective_distance = o.projective_distance;
  ip.distance_scaled_truncation = o.distance_scaled_truncation;
  ip.truncation_distance_scale = o.truncation_distance_scale;
  ip.has_color = has_color;
  const bool color = p.config.color == KF_COLOR_FLOAT;
  switch (p.config.voxel) {
    case KF_VOXEL_QUANTIZED:
      color ? launch_blocks_typed<KF_VOXEL_QUANTIZED, true>(p, table, width, height, k, T, ip, state, s)
            : launch_blocks_typed<KF_VOXEL_QUANTIZED, false>(p, table, width, height, k, T, ip, state, s);
      break;
    case KF_VOXEL_BF16:
      color ? launch_blocks_typed<KF_VOXEL_BF16, true>(p, table, width, height, k, T, ip, state, s)
            : launch_blocks_typed<KF_VOXEL_BF16, false>(p, table, width, height, k, T, ip, state, s);
      break;
    default:
      color ? launch_blocks_typed<KF_VOXEL_FLOAT, true>(p, table, width, height, k, T, ip, state, s)
            : launch_blocks_typed<KF_VOXEL_FLOAT, false>(p, table, width, height, k, T, ip, state, s);
      break;
  }
  // the band-march bitmap (EmptySpaceIndex::rebuild after integration)
  launch_band_rebuild(p, s);
  // raycast skip bits
  if (p.voxel_bits.count == 0) return;
  stencil_bits_kernel<<<ceil_div(blocks * 8u, 256), 256, 0, s>>>(
      reinterpret_cast<const uint4*>(p.voxel_bits.ptr), reinterpret_cast<uint4*>(p.stencil_bits.ptr),
      p.brick_class.ptr, p.brick_dirty.ptr, p.view.bx, p.view.by, p.view.bz, p.config.raycast.corner_policy == KF_CORNERS_REQUIRE_ALL,
      state);
  check(cudaGetLastError(), "stencil_bits_kernel launch");
  const uint32_t bricks = static_cast<uint32_t>(p.brick_radius.count);
  uint8_t* run_x = p.radius_scratch.ptr;
  uint8_t* square_xy = p.radius_scratch.ptr + bricks;
  brick_radius_kernel<<<ceil_div(bricks, 256u), 256, 0, s>>>(p.brick_class.ptr, nullptr, run_x, p.view.bx, p.view.by,
                                                              p.view.bz, 0, state);
  brick_radius_kernel<<<ceil_div(bricks, 256u), 256, 0, s>>>(p.brick_class.ptr, run_x, square_xy, p.view.bx,
                                                              p.view.by, p.view.bz, 1, state);
  brick_radius_kernel<<<ceil_div(bricks, 256u), 256, 0, s>>>(p.brick_class.ptr, square_xy, p.brick_radius.ptr,
                                                              p.view.bx, p.view.by, p.view.bz, 2, state);
  check(cudaGetLastError(), "brick_radius_kernel launch");
}

void launch_fill_volume(Pipeline& p, cudaStream_t s) {
  const unsigned grid = 148 * 8;
  float4* colors = p.config.color == KF_COLOR_FLOAT ? p.colors.ptr : nullptr;
  switch (p.config.voxel) {
    case KF_VOXEL_QUANTIZED:
      fill_kernel<KF_VOXEL_QUANTIZED><<<grid, 256, 0, s>>>(p.voxels.ptr, colors, p.voxel_count);
      break;
    case KF_VOXEL_BF16:
      fill_kernel<KF_VOXEL_BF16><<<grid, 256, 0, s>>>(p.voxels.ptr, colors, p.voxel_count);
      break;
    default:
      fill_kernel<KF_VOXEL_FLOAT><<<grid, 256, 0, s>>>(p.voxels.ptr, colors, p.voxel_count);
      break;
  }
  check(cudaGetLastError(), "fill_kernel launch");
  reset_blocks(p, s);
}

uint64_t count_observed(Pipeline& p) {
  DeviceArray<unsigned long long> result(1);
  check(cudaMemsetAsync(result.ptr, 0, sizeof(unsigned long long), p.stream), "count clear");
  const unsigned grid = 148 * 8;
  switch (p.config.voxel) {
    case KF_VOXEL_QUANTIZED:
      count_observed_kernel<KF_VOXEL_QUANTIZED><<<grid, 256, 0, p.stream>>>(p.voxels.ptr, p.voxel_count, result.ptr);
      break;
    case KF_VOXEL_BF16:
      count_observed_kernel<KF_VOXEL_BF16><<<grid, 256, 0, p.stream>>>(p.voxels.ptr, p.voxel_count, result.ptr);
      break;
    default:
      count_observed_kernel<KF_VOXEL_FLOAT><<<grid, 256, 0, p.stream>>>(p.voxels.ptr, p.voxel_count, result.ptr);
      break;
  }
  check(cudaGetLastError(), "count_observed_kernel launch");
  unsigned long long host = 0;
  check(cudaMemcpyAsync(&host, result.ptr, sizeof(host), cudaMemcpyDeviceToHost, p.stream), "count download");
  check(cudaStreamSynchronize(p.stream), "count observed");
  return host;
}

}  // namespace kf
