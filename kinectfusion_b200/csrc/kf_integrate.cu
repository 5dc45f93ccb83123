// kf_integrate.cu - projective TSDF integration into a dense volume
// (IntegrationContext::observe/fuse + ClassicTsdf/AngleWeightedTsdf,
// tsdf_integration.hpp:127-342; reference device sweep tsdf_integration.cu:61-107).
//
// Design:
//  * A per-frame pixel table (one float4 per depth pixel: depth in metres or
//    NaN, |K^-1 [u v 1]|, the rule's observation weight, RGBA8 colour) holds
//    everything of observe() that depends on the pixel only.  It is the same
//    float expression as the per-voxel host code, evaluated once per pixel.
//  * One thread per (x, y) column of voxels streams z.  The world point's x/y
//    part of each row of world_to_camera is constant along a column and is
//    hoisted; the per-voxel remainder is the host expression verbatim.
//  * Each column's z range is clipped to the camera frustum with a one-voxel
//    and two-pixel margin (conservative: a skipped voxel provably projects
//    outside the image or behind the camera); inside it every voxel runs the
//    exact host test, so results are bit-identical to the host sweep.
//  * Voxels are read and written with one 8-byte (float) or 4-byte
//    (int16/bf16) access each, coalesced along x across the warp.
#include <algorithm>
#include <cmath>

#include "kf_internal.h"

namespace kf {
namespace {

struct IntegParams {
  float observation_weight_unused;
  float max_weight;
  int projective_distance;
  int distance_scaled_truncation;
  float truncation_distance_scale;
  int has_color;
};

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

// Conservative z interval [lo, hi] (in voxel steps) of a column whose camera
// point is affine in z: P(z) = a + b z.  Keeps every z where P.z > 0 and the
// projection may land inside the image (two-pixel margin).
__device__ __forceinline__ bool column_range(f3 a, f3 b, const Intr& k, float width, float height,
                                             float zmax, float& lo, float& hi) {
  lo = 0.0f;
  hi = zmax;
  // constraint alpha + beta z > 0
  auto clip = [&](float alpha, float beta) {
    if (fabsf(beta) < 1e-20f) {
      if (!(alpha > -1e-6f)) {
        lo = 1.0f;
        hi = 0.0f;
      }
      return;
    }
    const float root = -alpha / beta;
    if (beta > 0.0f) {
      lo = fmaxf(lo, root);
    } else {
      hi = fminf(hi, root);
    }
  };
  // depth in front of the camera plane
  clip(a.z, b.z);
  const float m = 2.0f;
  // fx x + (cx - (-0.5 - m)) z > 0   (left edge)
  clip(k.fx * a.x + (k.cx + 0.5f + m) * a.z, k.fx * b.x + (k.cx + 0.5f + m) * b.z);
  // (W - 0.5 + m - cx) z - fx x > 0  (right edge)
  clip((width - 0.5f + m - k.cx) * a.z - k.fx * a.x, (width - 0.5f + m - k.cx) * b.z - k.fx * b.x);
  clip(k.fy * a.y + (k.cy + 0.5f + m) * a.z, k.fy * b.y + (k.cy + 0.5f + m) * b.z);
  clip((height - 0.5f + m - k.cy) * a.z - k.fy * a.y, (height - 0.5f + m - k.cy) * b.z - k.fy * b.y);
  lo = floorf(lo) - 1.0f;
  hi = ceilf(hi) + 1.0f;
  lo = fmaxf(lo, 0.0f);
  hi = fminf(hi, zmax);
  return lo <= hi;
}

template <int Kind, bool Color>
__global__ void __launch_bounds__(256)
    integrate_kernel(VolumeDev v, const float4* __restrict__ table, uint32_t width, uint32_t height,
                     Intr k, Rigid T, IntegParams ip, const IcpState* __restrict__ state,
                     unsigned long long* __restrict__ counters) {
  using VT = VoxelTraits<Kind>;
  using Raw = typename VT::Raw;
  if (state != nullptr) {
    if (state->failed) return;
    const float* w = state->world_to_camera;
    T = Rigid{{w[0], w[1], w[2]}, {w[3], w[4], w[5]}, {w[6], w[7], w[8]}, {w[9], w[10], w[11]}};
  }
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= v.rx || y >= v.ry) return;

  // World x/y of the column and the hoisted first two terms of each dot
  // product: dot(row, p) = (row.x * p.x + row.y * p.y) + row.z * p.z.
  const float wx = v.origin.x + ((static_cast<float>(x) + 0.5f) * v.voxel_size);
  const float wy = v.origin.y + ((static_cast<float>(y) + 0.5f) * v.voxel_size);
  const float hx = (T.rx.x * wx) + (T.rx.y * wy);
  const float hy = (T.ry.x * wx) + (T.ry.y * wy);
  const float hz = (T.rz.x * wx) + (T.rz.y * wy);

  // Affine model of the camera point along z for the frustum clip.
  const float w0 = v.origin.z + (0.5f * v.voxel_size);
  const f3 a = make((hx + T.rx.z * w0) + T.t.x, (hy + T.ry.z * w0) + T.t.y, (hz + T.rz.z * w0) + T.t.z);
  const f3 b = make(T.rx.z * v.voxel_size, T.ry.z * v.voxel_size, T.rz.z * v.voxel_size);
  float lo, hi;
  const bool visible = column_range(a, b, k, static_cast<float>(width), static_cast<float>(height),
                                    static_cast<float>(v.rz - 1), lo, hi);
  const uint32_t z_first = visible ? static_cast<uint32_t>(lo) : 1u;
  const uint32_t z_last = visible ? static_cast<uint32_t>(hi) : 0u;
  unsigned updates = 0, color_updates = 0;

  Raw* __restrict__ voxels = reinterpret_cast<Raw*>(v.voxels);
  const size_t column = static_cast<size_t>(y) * v.rx + x;
  const size_t slice = static_cast<size_t>(v.rx) * v.ry;
  const float trunc_base = v.truncation;

  for (uint32_t z = z_first; z <= z_last; ++z) {
    const float wz = v.origin.z + ((static_cast<float>(z) + 0.5f) * v.voxel_size);
    const f3 cp = make((hx + (T.rx.z * wz)) + T.t.x, (hy + (T.ry.z * wz)) + T.t.y,
                       (hz + (T.rz.z * wz)) + T.t.z);
    if (cp.z <= 0.0f) continue;
    float px, py;
    project(k, cp, px, py);
    const long rx = lroundf(px);
    const long ry = lroundf(py);
    if (rx < 0 || ry < 0 || rx >= static_cast<long>(width) || ry >= static_cast<long>(height)) continue;
    const float4 tb = __ldg(table + (static_cast<size_t>(ry) * width + static_cast<size_t>(rx)));
    const float sd = tb.x;
    if (isnan(sd)) continue;
    const float truncation =
        ip.distance_scaled_truncation ? trunc_base + (ip.truncation_distance_scale * sd) : trunc_base;
    const float sdf = ip.projective_distance ? sd - (norm(cp) / tb.y) : sd - cp.z;
    if (sdf < -truncation) continue;
    const float tsdf = clampf(sdf / truncation, -1.0f, 1.0f);
    const float ow = tb.z;
    if (ow <= 0.0f) continue;
    // BasicVoxel::fused (volume.hpp:137-146)
    const size_t index = static_cast<size_t>(z) * slice + column;
    const Raw old = voxels[index];
    const float t0 = VT::tsdf(old);
    const float w0v = VT::weight(old);
    const float avg = ((t0 * w0v) + (tsdf * ow)) / (w0v + ow);
    const float sum_w = w0v + ow;
    voxels[index] = VT::encode(avg, ip.max_weight < sum_w ? ip.max_weight : sum_w);
    ++updates;
    if constexpr (Color) {
      if (ip.has_color && sdf <= truncation * 0.5f) {
        ++color_updates;
        // ColorVoxel::fused (volume.hpp:160-170)
        const float4 cv = v.colors[index];
        const f3 c = color_from_pixel(__float_as_uint(tb.w));
        const f3 avgc = ((make(cv.x, cv.y, cv.z) * cv.w) + (c * ow)) / (cv.w + ow);
        const float cw = cv.w + ow;
        v.colors[index] = make_float4(avgc.x, avgc.y, avgc.z, ip.max_weight < cw ? ip.max_weight : cw);
      }
    }
  }
  // One atomic per warp for the voxel-update counters.
  const unsigned mask = __activemask();
  const unsigned total = __reduce_add_sync(mask, updates);
  const unsigned total_color = __reduce_add_sync(mask, color_updates);
  if ((threadIdx.x & 31u) == static_cast<unsigned>(__ffs(mask) - 1) && counters != nullptr) {
    if (total) atomicAdd(counters, static_cast<unsigned long long>(total));
    if (total_color) atomicAdd(counters + 1, static_cast<unsigned long long>(total_color));
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

template <int Kind, bool Color>
void launch_integrate_typed(Pipeline& p, const float4* table, uint32_t width, uint32_t height, Intr k,
                            Rigid T, int has_color, const IcpState* state, cudaStream_t s) {
  const kf_integration_options& o = p.config.integration;
  IntegParams ip;
  ip.observation_weight_unused = o.observation_weight;
  ip.max_weight = o.max_weight;
  ip.projective_distance = o.projective_distance;
  ip.distance_scaled_truncation = o.distance_scaled_truncation;
  ip.truncation_distance_scale = o.truncation_distance_scale;
  ip.has_color = has_color;
  const dim3 block(32, 8);
  const dim3 grid(ceil_div(p.view.rx, 32), ceil_div(p.view.ry, 8));
  if (state == nullptr && p.kernel_start != nullptr) check(cudaEventRecord(p.kernel_start, s), "event record");
  integrate_kernel<Kind, Color><<<grid, block, 0, s>>>(p.view, table, width, height, k, T, ip, state,
                                                       p.counters.ptr);
  check(cudaGetLastError(), "integrate_kernel launch");
  if (state == nullptr && p.kernel_stop != nullptr) check(cudaEventRecord(p.kernel_stop, s), "event record");
}

}  // namespace

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

void launch_integrate(Pipeline& p, const float4* table, uint32_t width, uint32_t height, Intr k, Rigid T,
                      int has_color, const IcpState* state, cudaStream_t s) {
  const bool color = p.config.color == KF_COLOR_FLOAT;
  switch (p.config.voxel) {
    case KF_VOXEL_QUANTIZED:
      color ? launch_integrate_typed<KF_VOXEL_QUANTIZED, true>(p, table, width, height, k, T, has_color, state, s)
            : launch_integrate_typed<KF_VOXEL_QUANTIZED, false>(p, table, width, height, k, T, has_color, state, s);
      break;
    case KF_VOXEL_BF16:
      color ? launch_integrate_typed<KF_VOXEL_BF16, true>(p, table, width, height, k, T, has_color, state, s)
            : launch_integrate_typed<KF_VOXEL_BF16, false>(p, table, width, height, k, T, has_color, state, s);
      break;
    default:
      color ? launch_integrate_typed<KF_VOXEL_FLOAT, true>(p, table, width, height, k, T, has_color, state, s)
            : launch_integrate_typed<KF_VOXEL_FLOAT, false>(p, table, width, height, k, T, has_color, state, s);
      break;
  }
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
