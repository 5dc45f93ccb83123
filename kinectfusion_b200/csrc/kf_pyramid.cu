// kf_pyramid.cu - bilateral filter, 2x2 downsample and vertex/normal maps of
// the depth pyramid (depth_processing.hpp:54-284, depth_processing.cu:70-122).
//
// Two kernels per frame: the bilateral filter (level 0), then one fused
// kernel per level that writes the vertex map, the normal map and, for every
// pixel of the next level, its 2x2 downsample.  Normals recompute the four
// neighbour vertices from the depth image instead of re-reading the vertex
// map, which keeps one level in one launch; the recomputation is the same
// float expression, so the values are identical.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "kf_internal.h"

namespace kf {
namespace {

struct DepthParams {
  float depth_scale, min_depth, max_depth;
  float max_normal_depth_jump, max_downsample_depth_jump;
  int radius;
  float spatial_scale, range_scale;
};

DepthParams depth_params(const kf_depth_options& o) {
  DepthParams p;
  p.depth_scale = o.depth_scale;
  p.min_depth = o.min_depth;
  p.max_depth = o.max_depth;
  p.max_normal_depth_jump = o.max_normal_depth_jump;
  p.max_downsample_depth_jump = o.max_downsample_depth_jump;
  p.radius = o.bilateral_radius;
  // gaussian_exponent_scale (depth_processing.hpp:118-121)
  p.spatial_scale = -0.5f / (o.bilateral_spatial_sigma * o.bilateral_spatial_sigma);
  p.range_scale = -0.5f / (o.bilateral_depth_sigma * o.bilateral_depth_sigma);
  return p;
}

constexpr int kTileX = 32;
constexpr int kTileY = 8;

// BilateralFilter::operator() (depth_processing.hpp:71-115).  The Gaussian is
// exp evaluated in double and rounded once to float: the correctly rounded
// value of the float exponent, which the CPU oracle computes the same way.
__global__ void __launch_bounds__(kTileX* kTileY)
    bilateral_kernel(const uint16_t* __restrict__ in, uint16_t* __restrict__ out, int width,
                     int height, DepthParams p) {
  const int col = blockIdx.x * kTileX + threadIdx.x;
  const int row = blockIdx.y * kTileY + threadIdx.y;
  if (col >= width || row >= height) return;
  float center;
  uint16_t result = 0;
  if (depth_in_range(__ldg(in + row * width + col), p.depth_scale, p.min_depth, p.max_depth, center)) {
    const int x_begin = max(col - p.radius, 0);
    const int y_begin = max(row - p.radius, 0);
    const int x_end = min(col + p.radius, width - 1);
    const int y_end = min(row + p.radius, height - 1);
    float weighted_sum = 0.0f;
    float weight_sum = 0.0f;
    for (int y = y_begin; y <= y_end; ++y) {
      for (int x = x_begin; x <= x_end; ++x) {
        const uint16_t raw = __ldg(in + y * width + x);
        float sample;
        if (!depth_in_range(raw, p.depth_scale, p.min_depth, p.max_depth, sample)) continue;
        const float d2 = static_cast<float>(((x - col) * (x - col)) + ((y - row) * (y - row)));
        const float dd = sample - center;
        const float arg = (d2 * p.spatial_scale) + (dd * dd * p.range_scale);
        const float weight = static_cast<float>(exp(static_cast<double>(arg)));
        weighted_sum += weight * static_cast<float>(raw);
        weight_sum += weight;
      }
    }
    if (weight_sum > 0.0f) {
      result = static_cast<uint16_t>(lroundf(weighted_sum / weight_sum));
    }
  }
  out[row * width + col] = result;
}

// VertexProjection::operator() (depth_processing.hpp:215-226), identity pose.
__device__ __forceinline__ f3 vertex_at(const uint16_t* __restrict__ depth, int width, int x, int y,
                                        const Intr& k, const DepthParams& p) {
  float d;
  if (!depth_in_range(__ldg(depth + y * width + x), p.depth_scale, p.min_depth, p.max_depth, d)) {
    return nan3();
  }
  return back_project(k, static_cast<float>(x), static_cast<float>(y), d);
}

// One level: vertex + NormalEstimation (depth_processing.hpp:251-279) +
// BlockDownsample into the next level (depth_processing.hpp:153-187).
__global__ void __launch_bounds__(kTileX* kTileY)
    level_kernel(const uint16_t* __restrict__ depth, int width, int height, Intr k, DepthParams p,
                 float* __restrict__ vertices, float* __restrict__ normals,
                 uint16_t* __restrict__ next) {
  const int col = blockIdx.x * kTileX + threadIdx.x;
  const int row = blockIdx.y * kTileY + threadIdx.y;
  if (col >= width || row >= height) return;
  const f3 c = vertex_at(depth, width, col, row, k, p);
  const size_t pix = static_cast<size_t>(row) * width + col;
  store3(vertices + pix * 3, c);

  f3 n = nan3();
  if (col != 0 && row != 0 && col + 1 < width && row + 1 < height) {
    const f3 l = vertex_at(depth, width, col - 1, row, k, p);
    const f3 r = vertex_at(depth, width, col + 1, row, k, p);
    const f3 t = vertex_at(depth, width, col, row - 1, k, p);
    const f3 b = vertex_at(depth, width, col, row + 1, k, p);
    if (finite3((((c + l) + r) + t) + b) &&
        !(fabsf(r.z - l.z) > p.max_normal_depth_jump || fabsf(b.z - t.z) > p.max_normal_depth_jump)) {
      const f3 nn = cross(b - t, r - l);
      const float length = norm(nn);
      if (length > 0.0f) n = nn / length;
    }
  }
  store3(normals + pix * 3, n);

  if (next != nullptr) {
    const int nw = width / 2, nh = height / 2;
    if (col < nw && row < nh) {
      uint32_t sum = 0, count = 0;
      uint16_t lo = 0xFFFF, hi = 0;
#pragma unroll
      for (int dy = 0; dy < 2; ++dy) {
#pragma unroll
        for (int dx = 0; dx < 2; ++dx) {
          const uint16_t s = __ldg(depth + (row * 2 + dy) * width + (col * 2 + dx));
          if (s == 0) continue;
          sum += s;
          ++count;
          lo = s < lo ? s : lo;
          hi = hi < s ? s : hi;
        }
      }
      uint16_t result = 0;
      if (count != 0) {
        const float max_m = static_cast<float>(hi) / p.depth_scale;
        const float min_m = static_cast<float>(lo) / p.depth_scale;
        if (!(max_m - min_m > p.max_downsample_depth_jump)) {
          result = static_cast<uint16_t>((sum + (count / 2u)) / count);
        }
      }
      next[row * nw + col] = result;
    }
  }
}

kf_intrinsics scaled(kf_intrinsics k, uint32_t level) {
  // CameraIntrinsics::scaled (rgbd.hpp:66-70)
  const float s = 1.0f / static_cast<float>(1u << level);
  return kf_intrinsics{k.fx * s, k.fy * s, k.cx * s, k.cy * s};
}

void validate(const kf_depth_options& o) {
  // DepthProcessingOptions::validated (depth_processing.cpp:74-94)
  require(o.levels > 0u, "Depth pyramid must have at least one level");
  require(o.levels <= 4u, "Depth pyramid supports at most 4 levels");
  require(o.depth_scale > 0.0f, "Depth scale must be positive");
  require(o.min_depth >= 0.0f && o.max_depth > o.min_depth, "Depth range is invalid");
  require(o.max_normal_depth_jump >= 0.0f, "Normal depth jump threshold must be non-negative");
  require(o.max_downsample_depth_jump >= 0.0f, "Downsample depth jump threshold must be non-negative");
  require(o.bilateral_radius >= 0, "Bilateral filter radius must be non-negative");
  require(o.bilateral_spatial_sigma > 0.0f, "Bilateral spatial sigma must be positive");
  require(o.bilateral_depth_sigma > 0.0f, "Bilateral depth sigma must be positive");
}

}  // namespace

uint32_t Pyramid::prepare(uint32_t w, uint32_t h, kf_intrinsics k) {
  require(w > 0 && h > 0, "Depth image must be non-empty");
  if (raw.count != static_cast<size_t>(w) * h) raw.resize(static_cast<size_t>(w) * h);
  width = w;
  height = h;
  intrinsics = k;
  if (levels.size() < options.levels) levels.resize(options.levels);
  uint32_t lw = w, lh = h, count = 0;
  for (uint32_t level = 0; level < options.levels; ++level) {
    if (lw == 0 || lh == 0) break;
    PyramidLevelBuffers& b = levels[level];
    const size_t n = static_cast<size_t>(lw) * lh;
    if (b.depth.count != n) b.depth.resize(n);
    if (b.vertices.count != n * 3) b.vertices.resize(n * 3);
    if (b.normals.count != n * 3) b.normals.resize(n * 3);
    b.width = lw;
    b.height = lh;
    b.intrinsics = scaled(k, level);
    ++count;
    lw /= 2;
    lh /= 2;
  }
  level_count = count;
  return count;
}

void Pyramid::launch(cudaStream_t s) const {
  const DepthParams p = depth_params(options);
  for (uint32_t level = 0; level < level_count; ++level) {
    const PyramidLevelBuffers& b = levels[level];
    const dim3 block(kTileX, kTileY);
    const dim3 grid(ceil_div(b.width, kTileX), ceil_div(b.height, kTileY));
    if (level == 0) {
      if (!options.bilateral_filter || options.bilateral_radius == 0) {
        check(cudaMemcpyAsync(b.depth.ptr, raw.ptr, raw.bytes(), cudaMemcpyDeviceToDevice, s),
              "pyramid level-0 copy");
      } else {
        bilateral_kernel<<<grid, block, 0, s>>>(raw.ptr, b.depth.ptr, static_cast<int>(b.width),
                                                static_cast<int>(b.height), p);
        check(cudaGetLastError(), "bilateral_kernel launch");
      }
    }
    uint16_t* next = level + 1 < level_count ? levels[level + 1].depth.ptr : nullptr;
    level_kernel<<<grid, block, 0, s>>>(b.depth.ptr, static_cast<int>(b.width),
                                        static_cast<int>(b.height), intr_from(b.intrinsics), p,
                                        b.vertices.ptr, b.normals.ptr, next);
    check(cudaGetLastError(), "level_kernel launch");
  }
}

}  // namespace kf

using namespace kf;

extern "C" {

void kf_default_depth_options(kf_depth_options* o) {
  // DepthProcessingOptions defaults (depth_processing.hpp:24-41, rgbd.hpp:15-17)
  o->levels = 3;
  o->depth_scale = 5000.0f;
  o->min_depth = 0.4f;
  o->max_depth = 8.0f;
  o->max_normal_depth_jump = 0.1f;
  o->max_downsample_depth_jump = 0.1f;
  o->bilateral_filter = 1;
  o->bilateral_radius = 2;
  o->bilateral_spatial_sigma = 2.0f;
  o->bilateral_depth_sigma = 0.08f;
}

kf_status kf_pyramid_create(const kf_depth_options* options, kf_pyramid** out) {
  return guarded([&] {
    require(options != nullptr && out != nullptr, "kf_pyramid_create: null argument");
    validate(*options);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
      throw CudaError("no CUDA device available");
    }
    auto* p = new kf_pyramid();
    p->impl.options = *options;
    *out = p;
  });
}

kf_status kf_pyramid_destroy(kf_pyramid* pyramid) {
  return guarded([&] { delete pyramid; });
}

kf_status kf_pyramid_build(kf_pyramid* pyramid, const uint16_t* depth, uint32_t width, uint32_t height,
                           kf_intrinsics intrinsics, int32_t memory, uint32_t* level_count) {
  return guarded([&] {
    require(pyramid != nullptr && depth != nullptr, "kf_pyramid_build: null argument");
    Pyramid& p = pyramid->impl;
    const uint32_t count = p.prepare(width, height, intrinsics);
    const cudaMemcpyKind kind = memory == KF_MEMORY_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    check(cudaMemcpyAsync(p.raw.ptr, depth, p.raw.bytes(), kind, 0), "pyramid depth upload");
    p.launch(0);
    check(cudaStreamSynchronize(0), "pyramid build");
    if (level_count) *level_count = count;
  });
}

kf_status kf_pyramid_level(const kf_pyramid* pyramid, uint32_t index, kf_level_view* out) {
  return guarded([&] {
    require(pyramid != nullptr && out != nullptr, "kf_pyramid_level: null argument");
    const Pyramid& p = pyramid->impl;
    require(index < p.level_count, "kf_pyramid_level: level index out of range");
    const PyramidLevelBuffers& b = p.levels[index];
    out->depth = b.depth.ptr;
    out->vertices = b.vertices.ptr;
    out->normals = b.normals.ptr;
    out->width = b.width;
    out->height = b.height;
    out->intrinsics = b.intrinsics;
  });
}

kf_status kf_pyramid_raw_depth(const kf_pyramid* pyramid, const uint16_t** depth) {
  return guarded([&] {
    require(pyramid != nullptr && depth != nullptr, "kf_pyramid_raw_depth: null argument");
    const Pyramid& p = pyramid->impl;
    require(p.level_count > 0, "kf_pyramid_raw_depth: no frame built yet");
    *depth = p.raw.ptr;
  });
}

kf_status kf_pyramid_download_level(const kf_pyramid* pyramid, uint32_t index, uint16_t* depth,
                                    float* vertices, float* normals) {
  return guarded([&] {
    require(pyramid != nullptr, "kf_pyramid_download_level: null pyramid");
    const Pyramid& p = pyramid->impl;
    require(index < p.level_count, "kf_pyramid_download_level: level index out of range");
    const PyramidLevelBuffers& b = p.levels[index];
    if (depth) check(cudaMemcpy(depth, b.depth.ptr, b.depth.bytes(), cudaMemcpyDeviceToHost), "download depth");
    if (vertices)
      check(cudaMemcpy(vertices, b.vertices.ptr, b.vertices.bytes(), cudaMemcpyDeviceToHost), "download vertices");
    if (normals)
      check(cudaMemcpy(normals, b.normals.ptr, b.normals.bytes(), cudaMemcpyDeviceToHost), "download normals");
  });
}

}  // extern "C"
