// kf_tune.cu - launch-shape autotuner (no counterpart in the reference).
//
// Picks, per pipeline, the march CTA shape and the fusion grid that run a
// short sequence of frames fastest on this GPU.  Only shapes that leave every
// output bit unchanged are tuned: the march's rays are independent of the CTA
// they share (a cooperative warp only takes samples the ray's own march
// would take), and each fused brick is independent of the grid that
// strides over the list.  The ICP grid is not tuned: it sets the order of the
// FP32 reduction.  The candidates run on a scratch pipeline of the same
// configuration, reset before each candidate and fed the same frames.
#include <cstring>
#include <vector>

#include "kf_internal.h"

using namespace kf;

namespace {

struct Scratch {
  kf_pipeline* pipeline = nullptr;
  kf_pyramid* pyramid = nullptr;
  kf_tracker* tracker = nullptr;
  cudaEvent_t start = nullptr, stop = nullptr;
  ~Scratch() {
    if (start) cudaEventDestroy(start);
    if (stop) cudaEventDestroy(stop);
    if (tracker) kf_tracker_destroy(tracker);
    if (pyramid) kf_pyramid_destroy(pyramid);
    if (pipeline) kf_pipeline_destroy(pipeline);
  }
};

void ok(kf_status st, const char* what) {
  if (st != KF_OK) throw CudaError(std::string(what) + ": " + kf_last_error());
}

// Device time of frames 1..count-1 (frame 0 is fused without tracking),
// replayed twice: the first pass captures the frame graphs.
float time_frames(Scratch& s, const uint16_t* frames, uint32_t count, uint32_t width, uint32_t height,
                  kf_intrinsics k) {
  const size_t n = static_cast<size_t>(width) * height;
  const kf_rigid identity = {{1, 0, 0, 0, 1, 0, 0, 0, 1}, {0, 0, 0}};
  Pipeline& p = s.pipeline->impl;
  float ms = 0.0f;
  for (int pass = 0; pass < 2; ++pass) {
    ok(kf_pipeline_reset(s.pipeline), "autotune reset");
    ok(kf_frame_set_pose(s.pipeline, s.tracker, &identity), "autotune pose");
    ok(kf_frame_enqueue(s.pipeline, s.pyramid, s.tracker, frames, nullptr, width, height, k, KF_MEMORY_DEVICE,
                        nullptr, 1),
       "autotune frame");
    check(cudaEventRecord(s.start, p.stream), "autotune event");
    for (uint32_t f = 1; f < count; ++f) {
      ok(kf_frame_enqueue(s.pipeline, s.pyramid, s.tracker, frames + f * n, nullptr, width, height, k,
                          KF_MEMORY_DEVICE, nullptr, 0),
         "autotune frame");
    }
    check(cudaEventRecord(s.stop, p.stream), "autotune event");
    check(cudaEventSynchronize(s.stop), "autotune sync");
    check(cudaEventElapsedTime(&ms, s.start, s.stop), "autotune time");
  }
  return ms;
}

void apply(Pipeline& p, const kf_launch_shapes& shapes) {
  if (p.raycast_block_x == shapes.raycast_block_x && p.raycast_block_y == shapes.raycast_block_y &&
      p.integrate_ctas == shapes.integrate_ctas && p.raycast_lanes[0] == shapes.raycast_lanes[0] &&
      p.raycast_lanes[1] == shapes.raycast_lanes[1] && p.raycast_lanes[2] == shapes.raycast_lanes[2]) {
    return;
  }
  check(cudaStreamSynchronize(p.stream), "launch shapes");
  p.raycast_block_x = shapes.raycast_block_x;
  p.raycast_block_y = shapes.raycast_block_y;
  p.integrate_ctas = shapes.integrate_ctas;
  for (int i = 0; i < 3; ++i) p.raycast_lanes[i] = shapes.raycast_lanes[i];
  p.clear_graphs();  // the graphs hold the old shapes
}

void validate(const kf_launch_shapes& s) {
  require(s.raycast_block_x > 0 && s.raycast_block_y > 0 && s.raycast_block_x * s.raycast_block_y <= 64,
          "Raycast CTA shape must have 1..64 threads");
  require(s.integrate_ctas > 0 && s.integrate_ctas <= 65535u, "Fusion grid must have 1..65535 CTAs");
  for (int i = 0; i < 3; ++i) {
    const uint32_t l = s.raycast_lanes[i];
    require(l >= 1 && l <= 32 && (l & (l - 1)) == 0, "Lanes per ray must be 1, 2, 4, 8, 16 or 32");
  }
}

}  // namespace

extern "C" {

kf_status kf_pipeline_get_launch_shapes(kf_pipeline* pipeline, kf_launch_shapes* shapes) {
  return guarded([&] {
    require(pipeline != nullptr && shapes != nullptr, "kf_pipeline_get_launch_shapes: null argument");
    const Pipeline& p = pipeline->impl;
    shapes->raycast_block_x = p.raycast_block_x;
    shapes->raycast_block_y = p.raycast_block_y;
    shapes->integrate_ctas = p.integrate_ctas;
    for (int i = 0; i < 3; ++i) shapes->raycast_lanes[i] = p.raycast_lanes[i];
  });
}

kf_status kf_pipeline_set_launch_shapes(kf_pipeline* pipeline, const kf_launch_shapes* shapes) {
  return guarded([&] {
    require(pipeline != nullptr && shapes != nullptr, "kf_pipeline_set_launch_shapes: null argument");
    validate(*shapes);
    apply(pipeline->impl, *shapes);
  });
}

kf_status kf_pipeline_set_concurrent(kf_pipeline* pipeline, int32_t concurrent) {
  return guarded([&] {
    require(pipeline != nullptr, "kf_pipeline_set_concurrent: null pipeline");
    Pipeline& p = pipeline->impl;
    const bool want = concurrent != 0;
    if (p.concurrent == want) return;
    check(cudaStreamSynchronize(p.stream), "concurrency switch");
    p.concurrent = want;
    p.clear_graphs();  // the graphs hold the other form of the ICP levels
  });
}

kf_status kf_pipeline_autotune(kf_pipeline* pipeline, const uint16_t* frames, uint32_t count, uint32_t width,
                               uint32_t height, kf_intrinsics intrinsics, kf_launch_shapes* chosen,
                               float* best_ms) {
  return guarded([&] {
    require(pipeline != nullptr && frames != nullptr && chosen != nullptr, "kf_pipeline_autotune: null argument");
    require(count >= 2, "kf_pipeline_autotune: at least two frames");
    Scratch s;
    ok(kf_pipeline_create(&pipeline->impl.config, &s.pipeline), "autotune pipeline");
    kf_depth_options depth;
    kf_default_depth_options(&depth);
    ok(kf_pyramid_create(&depth, &s.pyramid), "autotune pyramid");
    kf_icp_options icp;
    kf_default_icp_options(&icp);
    ok(kf_tracker_create(&icp, &s.tracker), "autotune tracker");
    check(cudaEventCreate(&s.start), "autotune event");
    check(cudaEventCreate(&s.stop), "autotune event");
    Pipeline& sp = s.pipeline->impl;
    kf_launch_shapes best{sp.raycast_block_x, sp.raycast_block_y, sp.integrate_ctas,
                          {sp.raycast_lanes[0], sp.raycast_lanes[1], sp.raycast_lanes[2]}};
    float best_time = time_frames(s, frames, count, width, height, intrinsics);
    // the march CTA first, then the lanes per ray, then the fusion grid
    const uint32_t shapes[][2] = {{8, 8}, {16, 4}, {32, 2}, {4, 16}, {8, 4}, {16, 2}};
    for (const auto& sh : shapes) {
      kf_launch_shapes c = best;
      c.raycast_block_x = sh[0];
      c.raycast_block_y = sh[1];
      apply(sp, c);
      const float t = time_frames(s, frames, count, width, height, intrinsics);
      if (t < best_time) {
        best_time = t;
        best = c;
      }
    }
    // lanes per ray of each render-size class (one class at a time)
    for (int cls = 0; cls < 3; ++cls) {
      for (uint32_t lanes : {1u, 2u, 4u, 8u, 16u, 32u}) {
        if (lanes == best.raycast_lanes[cls]) continue;
        kf_launch_shapes c = best;
        c.raycast_lanes[cls] = lanes;
        apply(sp, c);
        const float t = time_frames(s, frames, count, width, height, intrinsics);
        if (t < best_time) {
          best_time = t;
          best = c;
        }
      }
    }
    const uint32_t grids[] = {148 * 8, 148 * 16, 148 * 24, 148 * 32, 148 * 48};
    for (uint32_t g : grids) {
      kf_launch_shapes c = best;
      c.integrate_ctas = g;
      apply(sp, c);
      const float t = time_frames(s, frames, count, width, height, intrinsics);
      if (t < best_time) {
        best_time = t;
        best = c;
      }
    }
    apply(pipeline->impl, best);
    *chosen = best;
    if (best_ms) *best_ms = best_time;
  });
}

}  // extern "C"
