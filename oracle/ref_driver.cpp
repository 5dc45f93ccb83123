// ref_driver.cpp - drives the reference's OWN host implementation, compiled
// from its sources (see ref_build.sh), behind a small C ABI for the tests.
//
// TEST INFRASTRUCTURE ONLY.  This file is this project's code; everything it
// calls (DepthProcessor<kHost>, DenseRep / BlockRep<kHost>, TsdfIntegrator,
// Raycaster, EmptySpaceIndex, ProjectiveIcpTracker, HostCorrespondenceSearch,
// MarchingCubes) is the reference's, from include/kinectfusion/*.hpp and
// src/kinectfusion/*.cpp, built against this project's Eigen stand-in
// (ref_shim/Eigen).  The tests use it to pin oracle/kf_oracle.c (the C
// restatement the device is checked against) to the reference's arithmetic.
//
// The representation wrapper below does what the reference's
// BasicHostPipeline does (src/kinectfusion/pipeline.cpp:23-103: integrate,
// then rebuild the skip index of flat storage; render through the index) and
// also exposes the raw voxel storage, which the type-erased Pipeline hides.
// The frame loop follows Reconstruction::process_frame / track_pose /
// integrate_members (src/app/reconstruction.cpp:184-277), whose app TU needs
// libraries that are not installed here.
#include <Eigen/Core>
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <exception>
#include <kinectfusion/block_rep.hpp>
#include <kinectfusion/depth_processing.hpp>
#include <kinectfusion/icp_correspondence.hpp>
#include <kinectfusion/icp_optimizer.hpp>
#include <kinectfusion/marching_cubes.hpp>
#include <kinectfusion/pipeline.hpp>
#include <kinectfusion/raycasting.hpp>
#include <kinectfusion/tsdf_integration.hpp>
#include <kinectfusion/volume.hpp>
#include <kinectfusion/volume_representation.hpp>
#include <memory>
#include <optional>
#include <string>
#include <type_traits>
#include <variant>
#include <vector>

#include "../include/kf_b200.h"

namespace kf = kinectfusion;

namespace {

thread_local std::string g_error;

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  } catch (...) {
    g_error = "unknown exception";
    return 1;
  }
}

Eigen::Matrix4f to_matrix(const kf_rigid& r) {
  Eigen::Matrix4f m = Eigen::Matrix4f::Identity();
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) m(i, j) = r.r[i * 3 + j];
    m(i, 3) = r.t[i];
  }
  return m;
}

kf_rigid to_rigid(const Eigen::Matrix4f& m) {
  kf_rigid r{};
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) r.r[i * 3 + j] = m(i, j);
    r.t[i] = m(i, 3);
  }
  return r;
}

kf::CameraIntrinsics to_intrinsics(const kf_intrinsics& k) {
  return kf::CameraIntrinsics{.fx = k.fx, .fy = k.fy, .cx = k.cx, .cy = k.cy};
}

kf::DepthProcessingOptions to_depth_options(const kf_depth_options& o) {
  kf::DepthProcessingOptions d;
  d.levels = o.levels;
  d.depth_scale = o.depth_scale;
  d.min_depth = o.min_depth;
  d.max_depth = o.max_depth;
  d.max_normal_depth_jump = o.max_normal_depth_jump;
  d.max_downsample_depth_jump = o.max_downsample_depth_jump;
  d.bilateral_filter = o.bilateral_filter != 0;
  d.bilateral_radius = o.bilateral_radius;
  d.bilateral_spatial_sigma = o.bilateral_spatial_sigma;
  d.bilateral_depth_sigma = o.bilateral_depth_sigma;
  return d;
}

kf::ProjectiveIcpOptions to_icp_options(const kf_icp_options& o) {
  kf::ProjectiveIcpOptions r;
  r.min_correspondences = o.min_correspondences;
  r.max_point_distance = o.max_point_distance;
  r.min_normal_dot = o.min_normal_dot;
  r.min_update_translation = o.min_update_translation;
  r.min_update_rotation = o.min_update_rotation;
  r.max_update_translation = o.max_update_translation;
  r.max_update_rotation = o.max_update_rotation;
  r.min_system_eigenvalue = o.min_system_eigenvalue;
  r.max_condition_number = o.max_condition_number;
  r.damping = kf::IcpDamping{.mode = static_cast<kf::IcpDampingMode>(o.damping_mode), .lambda = o.damping_lambda};
  r.adaptive_damping = o.adaptive_damping != 0;
  r.schedule = kf::IcpDampingSchedule{.increase = o.lambda_increase,
                                      .decrease = o.lambda_decrease,
                                      .min_lambda = o.min_lambda,
                                      .max_lambda = o.max_lambda};
  return r;
}

// Same enumerator order as pipeline.hpp:24-26, raycasting.hpp:22 and
// volume_sampler.hpp's CornerPolicy.
kf::PipelineConfig to_config(const kf_pipeline_config& c) {
  kf::PipelineConfig p;
  p.name = "reference";
  p.space = kf::MemorySpace::kHost;
  if (c.tsdf_rule == KF_RULE_CLASSIC) {
    p.tsdf_rule = kf::ClassicTsdf{};
  } else {
    p.tsdf_rule = kf::AngleWeightedTsdf{};
  }
  const kf_integration_options& i = c.integration;
  p.integration = kf::TsdfIntegrationOptions{.depth_scale = i.depth_scale,
                                             .observation_weight = i.observation_weight,
                                             .max_weight = i.max_weight,
                                             .min_depth = i.min_depth,
                                             .max_depth = i.max_depth,
                                             .projective_distance = i.projective_distance != 0,
                                             .distance_scaled_truncation = i.distance_scaled_truncation != 0,
                                             .truncation_distance_scale = i.truncation_distance_scale,
                                             .mode = static_cast<kf::IntegrationMode>(i.mode)};
  const kf_raycast_options& r = c.raycast;
  p.raycast = kf::RaycastOptions{.min_depth = r.min_depth,
                                 .max_depth = r.max_depth,
                                 .step_scale = r.step_scale,
                                 .tsdf_corner_policy = static_cast<kf::CornerPolicy>(r.corner_policy),
                                 .cell_gradient_normals = r.cell_gradient_normals != 0,
                                 .seed_from_previous = r.seed_from_previous != 0};
  p.volume = kf::VolumeGeometry{
      .resolution = kf::Size3{.x = c.volume.res_x, .y = c.volume.res_y, .z = c.volume.res_z},
      .voxel_size = c.volume.voxel_size,
      .origin = kf::make_vec3f(c.volume.origin[0], c.volume.origin[1], c.volume.origin[2]),
      .truncation_distance = c.volume.truncation_distance};
  p.voxel = static_cast<kf::VoxelStore>(c.voxel);
  p.color = static_cast<kf::ColorStore>(c.color);
  p.raycast_backend = static_cast<kf::RaycastBackend>(c.raycast_backend);
  p.storage = static_cast<kf::StorageLayout>(c.storage);
  p.sparse_block_capacity = c.sparse_block_capacity;
  return p;
}

// The host pipeline's work over one registered representation, with the raw
// storage exposed (what BasicHostPipeline does, pipeline.cpp:23-103).
class Model {
 public:
  virtual ~Model() = default;
  virtual void integrate(const kf::DepthFrame& frame) = 0;
  virtual kf::SurfaceMaps raycast(const kf::RaycastCamera& camera) = 0;
  virtual std::size_t observed() const = 0;
  virtual kf::MarchingCubes::Mesh mesh(float min_weight) const = 0;
  // which: 0 = voxels (dense) or pool (sparse), 1 = colours, 2 = block grid
  virtual std::size_t raw_bytes(int which) const = 0;
  virtual void copy_raw(int which, void* out) const = 0;
  virtual int overflowed() const = 0;
};

template <typename Rep>
class ModelOf final : public Model {
  static constexpr bool kFlat = kf::FlatVoxelRepresentation<Rep>;

 public:
  explicit ModelOf(const kf::PipelineConfig& config)
      : rep_(kf::RepresentationFactory::make<Rep>(config.volume, config.sparse_block_capacity)),
        index_(kFlat ? kf::EmptySpaceIndex<kf::MemorySpace::kHost>{config.raycast_backend, config.volume}
                     : kf::EmptySpaceIndex<kf::MemorySpace::kHost>{}),
        integrator_(config.tsdf_rule, config.integration),
        raycaster_(config.raycast) {}

  void integrate(const kf::DepthFrame& frame) override {
    kf::TsdfIntegrator::validate_frame(frame);
    rep_.integrate(frame.view(), integrator_.options(), integrator_.rule());
    if constexpr (kFlat) {
      index_.rebuild(rep_.view());
    }
  }

  kf::SurfaceMaps raycast(const kf::RaycastCamera& camera) override {
    if constexpr (kFlat) {
      return index_.visit([&](const auto& skip) { return raycaster_.render(rep_.sampler(), camera, skip); });
    } else {
      return raycaster_.render(rep_.sampler(), camera);
    }
  }

  std::size_t observed() const override { return rep_.observed_voxel_count(); }

  kf::MarchingCubes::Mesh mesh(float min_weight) const override {
    return kf::MarchingCubes::extract(rep_.view(), min_weight);
  }

  std::size_t raw_bytes(int which) const override {
    const auto v = rep_.view();
    using View = std::remove_cvref_t<decltype(v)>;
    using Geom = typename View::GeometryVoxel;
    using ColorVoxel = typename View::ColorFacet::Voxel;
    if constexpr (kFlat) {
      if (which == 0) return v.voxel_count() * sizeof(Geom);
      if (which == 1) return View::ColorFacet::kEnabled ? v.voxel_count() * sizeof(ColorVoxel) : 0;
      return 0;
    } else {
      const std::size_t slots = static_cast<std::size_t>(v.capacity) * kf::kVoxelBlockVolume;
      if (which == 0) return slots * sizeof(Geom);
      if (which == 1) return View::ColorFacet::kEnabled ? slots * sizeof(ColorVoxel) : 0;
      return v.blocks.count() * sizeof(std::uint32_t);
    }
  }

  void copy_raw(int which, void* out) const override {
    const auto v = rep_.view();
    const std::size_t bytes = raw_bytes(which);
    if (bytes == 0) return;
    if constexpr (kFlat) {
      std::memcpy(out, which == 0 ? static_cast<const void*>(v.voxels) : static_cast<const void*>(v.colors), bytes);
    } else {
      const void* src = which == 0   ? static_cast<const void*>(v.pool)
                        : which == 1 ? static_cast<const void*>(v.color_pool)
                                     : static_cast<const void*>(v.grid);
      std::memcpy(out, src, bytes);
    }
  }

  int overflowed() const override {
    if constexpr (kFlat) {
      return 0;
    } else {
      return rep_.overflowed() ? 1 : 0;
    }
  }

 private:
  Rep rep_;
  kf::EmptySpaceIndex<kf::MemorySpace::kHost> index_;
  kf::TsdfIntegrator integrator_;
  kf::Raycaster raycaster_;
};

std::unique_ptr<Model> make_model(const kf::PipelineConfig& config) {
  kf::Pipeline::require_valid_storage(config);
  return kf::Pipeline::visit_representation<kf::MemorySpace::kHost>(
      config, [&config]<typename Rep>() -> std::unique_ptr<Model> { return std::make_unique<ModelOf<Rep>>(config); });
}

void copy_vec3_image(const kf::image_proc::Vector3fImage& img, float* out) {
  if (out == nullptr) return;
  std::memcpy(out, img.data().data(), img.data().size() * sizeof(kf::Vec3f));
}

kf::image_proc::DepthImage depth_image(const uint16_t* depth, uint32_t w, uint32_t h) {
  kf::image_proc::DepthImage img{w, h};
  std::memcpy(img.data().data(), depth, static_cast<std::size_t>(w) * h * sizeof(uint16_t));
  return img;
}

kf::image_proc::Vector3fImage vec3_image(const float* data, uint32_t w, uint32_t h) {
  kf::image_proc::Vector3fImage img{w, h};
  std::memcpy(img.data().data(), data, static_cast<std::size_t>(w) * h * sizeof(kf::Vec3f));
  return img;
}

int32_t status_of(const kf::IcpOutcome& o) {
  if (o.result) {
    return std::holds_alternative<kf::Converged>(*o.result) ? KF_ICP_CONVERGED : KF_ICP_MAX_ITERATIONS;
  }
  switch (o.result.error()) {
    case kf::IcpFailure::kInvalidInput:
      return KF_ICP_INVALID_INPUT;
    case kf::IcpFailure::kTooFewCorrespondences:
      return KF_ICP_TOO_FEW_CORRESPONDENCES;
    case kf::IcpFailure::kUnconstrainedSystem:
      return KF_ICP_UNCONSTRAINED_SYSTEM;
    case kf::IcpFailure::kSolveFailed:
      return KF_ICP_SOLVE_FAILED;
    case kf::IcpFailure::kUpdateTooLarge:
      return KF_ICP_UPDATE_TOO_LARGE;
  }
  return KF_ICP_INVALID_INPUT;
}

void fill_outcome(const kf::IcpOutcome& o, kf_icp_outcome* out) {
  std::memset(out, 0, sizeof(*out));
  out->pose = to_rigid(o.pose);
  out->status = status_of(o);
  out->iterations = -1;  // not reported by the reference's outcome
  const kf::IcpDiagnostics& d = o.diagnostics;
  out->correspondences = d.correspondences;
  out->mean_point_distance = d.mean_point_distance;
  out->mean_squared_residual = d.mean_squared_residual;
  out->min_system_eigenvalue = d.min_system_eigenvalue;
  out->condition_number = d.condition_number;
  out->update_translation = d.update_translation;
  out->update_rotation = d.update_rotation;
  out->damping_lambda = d.damping_lambda;
  out->rejected_steps = d.rejected_steps;
}

// Reconstruction's IcpConsumer (reconstruction.cpp:41-73).
class IcpConsumer final : public kf::TrackingSurfaceConsumer {
 public:
  IcpConsumer(const kf::ProjectiveIcpTracker& tracker, const kf::CameraIntrinsics& intrinsics,
              const Eigen::Matrix4f& pose, unsigned int iterations)
      : tracker_(tracker), intrinsics_(intrinsics), pose_(pose), iterations_(iterations) {}
  void consume(const kf::HostTrackingSurfaces& surfaces) override {
    outcome_ = tracker_.estimate_pose(surfaces, intrinsics_, pose_, iterations_);
  }
  void consume(const kf::DeviceTrackingSurfaces& surfaces) override {
#ifdef KF_REF_CUDA
    outcome_ = tracker_.estimate_pose(surfaces, intrinsics_, pose_, iterations_);
#else
    (void)surfaces;
    throw std::logic_error("host surfaces only: this build has no CUDA path");
#endif
  }
  const kf::IcpOutcome& outcome() const { return outcome_; }

 private:
  const kf::ProjectiveIcpTracker& tracker_;
  kf::CameraIntrinsics intrinsics_;
  Eigen::Matrix4f pose_;
  unsigned int iterations_;
  kf::IcpOutcome outcome_;
};

}  // namespace

struct kfr_pipeline {
  kf::PipelineConfig config;
  std::unique_ptr<Model> model;
  kf::MarchingCubes::Mesh mesh;
};

extern "C" {

const char* kfr_last_error(void) { return g_error.c_str(); }

// DepthProcessor<kHost>::build_surface_pyramid (depth_processing.cpp:139-162).
// Outputs are packed level after level (level l is (w >> l) x (h >> l)).
int kfr_pyramid(const uint16_t* depth, uint32_t width, uint32_t height, const kf_intrinsics* intrinsics,
                const kf_depth_options* options, uint16_t* depth_out, float* vertices_out, float* normals_out,
                uint32_t* levels_out) {
  return guarded([&] {
    const kf::DepthProcessor<kf::MemorySpace::kHost> processor{to_depth_options(*options)};
    const kf::SurfacePyramid pyramid =
        processor.build_surface_pyramid(depth_image(depth, width, height), to_intrinsics(*intrinsics));
    std::size_t offset = 0;
    for (const auto& level : pyramid) {
      const std::size_t n = level.depth_image.width() * level.depth_image.height();
      std::memcpy(depth_out + offset, level.depth_image.data().data(), n * sizeof(uint16_t));
      copy_vec3_image(level.surface.vertices, vertices_out + 3 * offset);
      copy_vec3_image(level.surface.normals, normals_out + 3 * offset);
      offset += n;
    }
    *levels_out = static_cast<uint32_t>(pyramid.size());
  });
}

int kfr_pipeline_create(const kf_pipeline_config* config, kfr_pipeline** out) {
  return guarded([&] {
    auto p = std::make_unique<kfr_pipeline>();
    p->config = to_config(*config);
    p->model = make_model(p->config);
    *out = p.release();
  });
}

void kfr_pipeline_destroy(kfr_pipeline* p) { delete p; }

// Pipeline::integrate (pipeline.hpp:75-79) at the given world_to_camera.
int kfr_pipeline_integrate(kfr_pipeline* p, const uint16_t* depth, const uint32_t* color, const float* normals,
                           uint32_t width, uint32_t height, const kf_intrinsics* intrinsics,
                           const kf_rigid* world_to_camera) {
  return guarded([&] {
    const kf::image_proc::DepthImage d = depth_image(depth, width, height);
    std::optional<kf::image_proc::ColorImage> c;
    std::optional<kf::image_proc::Vector3fImage> n;
    if (color != nullptr) {
      c.emplace(width, height);
      std::memcpy(c->data().data(), color, static_cast<std::size_t>(width) * height * sizeof(uint32_t));
    }
    if (normals != nullptr) n.emplace(vec3_image(normals, width, height));
    const kf::DepthFrame frame{.depth = &d,
                               .color = c ? &*c : nullptr,
                               .normals = n ? &*n : nullptr,
                               .intrinsics = to_intrinsics(*intrinsics),
                               .world_to_camera = to_matrix(*world_to_camera)};
    p->model->integrate(frame);
  });
}

// Pipeline::raycast (pipeline.hpp:81).
int kfr_pipeline_raycast(kfr_pipeline* p, const kf_intrinsics* intrinsics, uint32_t width, uint32_t height,
                         const kf_rigid* camera_to_world, float* points, float* normals, uint32_t* colors) {
  return guarded([&] {
    const kf::RaycastCamera camera{.intrinsics = to_intrinsics(*intrinsics),
                                   .width = width,
                                   .height = height,
                                   .camera_to_world = to_matrix(*camera_to_world)};
    const kf::SurfaceMaps maps = p->model->raycast(camera);
    copy_vec3_image(maps.points, points);
    copy_vec3_image(maps.normals, normals);
    if (colors != nullptr) {
      std::memcpy(colors, maps.colors.data().data(), maps.colors.data().size() * sizeof(uint32_t));
    }
  });
}

uint64_t kfr_pipeline_observed(const kfr_pipeline* p) { return p->model->observed(); }

uint64_t kfr_pipeline_raw_bytes(const kfr_pipeline* p, int32_t which) { return p->model->raw_bytes(which); }

int kfr_pipeline_copy_raw(const kfr_pipeline* p, int32_t which, void* out) {
  return guarded([&] { p->model->copy_raw(which, out); });
}

int32_t kfr_pipeline_overflowed(const kfr_pipeline* p) { return p->model->overflowed(); }

// MarchingCubes::extract over the pipeline's view (Pipeline::extract_mesh);
// the mesh is kept until the next call and copied out by kfr_pipeline_mesh_copy.
int kfr_pipeline_mesh(kfr_pipeline* p, float min_weight, uint64_t* vertices, uint64_t* triangles) {
  return guarded([&] {
    p->mesh = p->model->mesh(min_weight);
    *vertices = p->mesh.positions.size();
    *triangles = p->mesh.triangles.size();
  });
}

int kfr_pipeline_mesh_copy(const kfr_pipeline* p, float* positions, float* normals, float* colors,
                           uint32_t* triangles) {
  return guarded([&] {
    const auto& m = p->mesh;
    std::memcpy(positions, m.positions.data(), m.positions.size() * sizeof(kf::Vec3f));
    std::memcpy(normals, m.normals.data(), m.normals.size() * sizeof(kf::Vec3f));
    std::memcpy(colors, m.colors.data(), m.colors.size() * sizeof(kf::Vec3f));
    std::memcpy(triangles, m.triangles.data(), m.triangles.size() * 3 * sizeof(uint32_t));
  });
}

// One correspondence sweep in pixel order: HostCorrespondenceSearch::match +
// IcpNormalEquations::accumulate, as ProjectiveIcpTracker::find_correspondences
// (icp_optimizer.cpp:304-317).  sums = 21 JtJ, 6 Jtr, distance sum, squared
// residual sum.
int kfr_icp_equations(const float* live_vertices, const float* live_normals, uint32_t live_width,
                      uint32_t live_height, const float* model_points, const float* model_normals,
                      uint32_t model_width, uint32_t model_height, const kf_intrinsics* model_intrinsics,
                      const kf_rigid* camera, const kf_rigid* model, float max_point_distance, float min_normal_dot,
                      float* sums, uint64_t* count) {
  return guarded([&] {
    const auto lv = vec3_image(live_vertices, live_width, live_height);
    const auto ln = vec3_image(live_normals, live_width, live_height);
    const auto mv = vec3_image(model_points, model_width, model_height);
    const auto mn = vec3_image(model_normals, model_width, model_height);
    const kf::HostTrackingSurfaces surfaces{.live = {.vertices = lv.view(), .normals = ln.view()},
                                            .model = {.vertices = mv.view(), .normals = mn.view()}};
    const kf::IcpIterationTransforms transforms =
        kf::IcpIterationTransforms::from_poses(to_matrix(*camera), to_matrix(*model));
    const kf::HostCorrespondenceSearch search{
        surfaces, to_intrinsics(*model_intrinsics), transforms,
        kf::CorrespondenceGates{.max_point_distance = max_point_distance, .min_normal_dot = min_normal_dot}};
    kf::IcpNormalEquations equations;
    for (const auto [x, y] : kf::PixelIndices{live_width, live_height}) {
      if (const auto match = search.match(x, y)) equations.accumulate(*match);
    }
    for (std::size_t i = 0; i < kf::kIcpUpperTriangleSize; ++i) sums[i] = equations.jtj.at(i);
    for (std::size_t i = 0; i < kf::kIcpDof; ++i) sums[21 + i] = equations.jtr.at(i);
    sums[27] = equations.distance_sum;
    sums[28] = equations.residual_sum_squares;
    *count = equations.count;
  });
}

// ProjectiveIcpTracker::estimate_pose(TrackingRequest) (icp_optimizer.cpp:46-56).
int kfr_icp_estimate(const float* live_vertices, const float* live_normals, uint32_t live_width,
                     uint32_t live_height, const float* model_points, const float* model_normals,
                     uint32_t model_width, uint32_t model_height, const kf_intrinsics* model_intrinsics,
                     const kf_rigid* model_camera_to_world, const kf_rigid* initial_camera_to_world,
                     uint32_t iterations, const kf_icp_options* options, kf_icp_outcome* outcome) {
  return guarded([&] {
    const auto lv = vec3_image(live_vertices, live_width, live_height);
    const auto ln = vec3_image(live_normals, live_width, live_height);
    const auto mv = vec3_image(model_points, model_width, model_height);
    const auto mn = vec3_image(model_normals, model_width, model_height);
    const kf::ProjectiveIcpTracker tracker{to_icp_options(*options)};
    const kf::TrackingRequest request{
        .surfaces = {.live = {.vertices = lv.view(), .normals = ln.view()},
                     .model = {.vertices = mv.view(), .normals = mn.view()}},
        .model_intrinsics = to_intrinsics(*model_intrinsics),
        .model_camera_to_world = to_matrix(*model_camera_to_world),
        .initial_camera_to_world = to_matrix(*initial_camera_to_world),
        .iterations = iterations};
    fill_outcome(tracker.estimate_pose(request), outcome);
  });
}

// One frame of Reconstruction::process_frame (reconstruction.cpp:184-277) for
// one pipeline: pyramid, per level (coarsest first) a model render at the
// current estimate and ICP, then integration at the tracked pose when every
// level succeeded.  `first` = the initial frame (reconstruction.cpp:143-182),
// fused at `pose` without tracking.  pose is camera_to_world in and out;
// level_status[l] receives the level's KF_ICP_* (KF_ICP_NOT_RUN if skipped).
int kfr_track_frame(kfr_pipeline* p, const uint16_t* depth, const uint32_t* color, uint32_t width, uint32_t height,
                    const kf_intrinsics* intrinsics, const kf_depth_options* depth_options,
                    const kf_icp_options* icp_options, const uint32_t* iterations_per_level, int32_t first,
                    kf_rigid* pose, int32_t* tracked, int32_t* level_status) {
  return guarded([&] {
    const kf::DepthProcessor<kf::MemorySpace::kHost> processor{to_depth_options(*depth_options)};
    const kf::image_proc::DepthImage raw = depth_image(depth, width, height);
    const kf::CameraIntrinsics k = to_intrinsics(*intrinsics);
    const kf::SurfacePyramid pyramid = processor.build_surface_pyramid(raw, k);
    const kf::ProjectiveIcpTracker tracker{to_icp_options(*icp_options)};
    Eigen::Matrix4f camera_to_world = to_matrix(*pose);
    for (int l = 0; l < 4; ++l) level_status[l] = KF_ICP_NOT_RUN;
    bool ok = true;
    if (!first) {
      Eigen::Matrix4f tracked_pose = camera_to_world;
      for (std::size_t level_index = pyramid.size(); level_index-- > 0;) {
        const auto& level = pyramid[level_index];
        // AppOptions::raycast_camera: the level's size and scaled intrinsics
        const kf::RaycastCamera camera{.intrinsics = k.scaled(static_cast<unsigned int>(level_index)),
                                       .width = level.depth_image.width(),
                                       .height = level.depth_image.height(),
                                       .camera_to_world = tracked_pose};
        const kf::SurfaceMaps model = p->model->raycast(camera);
        IcpConsumer consumer{tracker, level.intrinsics, tracked_pose, iterations_per_level[level_index]};
        consumer.consume(kf::HostTrackingSurfaces::from_render(kf::view(level.surface), kf::view(model)));
        const kf::IcpOutcome& outcome = consumer.outcome();
        level_status[level_index] = status_of(outcome);
        tracked_pose = outcome.pose;
        if (!outcome.result) {
          ok = false;
          break;
        }
      }
      camera_to_world = tracked_pose;
    }
    if (ok) {
      std::optional<kf::image_proc::ColorImage> c;
      if (color != nullptr) {
        c.emplace(width, height);
        std::memcpy(c->data().data(), color, static_cast<std::size_t>(width) * height * sizeof(uint32_t));
      }
      const kf::DepthFrame frame{.depth = &raw,
                                 .color = c ? &*c : nullptr,
                                 .normals = &pyramid.front().surface.normals,
                                 .intrinsics = k,
                                 .world_to_camera = camera_to_world.inverse()};
      p->model->integrate(frame);
    }
    *pose = to_rigid(camera_to_world);
    *tracked = ok ? 1 : 0;
  });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The reference's own CUDA pipeline (built only into libkf_ref_cuda.so, with
// the reference's src/kinectfusion/cuda/*.cu): Pipeline::create with
// MemorySpace::kDevice (device_pipeline.cu), the device PyramidSource
// (depth_processing.cu) and ProjectiveIcpTracker's device correspondence
// sweep, driven by the loop of Reconstruction::process_frame.  Used to time
// the reference's GPU path on the same GPU and to compare outputs.
#ifdef KF_REF_CUDA
#include <cuda_runtime_api.h>

struct kfr_device {
  kf::PipelineConfig config;
  std::unique_ptr<kf::Pipeline> pipeline;
  std::unique_ptr<kf::PyramidSource> pyramid;
  std::unique_ptr<kf::ProjectiveIcpTracker> tracker;
  kf::image_proc::DepthImage depth;
  kf::image_proc::ColorImage color;
};

extern "C" {

int kfr_dev_available(void) {
  int count = 0;
  return cudaGetDeviceCount(&count) == cudaSuccess && count > 0 ? 1 : 0;
}

// device_solve / capture_graph: the reference's --icp-device-solve and
// --icp-capture-graph switches (app_options.cpp:138-141).
int kfr_dev_create(const kf_pipeline_config* config, const kf_depth_options* depth_options,
                   const kf_icp_options* icp_options, int32_t device_solve, int32_t capture_graph, kfr_device** out) {
  return guarded([&] {
    auto d = std::make_unique<kfr_device>();
    d->config = to_config(*config);
    d->config.space = kf::MemorySpace::kDevice;
    kf::Pipeline::Creation creation = kf::Pipeline::create(d->config);
    if (creation.space != kf::MemorySpace::kDevice) {
      throw std::runtime_error("reference device pipeline unavailable: " + creation.fallback_reason);
    }
    d->pipeline = std::move(creation.pipeline);
    kf::PyramidSource::Creation pyr = kf::PyramidSource::create(kf::MemorySpace::kDevice,
                                                                to_depth_options(*depth_options));
    if (!pyr.fallback_reason.empty()) throw std::runtime_error(pyr.fallback_reason);
    d->pyramid = std::move(pyr.source);
    kf::ProjectiveIcpOptions icp = to_icp_options(*icp_options);
    icp.device_solve = device_solve != 0;
    icp.device_graph_build = capture_graph ? kf::IcpGraphBuild::kCaptured : kf::IcpGraphBuild::kExplicit;
    d->tracker = std::make_unique<kf::ProjectiveIcpTracker>(icp);
    *out = d.release();
  });
}

void kfr_dev_destroy(kfr_device* d) { delete d; }

// One frame of Reconstruction::process_frame on the reference's device path
// (reconstruction.cpp:184-277): the host frame is uploaded by the device
// pyramid source, each level renders the model on the device and tracks
// (host or device solve), the frame is integrated from the pyramid's upload.
int kfr_dev_frame(kfr_device* d, const uint16_t* depth, const uint32_t* color, uint32_t width, uint32_t height,
                  const kf_intrinsics* intrinsics, const uint32_t* iterations_per_level, int32_t first,
                  kf_rigid* pose, int32_t* tracked, int32_t* level_status) {
  return guarded([&] {
    if (d->depth.width() != width || d->depth.height() != height) {
      d->depth = kf::image_proc::DepthImage{width, height};
      d->color = kf::image_proc::ColorImage{width, height};
    }
    std::memcpy(d->depth.data().data(), depth, static_cast<std::size_t>(width) * height * sizeof(uint16_t));
    if (color != nullptr) {
      std::memcpy(d->color.data().data(), color, static_cast<std::size_t>(width) * height * sizeof(uint32_t));
    }
    const kf::CameraIntrinsics k = to_intrinsics(*intrinsics);
    const std::size_t levels = d->pyramid->build(d->depth, k);
    Eigen::Matrix4f camera_to_world = to_matrix(*pose);
    for (int l = 0; l < 4; ++l) level_status[l] = KF_ICP_NOT_RUN;
    bool ok = levels > 0;
    if (!first && ok) {
      Eigen::Matrix4f tracked_pose = camera_to_world;
      for (std::size_t level_index = levels; level_index-- > 0;) {
        const unsigned int scale = 1U << level_index;
        const kf::RaycastCamera camera{.intrinsics = k.scaled(static_cast<unsigned int>(level_index)),
                                       .width = width / scale,
                                       .height = height / scale,
                                       .camera_to_world = tracked_pose};
        const kf::PyramidLevel level = d->pyramid->level(level_index);
        IcpConsumer consumer{*d->tracker, level.intrinsics, tracked_pose, iterations_per_level[level_index]};
        d->pipeline->track(camera, level, consumer);
        const kf::IcpOutcome& outcome = consumer.outcome();
        level_status[level_index] = status_of(outcome);
        tracked_pose = outcome.pose;
        if (!outcome.result) {
          ok = false;
          break;
        }
      }
      camera_to_world = tracked_pose;
    }
    if (ok) {
      kf::DepthFrame frame{.depth = &d->depth,
                           .color = color != nullptr ? &d->color : nullptr,
                           .normals = d->pyramid->host_normals(),
                           .intrinsics = k};
      const kf::DeviceDepthFrame* upload = d->pyramid->device_frame(frame);
      frame.world_to_camera = camera_to_world.inverse();
      d->pipeline->integrate(frame, upload);
    }
    *pose = to_rigid(camera_to_world);
    *tracked = ok ? 1 : 0;
  });
}

int kfr_dev_raycast(kfr_device* d, const kf_intrinsics* intrinsics, uint32_t width, uint32_t height,
                    const kf_rigid* camera_to_world, float* points, float* normals, uint32_t* colors) {
  return guarded([&] {
    const kf::RaycastCamera camera{.intrinsics = to_intrinsics(*intrinsics),
                                   .width = width,
                                   .height = height,
                                   .camera_to_world = to_matrix(*camera_to_world)};
    const kf::SurfaceMaps maps = d->pipeline->raycast(camera);
    copy_vec3_image(maps.points, points);
    copy_vec3_image(maps.normals, normals);
    if (colors != nullptr) {
      std::memcpy(colors, maps.colors.data().data(), maps.colors.data().size() * sizeof(uint32_t));
    }
  });
}

// Pipeline::host_view: the dense float (tsdf, weight) volume, x fastest.
int kfr_dev_host_view(kfr_device* d, float* voxels) {
  return guarded([&] {
    std::optional<kf::HostVolume> staging;
    const kf::ConstHostVolumeView v = d->pipeline->host_view(staging);
    std::memcpy(voxels, v.voxels, v.voxel_count() * sizeof(kf::Voxel));
  });
}

uint64_t kfr_dev_observed(const kfr_device* d) { return d->pipeline->observed_voxel_count(); }

int kfr_dev_synchronize(void) {
  return guarded([&] {
    if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("cudaDeviceSynchronize failed");
  });
}

}  // extern "C"
#endif  // KF_REF_CUDA
