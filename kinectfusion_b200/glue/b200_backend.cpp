// b200_backend.cpp - the reference's device seams defined over this library's
// C ABI (include/kf_b200.h), the file a maintainer adds to the reference in
// place of its src/kinectfusion/cuda/*.cu translation units.
//
// The reference picks its device backend at link time: a CPU-only build gets
// stubs (pipeline.cpp:120-127, depth_processing.cpp:59-72,
// tsdf_integration.cpp:9-13, icp_optimizer.cpp:171-206), a CUDA build the
// definitions in src/kinectfusion/cuda/.  Compiled with
// KINECTFUSION_HAS_CUDA beside the reference's own CPU translation units and
// linked with kinectfusion_b200/libkf_b200.so, this file provides:
//   * Pipeline::device_available / Pipeline::create_device
//     (pipeline.hpp:154-158, device_pipeline.cu:171-182): B200Pipeline;
//   * PyramidSource::create_device (depth_processing.hpp:460-462,
//     depth_processing.cu:169-172): B200PyramidSource;
//   * DepthUploader::create (tsdf_integration.hpp:108-109,
//     tsdf_integration.cu:180-182);
//   * BasicDeviceCorrespondenceSweep<Build>::{run, run_loop} and its special
//     members (icp_correspondence.hpp:352-377), which ProjectiveIcpTracker's
//     device requests call (icp_optimizer.cpp:58-160).
// Everything above the seams - the app's frame loop, the pipeline set, the
// tracker's host Gauss-Newton driver - is the reference's own code, unchanged.
// Errors map back to the reference's two exception kinds (validation.hpp:9-13,
// cuda/check.cuh:11-16).
#include <kf_b200.h>

#include <algorithm>
#include <array>
#include <cstdint>
#include <cstring>
#include <kinectfusion/depth_processing.hpp>
#include <kinectfusion/icp_correspondence.hpp>
#include <kinectfusion/marching_cubes.hpp>
#include <kinectfusion/pipeline.hpp>
#include <kinectfusion/raycasting.hpp>
#include <kinectfusion/tsdf_integration.hpp>
#include <kinectfusion/volume.hpp>
#include <memory>
#include <optional>
#include <stdexcept>
#include <type_traits>
#include <utility>
#include <variant>
#include <vector>

namespace kinectfusion {

// The reference leaves this upload type to its CUDA backend
// (tsdf_integration.hpp:88-91).  Here it names device buffers this library
// already holds: the pyramid's copy of the raw depth and its level-0 normals.
class DeviceDepthFrame {
 public:
  const std::uint16_t* depth = nullptr;  // device, width x height
  const float* normals = nullptr;        // device, width x height x 3
  kf_pyramid* pyramid = nullptr;         // the source of both (host copies on demand)
};

namespace {

void check(kf_status status) {
  if (status == KF_OK) return;
  if (status == KF_ERR_INVALID_ARGUMENT || status == KF_ERR_UNSUPPORTED) throw std::invalid_argument(kf_last_error());
  throw std::runtime_error(kf_last_error());
}

kf_rigid to_kf(const Eigen::Matrix4f& m) {
  kf_rigid r{};
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) r.r[i * 3 + j] = m(i, j);
    r.t[i] = m(i, 3);
  }
  return r;
}

kf_rigid to_kf(const RigidTransform& t) {
  const Vec3f rows[3] = {t.rotation.row_x, t.rotation.row_y, t.rotation.row_z};
  kf_rigid r{};
  for (int i = 0; i < 3; ++i) {
    r.r[i * 3 + 0] = rows[i].x;
    r.r[i * 3 + 1] = rows[i].y;
    r.r[i * 3 + 2] = rows[i].z;
  }
  r.t[0] = t.translation.x;
  r.t[1] = t.translation.y;
  r.t[2] = t.translation.z;
  return r;
}

RigidTransform from_kf(const kf_rigid& r) {
  return {.rotation = {.row_x = make_vec3f(r.r[0], r.r[1], r.r[2]),
                       .row_y = make_vec3f(r.r[3], r.r[4], r.r[5]),
                       .row_z = make_vec3f(r.r[6], r.r[7], r.r[8])},
          .translation = make_vec3f(r.t[0], r.t[1], r.t[2])};
}

kf_intrinsics to_kf(const CameraIntrinsics& k) { return {k.fx, k.fy, k.cx, k.cy}; }

CameraIntrinsics from_kf(const kf_intrinsics& k) {
  return CameraIntrinsics{.fx = k.fx, .fy = k.fy, .cx = k.cx, .cy = k.cy};
}

// PipelineConfig (pipeline.hpp:29-46) -> kf_pipeline_config: the storage,
// backend and mode enumerators share their order.
kf_pipeline_config to_kf(const PipelineConfig& c) {
  kf_pipeline_config k;
  kf_default_pipeline_config(&k);
  k.volume = {static_cast<uint32_t>(c.volume.resolution.x), static_cast<uint32_t>(c.volume.resolution.y),
              static_cast<uint32_t>(c.volume.resolution.z), c.volume.voxel_size,
              {c.volume.origin.x, c.volume.origin.y, c.volume.origin.z}, c.volume.truncation_distance};
  k.voxel = static_cast<int32_t>(c.voxel);
  k.color = static_cast<int32_t>(c.color);
  k.storage = static_cast<int32_t>(c.storage);
  k.sparse_block_capacity = c.sparse_block_capacity;
  k.tsdf_rule = std::holds_alternative<ClassicTsdf>(c.tsdf_rule) ? KF_RULE_CLASSIC : KF_RULE_ANGLE_WEIGHTED;
  k.integration = {c.integration.depth_scale,
                   c.integration.observation_weight,
                   c.integration.max_weight,
                   c.integration.min_depth,
                   c.integration.max_depth,
                   c.integration.projective_distance ? 1 : 0,
                   c.integration.distance_scaled_truncation ? 1 : 0,
                   c.integration.truncation_distance_scale,
                   static_cast<int32_t>(c.integration.mode)};
  k.raycast = {c.raycast.min_depth,
               c.raycast.max_depth,
               c.raycast.step_scale,
               static_cast<int32_t>(c.raycast.tsdf_corner_policy),
               c.raycast.cell_gradient_normals ? 1 : 0,
               c.raycast.seed_from_previous ? 1 : 0};
  k.raycast_backend = static_cast<int32_t>(c.raycast_backend);
  return k;
}

kf_raycast_camera to_kf(const RaycastCamera& cam) {
  return {to_kf(cam.intrinsics), static_cast<uint32_t>(cam.width), static_cast<uint32_t>(cam.height),
          to_kf(cam.camera_to_world)};
}

template <typename T>
image_proc::ImageView<const T, MemorySpace::kDevice> device_view(const void* data, std::size_t width,
                                                                std::size_t height) {
  return {.data = static_cast<const T*>(data), .width = width, .height = height};
}

// ---- the volume: Pipeline over kf_pipeline (device_pipeline.cu:26-167) --------------------
class B200Pipeline final : public Pipeline {
 public:
  explicit B200Pipeline(const PipelineConfig& config)
      : Pipeline(config.name), geometry_(config.volume), has_color_(config.color == ColorStore::kFloat) {
    const kf_pipeline_config k = to_kf(config);
    check(kf_pipeline_create(&k, &handle_));
  }
  ~B200Pipeline() override { kf_pipeline_destroy(handle_); }

  void integrate(const DepthFrame& frame, const DeviceDepthFrame* upload) override {
    TsdfIntegrator::validate_frame(frame);
    const std::size_t w = frame.depth->width(), h = frame.depth->height();
    const kf_intrinsics k = to_kf(frame.intrinsics);
    const kf_rigid w2c = to_kf(frame.world_to_camera);
    if (upload != nullptr && upload->depth != nullptr && !(has_color_ && frame.color != nullptr)) {
      // the frame is on the device already (the pyramid's upload); a volume
      // without colour ignores the frame's colour
      const kf_frame_view v{upload->depth, nullptr, upload->normals, static_cast<uint32_t>(w),
                            static_cast<uint32_t>(h), k, w2c, KF_MEMORY_DEVICE};
      check(kf_pipeline_integrate(handle_, &v));
      return;
    }
    // host inputs; a device upload without host normals lends them
    std::vector<float> normals;
    const float* n = frame.normals != nullptr ? &frame.normals->data().data()->x : nullptr;
    if (n == nullptr && upload != nullptr && upload->pyramid != nullptr) {
      normals.resize(w * h * 3);
      check(kf_pyramid_download_level(upload->pyramid, 0, nullptr, nullptr, normals.data()));
      n = normals.data();
    }
    const kf_frame_view v{frame.depth->data().data(), frame.color != nullptr ? frame.color->data().data() : nullptr,
                          n, static_cast<uint32_t>(w), static_cast<uint32_t>(h), k, w2c, KF_MEMORY_HOST};
    check(kf_pipeline_integrate(handle_, &v));
  }

  [[nodiscard]] SurfaceMaps raycast(const RaycastCamera& camera) override {
    Raycaster::validate_camera(camera);
    SurfaceMaps maps = SurfaceMaps::allocate(camera.width, camera.height);
    const kf_raycast_camera k = to_kf(camera);
    const kf_surface_maps out{&maps.points.data().data()->x, &maps.normals.data().data()->x,
                              maps.colors.data().data(), k.width, k.height, KF_MEMORY_HOST};
    check(kf_pipeline_raycast(handle_, &k, &out));
    return maps;
  }

  // The model rendered on the device at the camera; the tracker gets device
  // views of it and of the live level, valid during the call
  // (pipeline.hpp:82-85).
  void track(const RaycastCamera& camera, const PyramidLevel& live, TrackingSurfaceConsumer& consumer) override {
    Raycaster::validate_camera(camera);
    const kf_raycast_camera k = to_kf(camera);
    kf_surface_maps model{};
    check(kf_pipeline_render_model(handle_, &k, &model));
    const DeviceTrackingSurfaces surfaces{
        .live = std::get<ConstDeviceSurfaceView>(live.surface),
        .model = {.vertices = device_view<Vec3f>(model.points, model.width, model.height),
                  .normals = device_view<Vec3f>(model.normals, model.width, model.height)}};
    consumer.consume(surfaces);
  }

  [[nodiscard]] std::size_t observed_voxel_count() const override {
    uint64_t n = 0;
    check(kf_pipeline_observed_voxel_count(handle_, &n));
    return n;
  }

  // Dense float staging copy (volume_representation.hpp:95-115).
  [[nodiscard]] ConstHostVolumeView host_view(std::optional<HostVolume>& staging) const override {
    staging.emplace(geometry_);
    const HostVolumeView v = staging->view();
    const std::size_t n = v.voxel_count();
    // A colourless storage leaves the staging volume's colour facet as
    // allocated, as materialize does (volume_representation.hpp:119-129).
    std::vector<float> tsdf(n), weight(n), color(has_color_ && v.colors != nullptr ? n * 4 : 0);
    check(kf_pipeline_download_volume(handle_, tsdf.data(), weight.data(), color.empty() ? nullptr : color.data()));
    for (std::size_t i = 0; i < n; ++i) v.voxels[i] = Voxel{.distance = tsdf[i], .weight = weight[i]};
    if (!color.empty()) {
      for (std::size_t i = 0; i < n; ++i) {
        v.colors[i] = ColorVoxel{.color = make_vec3f(color[i * 4], color[i * 4 + 1], color[i * 4 + 2]),
                                 .weight = color[i * 4 + 3]};
      }
    }
    return staging->view();
  }

  [[nodiscard]] MarchingCubes::Mesh extract_mesh(float min_weight) const override {
    kf_mesh m{};
    check(kf_pipeline_extract_mesh(handle_, min_weight, &m));
    MarchingCubes::Mesh out;
    out.positions.resize(m.vertex_count);
    out.normals.resize(m.vertex_count);
    out.colors.resize(m.vertex_count);
    out.triangles.resize(m.triangle_count);
    for (uint64_t i = 0; i < m.vertex_count; ++i) {
      out.positions[i] = make_vec3f(m.positions[i * 3], m.positions[i * 3 + 1], m.positions[i * 3 + 2]);
      out.normals[i] = make_vec3f(m.normals[i * 3], m.normals[i * 3 + 1], m.normals[i * 3 + 2]);
      out.colors[i] = make_vec3f(m.colors[i * 3], m.colors[i * 3 + 1], m.colors[i * 3 + 2]);
    }
    for (uint64_t i = 0; i < m.triangle_count; ++i) {
      out.triangles[i] = {m.triangles[i * 3], m.triangles[i * 3 + 1], m.triangles[i * 3 + 2]};
    }
    kf_mesh_free(&m);
    return out;
  }

 private:
  kf_pipeline* handle_ = nullptr;
  VolumeGeometry geometry_;
  bool has_color_;
};

// ---- the depth pyramid: PyramidSource over kf_pyramid (depth_processing.cu:123-167) ------
class B200PyramidSource final : public PyramidSource {
 public:
  explicit B200PyramidSource(const DepthProcessingOptions& o) {
    const DepthProcessingOptions v = DepthProcessingOptions::validated(o);
    const kf_depth_options k{v.levels,
                             v.depth_scale,
                             v.min_depth,
                             v.max_depth,
                             v.max_normal_depth_jump,
                             v.max_downsample_depth_jump,
                             v.bilateral_filter ? 1 : 0,
                             v.bilateral_radius,
                             v.bilateral_spatial_sigma,
                             v.bilateral_depth_sigma};
    check(kf_pyramid_create(&k, &handle_));
  }
  ~B200PyramidSource() override { kf_pyramid_destroy(handle_); }

  std::size_t build(const image_proc::DepthImage& raw, const CameraIntrinsics& intrinsics) override {
    uint32_t levels = 0;
    check(kf_pyramid_build(handle_, raw.data().data(), static_cast<uint32_t>(raw.width()),
                           static_cast<uint32_t>(raw.height()), to_kf(intrinsics), KF_MEMORY_HOST, &levels));
    levels_ = levels;
    return levels;
  }

  [[nodiscard]] PyramidLevel level(std::size_t index) const override {
    kf_level_view v{};
    check(kf_pyramid_level(handle_, static_cast<uint32_t>(index), &v));
    return {.surface = ConstDeviceSurfaceView{.vertices = device_view<Vec3f>(v.vertices, v.width, v.height),
                                              .normals = device_view<Vec3f>(v.normals, v.width, v.height)},
            .intrinsics = from_kf(v.intrinsics)};
  }

  [[nodiscard]] const image_proc::Vector3fImage* host_normals() const override { return nullptr; }

  [[nodiscard]] const DeviceDepthFrame* device_frame(const DepthFrame& /*frame*/) override {
    if (levels_ == 0) return nullptr;
    kf_level_view v{};
    check(kf_pyramid_level(handle_, 0, &v));
    check(kf_pyramid_raw_depth(handle_, &frame_.depth));
    frame_.normals = v.normals;
    frame_.pyramid = handle_;
    return &frame_;
  }

 private:
  kf_pyramid* handle_ = nullptr;
  std::size_t levels_ = 0;
  DeviceDepthFrame frame_;
};

// Frames of a pipeline set with no pyramid upload: integration reads host
// memory (kf_pipeline_integrate stages it), so the "upload" carries nothing.
class B200DepthUploader final : public DepthUploader {
 public:
  [[nodiscard]] const DeviceDepthFrame& upload(const DepthFrame& /*frame*/) override { return frame_; }

 private:
  DeviceDepthFrame frame_;
};

// The fields of CorrespondenceSearch<kDevice> (icp_correspondence.hpp:
// 221-301), which the reference's own sweep hands to its kernel by value.
struct SearchFields {
  DeviceTrackingSurfaces surfaces;
  CameraIntrinsics intrinsics;
  IcpIterationTransforms transforms;
  CorrespondenceGates gates;
};
static_assert(sizeof(SearchFields) == sizeof(DeviceCorrespondenceSearch) &&
                  std::is_trivially_copyable_v<DeviceCorrespondenceSearch>,
              "CorrespondenceSearch's layout is its four members in order");

SearchFields fields_of(const DeviceCorrespondenceSearch& search) {
  SearchFields f;
  std::memcpy(&f, &search, sizeof(f));
  return f;
}

kf_level_view live_view(const SearchFields& f) {
  const auto& live = f.surfaces.live;
  return {nullptr, &live.vertices.data->x, &live.normals.data->x, static_cast<uint32_t>(live.vertices.width),
          static_cast<uint32_t>(live.vertices.height), {}};
}

}  // namespace

// ---- link seams ---------------------------------------------------------------------------
bool Pipeline::device_available() {
  int32_t available = 0;
  return kf_device_available(&available) == KF_OK && available != 0;
}

std::unique_ptr<Pipeline> Pipeline::create_device(const PipelineConfig& config) {
  return std::make_unique<B200Pipeline>(config);
}

std::unique_ptr<PyramidSource> PyramidSource::create_device(const DepthProcessingOptions& options) {
  return std::make_unique<B200PyramidSource>(options);
}

std::unique_ptr<DepthUploader> DepthUploader::create() { return std::make_unique<B200DepthUploader>(); }

// Field by field (a struct's padding bytes are arbitrary).
inline bool same_options(const kf_icp_options& a, const kf_icp_options& b) {
  return a.min_correspondences == b.min_correspondences && a.max_point_distance == b.max_point_distance &&
         a.min_normal_dot == b.min_normal_dot && a.min_update_translation == b.min_update_translation &&
         a.min_update_rotation == b.min_update_rotation && a.max_update_translation == b.max_update_translation &&
         a.max_update_rotation == b.max_update_rotation && a.min_system_eigenvalue == b.min_system_eigenvalue &&
         a.max_condition_number == b.max_condition_number && a.damping_mode == b.damping_mode &&
         a.damping_lambda == b.damping_lambda && a.adaptive_damping == b.adaptive_damping &&
         a.lambda_increase == b.lambda_increase && a.lambda_decrease == b.lambda_decrease &&
         a.min_lambda == b.min_lambda && a.max_lambda == b.max_lambda;
}

// The sweep's scratch: one tracker of this library per sweep (its device
// state and partial sums), re-created only when the options it would be
// created with change.
template <GraphBuildStrategy Build>
struct BasicDeviceCorrespondenceSweep<Build>::Scratch {
  kf_tracker* tracker = nullptr;
  kf_icp_options options{};

  ~Scratch() {
    if (tracker != nullptr) kf_tracker_destroy(tracker);
  }

  kf_tracker* for_search(const CorrespondenceGates& g, const DeviceIcpLoopParams* p) {
    kf_icp_options o{};
    kf_default_icp_options(&o);
    o.max_point_distance = g.max_point_distance;
    o.min_normal_dot = g.min_normal_dot;
    if (p != nullptr) {
      // the device loop's own gates (DeviceIcpLoopParams, icp_correspondence.hpp:324-333)
      o.min_correspondences = p->min_correspondences;
      o.min_update_translation = p->min_update_translation;
      o.min_update_rotation = p->min_update_rotation;
      o.max_update_translation = p->max_update_translation;
      o.max_update_rotation = p->max_update_rotation;
      o.damping_mode = static_cast<int32_t>(p->damping.mode);
      o.damping_lambda = p->damping.lambda;
      o.adaptive_damping = p->adaptive_damping ? 1 : 0;
      o.lambda_increase = p->schedule.increase;
      o.lambda_decrease = p->schedule.decrease;
      o.min_lambda = p->schedule.min_lambda;
      o.max_lambda = p->schedule.max_lambda;
    } else if (tracker != nullptr) {
      // a plain sweep uses only the gates: keep the loop options in place
      kf_icp_options kept = options;
      kept.max_point_distance = o.max_point_distance;
      kept.min_normal_dot = o.min_normal_dot;
      o = kept;
    }
    if (tracker != nullptr && same_options(o, options)) return tracker;
    if (tracker != nullptr) kf_tracker_destroy(tracker);
    tracker = nullptr;
    check(kf_tracker_create(&o, &tracker));
    options = o;
    return tracker;
  }
};

template <GraphBuildStrategy Build>
BasicDeviceCorrespondenceSweep<Build>::BasicDeviceCorrespondenceSweep() : scratch_(std::make_unique<Scratch>()) {}
template <GraphBuildStrategy Build>
BasicDeviceCorrespondenceSweep<Build>::~BasicDeviceCorrespondenceSweep() = default;
template <GraphBuildStrategy Build>
BasicDeviceCorrespondenceSweep<Build>::BasicDeviceCorrespondenceSweep(BasicDeviceCorrespondenceSweep&&) noexcept =
    default;
template <GraphBuildStrategy Build>
BasicDeviceCorrespondenceSweep<Build>& BasicDeviceCorrespondenceSweep<Build>::operator=(
    BasicDeviceCorrespondenceSweep&&) noexcept = default;

// One sweep on the device: the 29 sums and the count of the reference's
// IcpNormalEquations (icp_correspondence.hpp:104-176), reduced in a fixed
// order on the device instead of FP32 atomics.
template <GraphBuildStrategy Build>
IcpNormalEquations BasicDeviceCorrespondenceSweep<Build>::run(const DeviceCorrespondenceSearch& search) {
  const SearchFields f = fields_of(search);
  kf_tracker* tracker = scratch_->for_search(f.gates, nullptr);
  const kf_level_view live = live_view(f);
  const auto& model = f.surfaces.model;
  const kf_rigid camera = to_kf(f.transforms.camera);
  const kf_rigid model_w2c = to_kf(f.transforms.model);
  std::array<float, 29> sums{};
  uint64_t count = 0;
  check(kf_icp_normal_equations(tracker, &live, &model.vertices.data->x, &model.normals.data->x,
                                static_cast<uint32_t>(model.vertices.width),
                                static_cast<uint32_t>(model.vertices.height), to_kf(f.intrinsics), &camera,
                                &model_w2c, sums.data(), &count));
  IcpNormalEquations e;
  e.count = count;
  std::copy_n(sums.begin(), kIcpUpperTriangleSize, e.jtj.begin());
  std::copy_n(sums.begin() + kIcpUpperTriangleSize, kIcpDof, e.jtr.begin());
  e.distance_sum = sums[27];
  e.residual_sum_squares = sums[28];
  return e;
}

// The whole level on the device (--icp-device-solve): this library's device
// Gauss-Newton loop with its FP64 solve and the same gates, one sync.
template <GraphBuildStrategy Build>
DeviceIcpLoopResult BasicDeviceCorrespondenceSweep<Build>::run_loop(const DeviceCorrespondenceSearch& search,
                                                                    unsigned int iterations,
                                                                    const DeviceIcpLoopParams& params) {
  const SearchFields f = fields_of(search);
  kf_tracker* tracker = scratch_->for_search(f.gates, &params);
  const kf_level_view live = live_view(f);
  const auto& model = f.surfaces.model;
  const kf_rigid model_w2c = to_kf(f.transforms.model);
  const kf_rigid initial = to_kf(f.transforms.camera);
  kf_icp_outcome o{};
  std::array<float, 29> sums{};
  check(kf_icp_level(tracker, &live, &model.vertices.data->x, &model.normals.data->x,
                     static_cast<uint32_t>(model.vertices.width), static_cast<uint32_t>(model.vertices.height),
                     to_kf(f.intrinsics), &model_w2c, &initial, iterations, &o, sums.data()));
  DeviceIcpLoopResult r{};
  r.transforms = {.camera = from_kf(o.pose), .model = f.transforms.model};
  r.equations.count = o.correspondences;
  std::copy_n(sums.begin(), kIcpUpperTriangleSize, r.equations.jtj.begin());
  std::copy_n(sums.begin() + kIcpUpperTriangleSize, kIcpDof, r.equations.jtr.begin());
  r.equations.distance_sum = sums[27];
  r.equations.residual_sum_squares = sums[28];
  r.best_camera = r.transforms.camera;
  r.lambda = o.damping_lambda;
  r.trials = o.iterations;
  r.rejected = static_cast<std::int32_t>(o.rejected_steps);
  r.update_translation = o.update_translation;
  r.update_rotation = o.update_rotation;
  // IcpFailure order of DeviceIcpLoopResult::status (icp_correspondence.hpp:335-346)
  switch (o.status) {
    case KF_ICP_CONVERGED:
      r.status = 1;
      break;
    case KF_ICP_TOO_FEW_CORRESPONDENCES:
      r.status = 2;
      break;
    case KF_ICP_SOLVE_FAILED:
      r.status = 3;
      break;
    case KF_ICP_UPDATE_TOO_LARGE:
      r.status = 4;
      break;
    default:
      r.status = 0;
      break;
  }
  return r;
}

template class BasicDeviceCorrespondenceSweep<ExplicitGraphBuild>;
template class BasicDeviceCorrespondenceSweep<CapturedGraphBuild>;

}  // namespace kinectfusion
