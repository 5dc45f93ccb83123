// kf_api.cu - C ABI entry points (include/kf_b200.h) for pipelines, trackers
// and the whole-frame CUDA graph.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "kf_internal.h"

namespace kf {

namespace {
thread_local std::string g_last_error;

void validate_geometry(const kf_volume_geometry& g) {
  // BasicVolume::validated (volume.hpp:496-507)
  require(g.res_x > 0 && g.res_y > 0 && g.res_z > 0, "Volume resolution must be positive");
  require(g.voxel_size > 0.0f, "Voxel size must be positive");
  require(g.truncation_distance > 0.0f, "Truncation distance must be positive");
  require(std::isfinite(g.origin[0]) && std::isfinite(g.origin[1]) && std::isfinite(g.origin[2]),
          "Volume origin must be finite");
}

void validate_integration(const kf_integration_options& o) {
  // TsdfIntegrator::validated (tsdf_integration.cpp:25-37)
  require(o.depth_scale > 0.0f, "Depth scale must be positive");
  require(o.observation_weight > 0.0f, "Observation weight must be positive");
  require(o.max_weight > 0.0f, "Max weight must be positive");
  require(o.min_depth >= 0.0f && o.max_depth > o.min_depth, "Depth range is invalid");
  require(o.truncation_distance_scale >= 0.0f, "Truncation distance scale must be non-negative");
}

void validate_raycast(const kf_raycast_options& o) {
  // Raycaster::validated (raycasting.cpp:15-20)
  require(o.min_depth >= 0.0f && o.max_depth > o.min_depth, "Raycast depth range is invalid");
  require(o.step_scale > 0.0f, "Raycast step scale must be positive");
}

bool rigid_finite(const kf_rigid& r) {
  for (float v : r.r)
    if (!std::isfinite(v)) return false;
  for (float v : r.t)
    if (!std::isfinite(v)) return false;
  return true;
}

void validate_camera(const kf_raycast_camera& c) {
  // Raycaster::validate_camera (raycasting.cpp:22-30)
  require(c.intrinsics.fx > 0.0f && c.intrinsics.fy > 0.0f, "Raycast intrinsics must have positive focal lengths");
  require(c.width > 0u && c.height > 0u, "Raycast dimensions must be positive");
  require(rigid_finite(c.camera_to_world), "Raycast camera_to_world must be finite");
}

void validate_frame(const kf_frame_view& f) {
  // TsdfIntegrator::validate_frame (tsdf_integration.cpp:39-48)
  require(f.depth != nullptr, "Depth frame requires a depth image");
  require(f.width > 0u && f.height > 0u, "Depth frame depth image must be non-empty");
  require(f.intrinsics.fx > 0.0f && f.intrinsics.fy > 0.0f, "Depth frame intrinsics must have positive focal lengths");
  require(rigid_finite(f.world_to_camera), "Depth frame world_to_camera must be finite");
}

size_t voxel_bytes_of(int kind) { return kind == KF_VOXEL_FLOAT ? 8 : 4; }

template <typename T>
const T* stage(const T* src, size_t count, int memory, DeviceArray<T>& own, cudaStream_t s) {
  if (src == nullptr) return nullptr;
  if (memory == KF_MEMORY_DEVICE) return src;
  if (own.count != count) own.resize(count);
  check(cudaMemcpyAsync(own.ptr, src, count * sizeof(T), cudaMemcpyHostToDevice, s), "frame upload");
  return own.ptr;
}

kf_rigid rigid_of_state(const IcpState& st) {
  kf_rigid r;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) r.r[i * 3 + j] = static_cast<float>(st.pose[i * 4 + j]);
    r.t[i] = static_cast<float>(st.pose[i * 4 + 3]);
  }
  return r;
}

void fill_outcome(const IcpState& st, kf_icp_outcome* out) {
  out->pose = rigid_of_state(st);
  for (int i = 0; i < 12; ++i) out->pose_f64[i] = st.pose[i];
  out->status = st.status;
  out->iterations = st.iterations;
  out->correspondences = st.correspondences;
  out->mean_point_distance = st.mean_point_distance;
  out->mean_squared_residual = st.mean_squared_residual;
  out->min_system_eigenvalue = st.min_system_eigenvalue;
  out->condition_number = st.condition_number;
  out->update_translation = st.update_translation;
  out->update_rotation = st.update_rotation;
  out->damping_lambda = st.damping_lambda;
  out->rejected_steps = st.rejected_steps;
}

}  // namespace

void set_last_error(const std::string& message) { g_last_error = message; }

void check(cudaError_t status, const char* what) {
  if (status != cudaSuccess) {
    throw CudaError(std::string(what) + ": " + cudaGetErrorString(status));
  }
}

void require(bool condition, const char* what) {
  if (!condition) throw InvalidArgument(what);
}

Pipeline::Maps& Pipeline::maps_for(uint32_t w, uint32_t h) {
  Maps& m = maps[{w, h}];
  const size_t n = static_cast<size_t>(w) * h;
  if (m.points.count != n * 3) {
    m.points.resize(n * 3);
    m.normals.resize(n * 3);
    m.colors.resize(n);
  }
  return m;
}

void Pipeline::clear_graphs() {
  for (auto& kv : graphs) {
    cudaGraphExecDestroy(kv.second.exec);
    cudaGraphDestroy(kv.second.graph);
  }
  ++graph_epoch;
  graphs.clear();
}

}  // namespace kf

using namespace kf;

extern "C" {

const char* kf_last_error(void) { return g_last_error.c_str(); }

int kf_abi_version(void) { return KF_B200_ABI_VERSION; }

kf_status kf_device_available(int32_t* available) {
  // Pipeline::device_available (device_pipeline.cu:171-174)
  return guarded([&] {
    require(available != nullptr, "kf_device_available: null argument");
    int count = 0;
    *available = (cudaGetDeviceCount(&count) == cudaSuccess && count > 0) ? 1 : 0;
  });
}

void kf_default_integration_options(kf_integration_options* o) {
  // TsdfIntegrationOptions defaults (tsdf_integration.hpp:21-50)
  o->depth_scale = 5000.0f;
  o->observation_weight = 1.0f;
  o->max_weight = 196.0f;
  o->min_depth = 0.4f;
  o->max_depth = 8.0f;
  o->projective_distance = 1;
  o->distance_scaled_truncation = 0;
  o->truncation_distance_scale = 0.01f;
  o->mode = KF_INTEGRATION_FULL;
}

void kf_default_raycast_options(kf_raycast_options* o) {
  // RaycastOptions defaults (raycasting.hpp:66-78)
  o->min_depth = 0.4f;
  o->max_depth = 8.0f;
  o->step_scale = 1.0f;
  o->corner_policy = KF_CORNERS_SKIP_MISSING;
  o->cell_gradient_normals = 0;
  o->seed_from_previous = 0;
}

void kf_default_icp_options(kf_icp_options* o) {
  // ProjectiveIcpOptions defaults (icp_optimizer.hpp:14-20, 80-101) and
  // icp_correspondence.hpp:24-34.
  o->min_correspondences = 64;
  o->max_point_distance = 0.05f;
  o->min_normal_dot = 0.9659258f;
  o->min_update_translation = 1.0e-5f;
  o->min_update_rotation = 1.0e-5f;
  o->max_update_translation = 0.15f;
  o->max_update_rotation = 0.35f;
  o->min_system_eigenvalue = 1.0e-6f;
  o->max_condition_number = 1.0e6f;
  o->damping_mode = KF_DAMPING_NONE;
  o->damping_lambda = 1.0e-3f;
  o->adaptive_damping = 0;
  o->lambda_increase = 10.0f;
  o->lambda_decrease = 0.1f;
  o->min_lambda = 1.0e-9f;
  o->max_lambda = 1.0e6f;
}

void kf_default_pipeline_config(kf_pipeline_config* c) {
  // PipelineConfig defaults (pipeline.hpp:29-46)
  std::memset(c, 0, sizeof(*c));
  c->voxel = KF_VOXEL_FLOAT;
  c->color = KF_COLOR_FLOAT;
  c->storage = KF_STORAGE_DENSE;
  c->sparse_block_capacity = 0;
  c->tsdf_rule = KF_RULE_ANGLE_WEIGHTED;
  kf_default_integration_options(&c->integration);
  kf_default_raycast_options(&c->raycast);
  c->raycast_backend = KF_RAYCAST_MARCH;
}

kf_status kf_pipeline_create(const kf_pipeline_config* config, kf_pipeline** out) {
  return guarded([&] {
    require(config != nullptr && out != nullptr, "kf_pipeline_create: null argument");
    const kf_pipeline_config& c = *config;
    // Pipeline::create + require_valid_storage (pipeline.cpp:104-147)
    if (c.storage == KF_STORAGE_SPARSE) {
      require(c.integration.mode == KF_INTEGRATION_BAND,
              "Sparse storage implies band integration (nothing is allocated far from surfaces); set "
              "integration = 'band'");
      require(c.raycast_backend == KF_RAYCAST_MARCH, "Sparse storage supports the plain march raycast backend");
    }
    validate_geometry(c.volume);
    validate_integration(c.integration);
    validate_raycast(c.raycast);
    require(c.voxel >= KF_VOXEL_FLOAT && c.voxel <= KF_VOXEL_BF16, "Unknown voxel store");
    require(c.color == KF_COLOR_FLOAT || c.color == KF_COLOR_NONE, "Unknown color store");
    require(c.tsdf_rule == KF_RULE_CLASSIC || c.tsdf_rule == KF_RULE_ANGLE_WEIGHTED, "Unknown TSDF rule");
    require(c.raycast_backend >= KF_RAYCAST_MARCH && c.raycast_backend <= KF_RAYCAST_BAND_MARCH,
            "Unknown raycast backend");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
      throw CudaError("no CUDA device available");
    }
    auto* h = new kf_pipeline();
    try {
      Pipeline& p = h->impl;
      p.config = c;
      check(cudaStreamCreateWithFlags(&p.stream, cudaStreamNonBlocking), "cudaStreamCreate");
      const kf_volume_geometry& g = c.volume;
      const uint64_t blocks = static_cast<uint64_t>((g.res_x + 7) / 8) * ((g.res_y + 7) / 8) * ((g.res_z + 7) / 8);
      require(blocks < 0xFFFFFFFFull, "Volume has too many blocks");
      // bricked storage: whole 8^3 bricks (edge blocks padded); a sparse
      // volume holds its pool of `capacity` bricks (BlockRep, block_rep.cu:76-96,
      // default capacity = blocks / 4)
      if (c.storage == KF_STORAGE_SPARSE) {
        p.sparse_capacity = c.sparse_block_capacity != 0 ? c.sparse_block_capacity : blocks / 4;
        require(p.sparse_capacity > 0 && p.sparse_capacity < 0xFFFFFFFFull, "Sparse block capacity out of range");
        p.voxel_count = p.sparse_capacity * 512;
        // the voxel-block hash: a power of two >= 2 x capacity entries
        uint64_t entries = 1024;
        while (entries < 2 * p.sparse_capacity) entries <<= 1;
        require(entries <= (1ull << 32), "Sparse block capacity out of range");
        p.block_table.resize(entries);
        p.null_bricks.resize(blocks);
        p.slot_block.resize(p.sparse_capacity);
        p.allocated.resize(2);
      } else {
        p.voxel_count = blocks * 512;
      }
      p.voxel_bytes = voxel_bytes_of(c.voxel);
      p.voxels.resize(p.voxel_count * p.voxel_bytes);
      if (c.color == KF_COLOR_FLOAT) p.colors.resize(p.voxel_count);
      VolumeDev& v = p.view;
      v.voxels = p.voxels.ptr;
      v.colors = c.color == KF_COLOR_FLOAT ? p.colors.ptr : nullptr;
      v.table = c.storage == KF_STORAGE_SPARSE ? p.block_table.ptr : nullptr;
      v.table_mask = c.storage == KF_STORAGE_SPARSE ? static_cast<uint32_t>(p.block_table.count - 1) : 0u;
      v.rx = g.res_x;
      v.ry = g.res_y;
      v.rz = g.res_z;
      v.bx = (g.res_x + 7) / 8;
      v.by = (g.res_y + 7) / 8;
      v.bz = (g.res_z + 7) / 8;
      v.voxel_size = g.voxel_size;
      v.inv_voxel_size = 1.0f / g.voxel_size;
      v.origin = make(g.origin[0], g.origin[1], g.origin[2]);
      v.truncation = g.truncation_distance;
      launch_fill_volume(p, p.stream);
      reset_sparse(p, p.stream);
      if (c.raycast_backend == KF_RAYCAST_BAND_MARCH) {
        // EmptySpaceIndex (raycasting.hpp:31-38): the band bitmap, empty for
        // a fresh (unobserved) volume
        const size_t words = static_cast<size_t>((blocks + 31) / 32);
        p.band_raw.resize(words);
        p.band_map.resize(words);
        check(cudaMemsetAsync(p.band_raw.ptr, 0, p.band_raw.bytes(), p.stream), "band bitmap init");
        check(cudaMemsetAsync(p.band_map.ptr, 0, p.band_map.bytes(), p.stream), "band bitmap init");
      }
      p.counters.resize(2);
      check(cudaMemsetAsync(p.counters.ptr, 0, p.counters.bytes(), p.stream), "counter init");
      check(cudaStreamSynchronize(p.stream), "volume fill");
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

kf_status kf_pipeline_destroy(kf_pipeline* pipeline) {
  return guarded([&] {
    if (pipeline == nullptr) return;
    Pipeline& p = pipeline->impl;
    if (p.stream) cudaStreamSynchronize(p.stream);
    p.clear_graphs();
    if (p.staging_done) cudaEventDestroy(p.staging_done);
    if (p.copy_stream) cudaStreamSynchronize(p.copy_stream);
    for (int i = 0; i < 2; ++i) {
      if (p.uploaded[i]) cudaEventDestroy(p.uploaded[i]);
      if (p.consumed[i]) cudaEventDestroy(p.consumed[i]);
    }
    if (p.copy_stream) cudaStreamDestroy(p.copy_stream);
    for (cudaEvent_t e : {p.fork_event, p.pyramid_event, p.inputs_event}) {
      if (e) cudaEventDestroy(e);
    }
    if (p.side_stream) cudaStreamDestroy(p.side_stream);
    for (cudaEvent_t e : p.result_ready) {
      if (e) cudaEventDestroy(e);
    }
    if (p.stream) cudaStreamDestroy(p.stream);
    delete pipeline;
  });
}

static void enqueue_reset(Pipeline& p) {
  launch_fill_volume(p, p.stream);
  reset_sparse(p, p.stream);
  reset_blocks(p, p.stream);  // the raycast's skip structures describe the volume
  if (p.band_map.count) {
    check(cudaMemsetAsync(p.band_raw.ptr, 0, p.band_raw.bytes(), p.stream), "band bitmap reset");
    check(cudaMemsetAsync(p.band_map.ptr, 0, p.band_map.bytes(), p.stream), "band bitmap reset");
  }
  check(cudaMemsetAsync(p.counters.ptr, 0, p.counters.bytes(), p.stream), "counter reset");
}

kf_status kf_pipeline_reset(kf_pipeline* pipeline) {
  return guarded([&] {
    require(pipeline != nullptr, "kf_pipeline_reset: null pipeline");
    enqueue_reset(pipeline->impl);
    check(cudaStreamSynchronize(pipeline->impl.stream), "volume reset");
  });
}

kf_status kf_pipeline_reset_async(kf_pipeline* pipeline) {
  return guarded([&] {
    require(pipeline != nullptr, "kf_pipeline_reset_async: null pipeline");
    enqueue_reset(pipeline->impl);
  });
}

kf_status kf_pipeline_integrate(kf_pipeline* pipeline, const kf_frame_view* frame) {
  return guarded([&] {
    require(pipeline != nullptr && frame != nullptr, "kf_pipeline_integrate: null argument");
    validate_frame(*frame);
    Pipeline& p = pipeline->impl;
    const kf_frame_view& f = *frame;
    const size_t n = static_cast<size_t>(f.width) * f.height;
    const uint16_t* depth = stage(f.depth, n, f.memory, p.own_depth, p.stream);
    const uint32_t* color = stage(f.color, n, f.memory, p.own_color, p.stream);
    const float* normals = stage(f.normals, n * 3, f.memory, p.own_normals, p.stream);
    if (p.pixel_table.count != n) p.pixel_table.resize(n);
    const Intr k = intr_from(f.intrinsics);
    launch_pixel_table(depth, color, normals, f.width, f.height, k, p.config.integration, p.config.tsdf_rule,
                       p.pixel_table.ptr, p.stream);
    launch_integrate(p, p.pixel_table.ptr, f.width, f.height, k, rigid_from(f.world_to_camera),
                     color != nullptr, nullptr, p.stream);
    check(cudaStreamSynchronize(p.stream), "integrate");
  });
}

kf_status kf_pipeline_raycast(kf_pipeline* pipeline, const kf_raycast_camera* camera, const kf_surface_maps* out) {
  return guarded([&] {
    require(pipeline != nullptr && camera != nullptr && out != nullptr, "kf_pipeline_raycast: null argument");
    validate_camera(*camera);
    require(out->width == camera->width && out->height == camera->height,
            "kf_pipeline_raycast: output maps must match the camera extent");
    require(out->points != nullptr && out->normals != nullptr && out->colors != nullptr,
            "kf_pipeline_raycast: null output map");
    Pipeline& p = pipeline->impl;
    const size_t n = static_cast<size_t>(camera->width) * camera->height;
    if (out->memory == KF_MEMORY_DEVICE) {
      launch_raycast(p, *camera, out->points, out->normals, out->colors, nullptr, p.stream);
    } else {
      Pipeline::Maps& m = p.maps_for(camera->width, camera->height);
      if (p.config.raycast.seed_from_previous) {
        check(cudaMemcpyAsync(m.points.ptr, out->points, n * 3 * sizeof(float), cudaMemcpyHostToDevice, p.stream),
              "seed upload");
      }
      launch_raycast(p, *camera, m.points.ptr, m.normals.ptr, m.colors.ptr, nullptr, p.stream);
      check(cudaMemcpyAsync(out->points, m.points.ptr, n * 3 * sizeof(float), cudaMemcpyDeviceToHost, p.stream),
            "points download");
      check(cudaMemcpyAsync(out->normals, m.normals.ptr, n * 3 * sizeof(float), cudaMemcpyDeviceToHost, p.stream),
            "normals download");
      check(cudaMemcpyAsync(out->colors, m.colors.ptr, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, p.stream),
            "colors download");
    }
    check(cudaStreamSynchronize(p.stream), "raycast");
  });
}

kf_status kf_pipeline_observed_voxel_count(kf_pipeline* pipeline, uint64_t* count) {
  return guarded([&] {
    require(pipeline != nullptr && count != nullptr, "kf_pipeline_observed_voxel_count: null argument");
    *count = count_observed(pipeline->impl);
  });
}

namespace {
// The block -> slot map of a sparse volume as a dense host array (one entry
// per block, kUnallocated when none), expanded from the device's voxel-block
// hash: the layout of the reference's block grid (block_rep.hpp:26-39).
std::vector<uint32_t> host_block_grid(const Pipeline& p) {
  std::vector<unsigned long long> table(p.block_table.count);
  check(cudaMemcpy(table.data(), p.block_table.ptr, table.size() * sizeof(unsigned long long),
                   cudaMemcpyDeviceToHost), "block table download");
  std::vector<uint32_t> grid(static_cast<size_t>(p.view.bx) * p.view.by * p.view.bz, kUnallocated);
  for (const unsigned long long e : table) {
    if (e == kEmptyEntry) continue;
    const uint32_t block = static_cast<uint32_t>(e >> 32);
    if (block < grid.size()) grid[block] = static_cast<uint32_t>(e);
  }
  return grid;
}

// Copies the bricked device volume to the host in the reference's x-fastest
// order (Size3::flatten, vector.hpp:61-67): elem_bytes per voxel.  Sparse
// volumes resolve each block through the block table; unallocated blocks read as
// `unallocated` (elem_bytes of an unobserved voxel).
void download_dense(const Pipeline& p, const void* device, size_t elem_bytes, void* out, const void* unallocated) {
  const kf_volume_geometry& g = p.config.volume;
  const uint64_t bx = (g.res_x + 7) / 8, by = (g.res_y + 7) / 8, bz = (g.res_z + 7) / 8;
  const bool sparse = p.view.table != nullptr;
  std::vector<uint8_t> raw((sparse ? p.sparse_capacity : bx * by * bz) * 512 * elem_bytes);
  check(cudaMemcpy(raw.data(), device, raw.size(), cudaMemcpyDeviceToHost), "volume download");
  std::vector<uint32_t> grid;
  if (sparse) grid = host_block_grid(p);
  uint8_t* dst = static_cast<uint8_t*>(out);
  for (uint64_t z = 0; z < g.res_z; ++z) {
    for (uint64_t y = 0; y < g.res_y; ++y) {
      for (uint64_t x0 = 0; x0 < g.res_x; x0 += 8) {
        const uint64_t block = ((z / 8) * by + (y / 8)) * bx + (x0 / 8);
        const uint64_t n = std::min<uint64_t>(8, g.res_x - x0);
        uint8_t* d = dst + ((z * g.res_y + y) * g.res_x + x0) * elem_bytes;
        const uint64_t slot = sparse ? grid[block] : block;
        if (sparse && grid[block] == kUnallocated) {
          for (uint64_t i = 0; i < n; ++i) std::memcpy(d + i * elem_bytes, unallocated, elem_bytes);
          continue;
        }
        const uint64_t src = (slot * 512 + ((z % 8) * 8 + (y % 8)) * 8) * elem_bytes;
        std::memcpy(d, raw.data() + src, n * elem_bytes);
      }
    }
  }
}

// Raw bytes of an unobserved voxel (volume.hpp:115-117) and colour.
struct Unobserved {
  uint8_t voxel[8];
  uint8_t color[16];
};
Unobserved unobserved_of(int kind) {
  Unobserved u{};
  if (kind == KF_VOXEL_FLOAT) {
    const float f[2] = {1.0f, 0.0f};
    std::memcpy(u.voxel, f, 8);
  } else {
    const uint32_t r = kind == KF_VOXEL_QUANTIZED ? 32767u : 0x3F80u;
    std::memcpy(u.voxel, &r, 4);
  }
  return u;
}
}  // namespace

kf_status kf_pipeline_block_stats(kf_pipeline* pipeline, uint64_t* attempts, uint64_t* capacity) {
  return guarded([&] {
    require(pipeline != nullptr && attempts != nullptr && capacity != nullptr,
            "kf_pipeline_block_stats: null argument");
    Pipeline& p = pipeline->impl;
    check(cudaStreamSynchronize(p.stream), "block stats sync");
    *attempts = 0;
    *capacity = p.sparse_capacity;
    if (p.allocated.count != 0) {
      check(cudaMemcpy(attempts, p.allocated.ptr, sizeof(uint64_t), cudaMemcpyDeviceToHost), "block stats");
    }
  });
}

kf_status kf_pipeline_listed_blocks(kf_pipeline* pipeline, uint64_t* blocks) {
  return guarded([&] {
    require(pipeline != nullptr && blocks != nullptr, "kf_pipeline_listed_blocks: null argument");
    Pipeline& p = pipeline->impl;
    check(cudaStreamSynchronize(p.stream), "listed blocks sync");
    unsigned n = 0;
    if (p.block_count.count != 0) {
      check(cudaMemcpy(&n, p.block_count.ptr, sizeof(unsigned), cudaMemcpyDeviceToHost), "listed blocks");
    }
    *blocks = n;
  });
}

kf_status kf_pipeline_download_block_grid(kf_pipeline* pipeline, uint32_t* grid, size_t count) {
  return guarded([&] {
    require(pipeline != nullptr && grid != nullptr, "kf_pipeline_download_block_grid: null argument");
    Pipeline& p = pipeline->impl;
    require(p.block_table.count != 0, "kf_pipeline_download_block_grid: the pipeline is not sparse");
    require(count == static_cast<size_t>(p.view.bx) * p.view.by * p.view.bz,
            "kf_pipeline_download_block_grid: grid size mismatch");
    check(cudaStreamSynchronize(p.stream), "grid download sync");
    const std::vector<uint32_t> dense = host_block_grid(p);
    std::memcpy(grid, dense.data(), count * sizeof(uint32_t));
  });
}

kf_status kf_pipeline_download_skip_structures(kf_pipeline* pipeline, uint8_t* brick_class, uint8_t* brick_radius,
                                               uint32_t* records, size_t bricks) {
  return guarded([&] {
    require(pipeline != nullptr && brick_class != nullptr && brick_radius != nullptr && records != nullptr,
            "kf_pipeline_download_skip_structures: null argument");
    Pipeline& p = pipeline->impl;
    require(p.view.table == nullptr && p.brick_class.count != 0 && p.brick_radius.count != 0,
            "kf_pipeline_download_skip_structures: no skip structures (sparse storage, or no integration yet)");
    require(bricks == static_cast<size_t>(p.view.bx) * p.view.by * p.view.bz && bricks == p.brick_class.count,
            "kf_pipeline_download_skip_structures: brick count mismatch");
    check(cudaStreamSynchronize(p.stream), "skip structures sync");
    check(cudaMemcpy(brick_class, p.brick_class.ptr, bricks, cudaMemcpyDeviceToHost), "brick class download");
    check(cudaMemcpy(brick_radius, p.brick_radius.ptr, bricks, cudaMemcpyDeviceToHost), "brick radius download");
    check(cudaMemcpy(records, p.stencil_bits.ptr, bricks * 32u * sizeof(uint32_t), cudaMemcpyDeviceToHost),
          "stencil records download");
  });
}

kf_status kf_pipeline_download_pool(kf_pipeline* pipeline, void* voxels, size_t bytes) {
  return guarded([&] {
    require(pipeline != nullptr && voxels != nullptr, "kf_pipeline_download_pool: null argument");
    Pipeline& p = pipeline->impl;
    require(p.block_table.count != 0, "kf_pipeline_download_pool: the pipeline is not sparse");
    require(bytes == p.sparse_capacity * 512u * p.voxel_bytes, "kf_pipeline_download_pool: pool size mismatch");
    check(cudaStreamSynchronize(p.stream), "pool download sync");
    check(cudaMemcpy(voxels, p.voxels.ptr, bytes, cudaMemcpyDeviceToHost), "pool download");
  });
}

kf_status kf_pipeline_download_band_bitmap(kf_pipeline* pipeline, uint32_t* words, size_t count) {
  return guarded([&] {
    require(pipeline != nullptr && words != nullptr, "kf_pipeline_download_band_bitmap: null argument");
    Pipeline& p = pipeline->impl;
    require(p.band_map.count != 0, "kf_pipeline_download_band_bitmap: the raycast backend is not band-march");
    require(count == p.band_map.count, "kf_pipeline_download_band_bitmap: word count mismatch");
    check(cudaStreamSynchronize(p.stream), "band bitmap download sync");
    check(cudaMemcpy(words, p.band_map.ptr, count * sizeof(uint32_t), cudaMemcpyDeviceToHost), "band download");
  });
}

kf_status kf_pipeline_download_raw(kf_pipeline* pipeline, void* voxels, size_t voxel_bytes, void* colors,
                                   size_t color_bytes) {
  return guarded([&] {
    require(pipeline != nullptr, "kf_pipeline_download_raw: null pipeline");
    Pipeline& p = pipeline->impl;
    check(cudaStreamSynchronize(p.stream), "download sync");
    const kf_volume_geometry& g = p.config.volume;
    const uint64_t dense = static_cast<uint64_t>(g.res_x) * g.res_y * g.res_z;
    if (voxels) {
      require(voxel_bytes == dense * p.voxel_bytes, "kf_pipeline_download_raw: voxel buffer size mismatch");
      download_dense(p, p.voxels.ptr, p.voxel_bytes, voxels, unobserved_of(p.config.voxel).voxel);
    }
    if (colors) {
      require(p.colors.count != 0, "kf_pipeline_download_raw: the pipeline stores no colour");
      require(color_bytes == dense * sizeof(float4), "kf_pipeline_download_raw: colour buffer size mismatch");
      download_dense(p, p.colors.ptr, sizeof(float4), colors, unobserved_of(p.config.voxel).color);
    }
  });
}

kf_status kf_pipeline_download_volume(kf_pipeline* pipeline, float* tsdf, float* weight, float* color) {
  return guarded([&] {
    require(pipeline != nullptr && tsdf != nullptr && weight != nullptr, "kf_pipeline_download_volume: null argument");
    Pipeline& p = pipeline->impl;
    check(cudaStreamSynchronize(p.stream), "download sync");
    const kf_volume_geometry& g = p.config.volume;
    const uint64_t dense = static_cast<uint64_t>(g.res_x) * g.res_y * g.res_z;
    std::vector<uint8_t> raw(dense * p.voxel_bytes);
    download_dense(p, p.voxels.ptr, p.voxel_bytes, raw.data(), unobserved_of(p.config.voxel).voxel);
    // host_dense_view decode (volume.hpp:28-100)
    for (uint64_t i = 0; i < dense; ++i) {
      if (p.config.voxel == KF_VOXEL_FLOAT) {
        std::memcpy(tsdf + i, raw.data() + i * 8, 4);
        std::memcpy(weight + i, raw.data() + i * 8 + 4, 4);
      } else {
        uint32_t r;
        std::memcpy(&r, raw.data() + i * 4, 4);
        const uint16_t d = static_cast<uint16_t>(r & 0xFFFFu);
        if (p.config.voxel == KF_VOXEL_QUANTIZED) {
          tsdf[i] = static_cast<float>(static_cast<int16_t>(d)) * (1.0f / 32767.0f);
        } else {
          const uint32_t bits = static_cast<uint32_t>(d) << 16;
          std::memcpy(tsdf + i, &bits, 4);
        }
        weight[i] = static_cast<float>(r >> 16) * (1.0f / 256.0f);
      }
    }
    if (color != nullptr) {
      require(p.colors.count != 0, "kf_pipeline_download_volume: the pipeline stores no colour");
      download_dense(p, p.colors.ptr, sizeof(float4), color, unobserved_of(p.config.voxel).color);
    }
  });
}

kf_status kf_pipeline_extract_mesh(kf_pipeline* pipeline, float min_weight, kf_mesh* out) {
  return guarded([&] {
    require(pipeline != nullptr && out != nullptr, "kf_pipeline_extract_mesh: null argument");
    std::memset(out, 0, sizeof(*out));
    require(std::isfinite(min_weight), "kf_pipeline_extract_mesh: min_weight must be finite");
    extract_mesh(pipeline->impl, min_weight, *out);
  });
}

void kf_mesh_free(kf_mesh* mesh) {
  if (mesh == nullptr) return;
  std::free(mesh->positions);
  std::free(mesh->normals);
  std::free(mesh->colors);
  std::free(mesh->triangles);
  std::memset(mesh, 0, sizeof(*mesh));
}

kf_status kf_pipeline_synchronize(kf_pipeline* pipeline) {
  return guarded([&] {
    require(pipeline != nullptr, "kf_pipeline_synchronize: null pipeline");
    check(cudaStreamSynchronize(pipeline->impl.stream), "pipeline synchronize");
  });
}

kf_status kf_pipeline_stream(kf_pipeline* pipeline, void** stream) {
  return guarded([&] {
    require(pipeline != nullptr && stream != nullptr, "kf_pipeline_stream: null argument");
    *stream = reinterpret_cast<void*>(pipeline->impl.stream);
  });
}

kf_status kf_pipeline_set_kernel_events(kf_pipeline* pipeline, void* start, void* stop) {
  return guarded([&] {
    require(pipeline != nullptr, "kf_pipeline_set_kernel_events: null pipeline");
    pipeline->impl.kernel_start = reinterpret_cast<cudaEvent_t>(start);
    pipeline->impl.kernel_stop = reinterpret_cast<cudaEvent_t>(stop);
  });
}

kf_status kf_pipeline_update_counts(kf_pipeline* pipeline, uint64_t* voxel_updates, uint64_t* color_updates) {
  return guarded([&] {
    require(pipeline != nullptr, "kf_pipeline_update_counts: null pipeline");
    Pipeline& p = pipeline->impl;
    unsigned long long host[2] = {0, 0};
    check(cudaMemcpyAsync(host, p.counters.ptr, sizeof(host), cudaMemcpyDeviceToHost, p.stream), "counter read");
    check(cudaStreamSynchronize(p.stream), "counter read");
    if (voxel_updates) *voxel_updates = host[0];
    if (color_updates) *color_updates = host[1];
  });
}

kf_status kf_tracker_create(const kf_icp_options* options, kf_tracker** out) {
  return guarded([&] {
    require(options != nullptr && out != nullptr, "kf_tracker_create: null argument");
    require(options->max_point_distance >= 0.0f, "ICP max point distance must be non-negative");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) throw CudaError("no CUDA device available");
    auto* t = new kf_tracker();
    try {
      t->impl.options = *options;
      t->impl.params = icp_params_from(*options);
      t->impl.state.resize(1);
      t->impl.partials.resize(2 * static_cast<size_t>(kIcpMaxGrid) * kIcpSlot);
      t->impl.staging.resize(1);
      prepare_icp_kernels();
      check(cudaMemset(t->impl.state.ptr, 0, sizeof(IcpState)), "tracker state init");
      const kf_rigid identity = {{1, 0, 0, 0, 1, 0, 0, 0, 1}, {0, 0, 0}};
      launch_icp_set_pose(t->impl.state.ptr, identity, 1, 0);
      check(cudaStreamSynchronize(0), "tracker state init");
    } catch (...) {
      delete t;
      throw;
    }
    *out = t;
  });
}

kf_status kf_tracker_destroy(kf_tracker* tracker) {
  return guarded([&] { delete tracker; });
}

kf_status kf_tracker_stall_next_level(kf_tracker* tracker) {
  return guarded([&] {
    require(tracker != nullptr, "kf_tracker_stall_next_level: null tracker");
    // a start far above any count the arrivals reach: no wait completes
    const unsigned long long unreachable = 1ull << 62;
    check(cudaMemcpy(reinterpret_cast<char*>(tracker->impl.state.ptr) + offsetof(IcpState, barrier) +
                         offsetof(IcpBarrier, base),
                     &unreachable, sizeof(unreachable), cudaMemcpyHostToDevice),
          "barrier stall");
  });
}

kf_status kf_pipeline_track(kf_pipeline* pipeline, kf_tracker* tracker, const kf_raycast_camera* camera,
                            const kf_level_view* live, uint32_t iterations, kf_icp_outcome* outcome) {
  return guarded([&] {
    require(pipeline && tracker && camera && live && outcome, "kf_pipeline_track: null argument");
    validate_camera(*camera);
    Pipeline& p = pipeline->impl;
    Tracker& t = tracker->impl;
    cudaStream_t s = p.stream;
    Pipeline::Maps& m = p.maps_for(camera->width, camera->height);
    IcpState* st = t.state.ptr;
    // IcpConsumer (reconstruction.cpp:63-67): the render pose is also the
    // initial pose.
    launch_icp_set_pose(st, camera->camera_to_world, 1, s);
    launch_raycast(p, *camera, m.points.ptr, m.normals.ptr, m.colors.ptr, nullptr, s);
    IcpLevelArgs a;
    a.live_vertices = live->vertices;
    a.live_normals = live->normals;
    a.live_width = live->width;
    a.live_height = live->height;
    a.model_points = m.points.ptr;
    a.model_normals = m.normals.ptr;
    a.model_width = camera->width;
    a.model_height = camera->height;
    a.model_intrinsics = intr_from(camera->intrinsics);
    const uint32_t steps = static_cast<size_t>(live->width) * live->height > 0 ? iterations : 0u;
    launch_icp_level(a, st, t.partials.ptr, t.params, steps, -1, 1, 1, s);
    check(cudaMemcpyAsync(t.staging.ptr, st, sizeof(IcpState), cudaMemcpyDeviceToHost, s), "ICP result download");
    check(cudaStreamSynchronize(s), "track");
    check_icp_barrier(*t.staging.ptr, st, s);
    fill_outcome(*t.staging.ptr, outcome);
  });
}

kf_status kf_pipeline_render_model(kf_pipeline* pipeline, const kf_raycast_camera* camera, kf_surface_maps* out) {
  return guarded([&] {
    require(pipeline && camera && out, "kf_pipeline_render_model: null argument");
    validate_camera(*camera);
    Pipeline& p = pipeline->impl;
    Pipeline::Maps& m = p.maps_for(camera->width, camera->height);
    launch_raycast(p, *camera, m.points.ptr, m.normals.ptr, m.colors.ptr, nullptr, p.stream);
    check(cudaStreamSynchronize(p.stream), "model render");
    out->points = m.points.ptr;
    out->normals = m.normals.ptr;
    out->colors = m.colors.ptr;
    out->width = camera->width;
    out->height = camera->height;
    out->memory = KF_MEMORY_DEVICE;
  });
}

kf_status kf_icp_level(kf_tracker* tracker, const kf_level_view* live, const float* model_points,
                       const float* model_normals, uint32_t model_width, uint32_t model_height,
                       kf_intrinsics model_intrinsics, const kf_rigid* model_world_to_camera,
                       const kf_rigid* initial_camera_to_world, uint32_t iterations, kf_icp_outcome* outcome,
                       float* sums) {
  return guarded([&] {
    require(tracker && live && model_points && model_normals && model_world_to_camera && initial_camera_to_world &&
                outcome,
            "kf_icp_level: null argument");
    require((live->vertices && live->normals) || static_cast<uint64_t>(live->width) * live->height == 0,
            "kf_icp_level: null live vertex or normal map");
    Tracker& t = tracker->impl;
    IcpState* st = t.state.ptr;
    cudaStream_t s = 0;  // the legacy stream, ordered with the caller's device maps
    launch_icp_set_pose(st, *initial_camera_to_world, 1, s);
    launch_icp_level_begin(st, t.params.damping_lambda, s);
    // the model transform is fixed for the level (IcpIterationTransforms)
    float model[12];
    std::memcpy(model, model_world_to_camera->r, 9 * sizeof(float));
    std::memcpy(model + 9, model_world_to_camera->t, 3 * sizeof(float));
    check(cudaMemcpyAsync(reinterpret_cast<char*>(st) + offsetof(IcpState, model), model, sizeof(model),
                          cudaMemcpyHostToDevice, s),
          "model upload");
    IcpLevelArgs a;
    a.live_vertices = live->vertices;
    a.live_normals = live->normals;
    a.live_width = live->width;
    a.live_height = live->height;
    a.model_points = model_points;
    a.model_normals = model_normals;
    a.model_width = model_width;
    a.model_height = model_height;
    a.model_intrinsics = intr_from(model_intrinsics);
    // the level start ran above (the model transform replaced after it)
    const uint32_t steps = static_cast<size_t>(live->width) * live->height > 0 ? iterations : 0u;
    launch_icp_level(a, st, t.partials.ptr, t.params, steps, -1, 0, 1, s);
    check(cudaMemcpyAsync(t.staging.ptr, st, sizeof(IcpState), cudaMemcpyDeviceToHost, s), "ICP result download");
    check(cudaStreamSynchronize(s), "ICP level");
    check_icp_barrier(*t.staging.ptr, st, s);
    fill_outcome(*t.staging.ptr, outcome);
    if (sums) std::memcpy(sums, t.staging.ptr->sums, kIcpSums * sizeof(float));
  });
}

kf_status kf_icp_normal_equations(kf_tracker* tracker, const kf_level_view* live, const float* model_points,
                                  const float* model_normals, uint32_t model_width, uint32_t model_height,
                                  kf_intrinsics model_intrinsics, const kf_rigid* camera,
                                  const kf_rigid* model_world_to_camera, float* sums, uint64_t* count) {
  return guarded([&] {
    require(tracker && live && model_points && model_normals && camera && model_world_to_camera && sums && count,
            "kf_icp_normal_equations: null argument");
    require((live->vertices && live->normals) || static_cast<uint64_t>(live->width) * live->height == 0,
            "kf_icp_normal_equations: null live vertex or normal map");
    Tracker& t = tracker->impl;
    IcpState* st = t.state.ptr;
    float cam[12], model[12];
    std::memcpy(cam, camera->r, 9 * sizeof(float));
    std::memcpy(cam + 9, camera->t, 3 * sizeof(float));
    std::memcpy(model, model_world_to_camera->r, 9 * sizeof(float));
    std::memcpy(model + 9, model_world_to_camera->t, 3 * sizeof(float));
    const int running = kIcpRunning;
    const unsigned zero = 0;
    check(cudaMemcpy(reinterpret_cast<char*>(st) + offsetof(IcpState, camera), cam, sizeof(cam),
                     cudaMemcpyHostToDevice), "camera upload");
    check(cudaMemcpy(reinterpret_cast<char*>(st) + offsetof(IcpState, model), model, sizeof(model),
                     cudaMemcpyHostToDevice), "model upload");
    check(cudaMemcpy(reinterpret_cast<char*>(st) + offsetof(IcpState, status), &running, sizeof(int),
                     cudaMemcpyHostToDevice), "status upload");
    check(cudaMemcpy(reinterpret_cast<char*>(st) + offsetof(IcpState, arrived), &zero, sizeof(unsigned),
                     cudaMemcpyHostToDevice), "ticket reset");
    IcpLevelArgs a;
    a.live_vertices = live->vertices;
    a.live_normals = live->normals;
    a.live_width = live->width;
    a.live_height = live->height;
    a.model_points = model_points;
    a.model_normals = model_normals;
    a.model_width = model_width;
    a.model_height = model_height;
    a.model_intrinsics = intr_from(model_intrinsics);
    launch_icp_sweep(a, st, t.partials.ptr, t.params, 0);
    check(cudaMemcpy(t.staging.ptr, st, sizeof(IcpState), cudaMemcpyDeviceToHost), "sums download");
    std::memcpy(sums, t.staging.ptr->sums, kIcpSums * sizeof(float));
    *count = t.staging.ptr->count;
  });
}

}  // extern "C"
