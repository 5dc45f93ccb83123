// kf_internal.h - host-side objects behind the C ABI (include/kf_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/kf_b200.h"
#include "kf_common.cuh"

namespace kf {

// ---- errors ----------------------------------------------------------------
// Misconfiguration (std::invalid_argument in the reference, validation.hpp:9-13).
struct InvalidArgument : std::runtime_error {
  using std::runtime_error::runtime_error;
};
// CUDA failure (std::runtime_error from cuda::check, cuda/check.cuh:11-16).
struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct Unsupported : std::runtime_error {
  using std::runtime_error::runtime_error;
};
// A bounded device-side wait gave up.
struct DeviceTimeout : std::runtime_error {
  using std::runtime_error::runtime_error;
};
// File read, write or decode failure (std::runtime_error in the reference,
// image_proc/read_png.cpp, src/app/frame_output.cpp).
struct IoError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void set_last_error(const std::string& message);
void check(cudaError_t status, const char* what);
void require(bool condition, const char* what);

// Runs `body`, mapping exceptions to kf_status codes and kf_last_error().
template <typename Body>
kf_status guarded(Body&& body) {
  try {
    body();
    return KF_OK;
  } catch (const InvalidArgument& e) {
    set_last_error(e.what());
    return KF_ERR_INVALID_ARGUMENT;
  } catch (const Unsupported& e) {
    set_last_error(e.what());
    return KF_ERR_UNSUPPORTED;
  } catch (const CudaError& e) {
    set_last_error(e.what());
    return KF_ERR_CUDA;
  } catch (const DeviceTimeout& e) {
    set_last_error(e.what());
    return KF_ERR_DEVICE_TIMEOUT;
  } catch (const IoError& e) {
    set_last_error(e.what());
    return KF_ERR_IO;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return KF_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return KF_ERR_INVALID_ARGUMENT;
  }
}

// Owning device allocation.
template <typename T>
struct DeviceArray {
  T* ptr = nullptr;
  size_t count = 0;
  DeviceArray() = default;
  explicit DeviceArray(size_t n) { resize(n); }
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  DeviceArray(DeviceArray&& o) noexcept : ptr(o.ptr), count(o.count) {
    o.ptr = nullptr;
    o.count = 0;
  }
  DeviceArray& operator=(DeviceArray&& o) noexcept {
    if (this != &o) {
      release();
      ptr = o.ptr;
      count = o.count;
      o.ptr = nullptr;
      o.count = 0;
    }
    return *this;
  }
  ~DeviceArray() { release(); }
  void resize(size_t n) {
    if (n == count) return;
    release();
    if (n > 0) {
      const cudaError_t s = cudaMalloc(reinterpret_cast<void**>(&ptr), n * sizeof(T));
      if (s != cudaSuccess) {
        ptr = nullptr;
        throw CudaError(std::string("cudaMalloc: ") + cudaGetErrorString(s));
      }
    }
    count = n;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    count = 0;
  }
  size_t bytes() const { return count * sizeof(T); }
};

template <typename T>
struct PinnedArray {
  T* ptr = nullptr;
  size_t count = 0;
  PinnedArray() = default;
  PinnedArray(const PinnedArray&) = delete;
  PinnedArray& operator=(const PinnedArray&) = delete;
  ~PinnedArray() { release(); }
  void resize(size_t n) {
    if (n <= count) return;
    release();
    check(cudaMallocHost(reinterpret_cast<void**>(&ptr), n * sizeof(T)), "cudaMallocHost");
    count = n;
  }
  void release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    count = 0;
  }
};

// ---- depth pyramid (PyramidSource, depth_processing.hpp:422-463) -----------
struct PyramidLevelBuffers {
  DeviceArray<uint16_t> depth;
  DeviceArray<float> vertices;
  DeviceArray<float> normals;
  uint32_t width = 0, height = 0;
  kf_intrinsics intrinsics{};
};

struct Pyramid {
  kf_depth_options options{};
  DeviceArray<uint16_t> raw;  // unfiltered input depth (integration reads it)
  uint32_t width = 0, height = 0;
  kf_intrinsics intrinsics{};
  std::vector<PyramidLevelBuffers> levels;
  uint32_t level_count = 0;
  cudaStream_t stream = nullptr;  // borrowed from the caller of build

  // Sizes buffers for a width x height frame; returns the level count.
  uint32_t prepare(uint32_t width, uint32_t height, kf_intrinsics intrinsics);
  // Launches the pyramid kernels over `raw` on `stream`.
  void launch(cudaStream_t stream) const;
};

// ---- ICP device state --------------------------------------------------------
constexpr int kIcpSums = 29;          // 21 JtJ + 6 Jtr + distance + residual^2
constexpr int kIcpSlot = 32;          // floats per CTA partial (29 sums + count)
constexpr int kIcpBlock = 512;          // one CTA per SM: 16 warps, as two CTAs of 256 threads
constexpr unsigned kIcpSegments = kIcpBlock / 32;  // the combine: one warp per segment of slots
constexpr int kIcpPixels = 1;         // live pixels per thread and grid step of a sweep
constexpr int kIcpMaxGrid = 148;      // one CTA per SM on a 148-SM B200
constexpr int kIcpRunning = -1;

// Grid barrier of the whole-level ICP kernel: the arrivals of every CTA at
// every barrier since the tracker's creation (never reset while the barrier
// completes), the count at which the next launch starts, and a sticky
// give-up flag set by a wait that ran out of polls.
struct IcpBarrier {
  unsigned long long count;
  unsigned long long base;
  unsigned broken;
  unsigned pad[3];
};

// Lives in device memory; one per tracker.  All poses are camera_to_world.
struct IcpState {
  double pose[12];       // FP64 pose, row-major 3x4
  float camera[12];      // float copy used by the correspondence search
  float model[12];       // model world_to_camera (float), fixed per level
  float world_to_camera[12];  // float inverse of the pose, for integration
  double best_pose[12];  // adaptive damping rollback target
  float best_sums[kIcpSums];
  unsigned long long best_count;
  float lambda;
  float best_cost;
  int have_best;
  int status;            // kIcpRunning while iterating, then KF_ICP_*
  int iterations;        // completed Gauss-Newton steps in this level
  unsigned arrived;      // CTA arrival ticket of the current sweep
  int failed;            // a previous level of this frame failed
  int level_status[4];
  int level_iterations[4];
  unsigned long long level_correspondences[4];
  // diagnostics (IcpDiagnostics, icp_optimizer.hpp:41-51)
  unsigned long long correspondences;
  float mean_point_distance;
  float mean_squared_residual;
  float min_system_eigenvalue;
  float condition_number;
  float update_translation;
  float update_rotation;
  float damping_lambda;
  unsigned long long rejected_steps;
  // last raw sweep (for kf_icp_normal_equations)
  float sums[kIcpSums];
  unsigned long long count;
  // last member: the whole-level kernel copies and writes back the state
  // before it, never the barrier other CTAs may be polling
  IcpBarrier barrier;
};

struct IcpParams {
  unsigned long long min_correspondences;
  float max_point_distance, min_normal_dot;
  float min_update_translation, min_update_rotation;
  float max_update_translation, max_update_rotation;
  float min_system_eigenvalue, max_condition_number;
  int damping_mode;
  float damping_lambda;
  int adaptive;
  float lambda_increase, lambda_decrease, min_lambda, max_lambda;
};

struct Tracker {
  kf_icp_options options{};
  IcpParams params{};
  DeviceArray<IcpState> state;
  DeviceArray<float> partials;  // 2 x kIcpMaxGrid x kIcpSlot, scratch of the sweeps
  PinnedArray<IcpState> staging;
};

// Geometry of one correspondence sweep.
struct IcpLevelArgs {
  const float* live_vertices;
  const float* live_normals;
  uint32_t live_width, live_height;
  const float* model_points;
  const float* model_normals;
  uint32_t model_width, model_height;
  Intr model_intrinsics;
};

IcpParams icp_params_from(const kf_icp_options& o);
unsigned icp_grid_for(uint32_t pixels);
// Per-device kernel attributes of the sweep (its shared-memory staging).
void prepare_icp_kernels();
// Begin a level: model world_to_camera from the current pose, status running,
// unless a previous level failed (then the level stays skipped).
void launch_icp_level_begin(IcpState* state, float damping_lambda, cudaStream_t stream);
// One correspondence sweep: the state's sums and count at its camera and
// model transforms (no solve).
void launch_icp_sweep(const IcpLevelArgs& args, IcpState* state, float* partials, const IcpParams& params,
                      cudaStream_t stream);
// A whole level in one cooperative launch: with `begin` the level start,
// then up to `iterations` Gauss-Newton steps (the loop leaves at the first
// non-running status), then the level end (level >= 0 records the frame's
// per-level results).  `partials` holds two sweeps' slots.
void launch_icp_level(const IcpLevelArgs& args, IcpState* state, float* partials, const IcpParams& params,
                      uint32_t iterations, int level, int begin, int want_values, cudaStream_t stream);
// The same level as launches that need no co-residency: a begin kernel,
// one sweep-and-step launch per iteration (later ones return at once once
// the level's status is settled), an end kernel.  Bit-identical to
// launch_icp_level at begin = 1, want_values = 0 (the same sweep grid,
// combine and step); for frame graphs that run beside others (batches).
void launch_icp_level_steps(const IcpLevelArgs& args, IcpState* state, float* partials, const IcpParams& params,
                            uint32_t iterations, int level, cudaStream_t stream);
// Throws DeviceTimeout when the downloaded state `host` shows a grid barrier
// that gave up; the device barrier is cleared first (ordered on `stream`).
void check_icp_barrier(const IcpState& host, IcpState* device, cudaStream_t stream);
// Set the device pose (FP64 + float) from a float rigid transform.
void launch_icp_set_pose(IcpState* state, kf_rigid pose, int reset_frame, cudaStream_t stream);

// ---- volume / pipeline --------------------------------------------------------
struct Pipeline {
  kf_pipeline_config config{};
  VolumeDev view{};
  DeviceArray<uint8_t> voxels;
  DeviceArray<float4> colors;
  size_t voxel_bytes = 0;
  uint64_t voxel_count = 0;
  // Exact empty-space skip of the raycast (8^3 bricks, x-major order).
  // Per-voxel bits, per brick 8 layers (z) of 16 bytes: 64 bits "observed
  // with tsdf exactly 1" then 64 bits "observed", bit y*8+x.
  DeviceArray<uint32_t> voxel_bits;
  // Per stencil base voxel, same layout: 64 bits "undecided" then 64 bits
  // "exactly 1.0" (when decided and clear: nullopt), for the trilinear
  // stencil based at that voxel under the pipeline's corner policy.
  DeviceArray<uint32_t> stencil_bits;
  DeviceArray<uint32_t> brick_dirty;     // per brick: voxel bits changed this frame
  // Per brick: 1 = every stencil based in the brick is nullopt, 2 = every
  // one is exactly 1.0 (all eight corners observed with tsdf exactly 1).
  DeviceArray<uint8_t> brick_class;
  // Per brick of class 1 or 2: the radius (in bricks, up to 7) of the cube of
  // bricks around it that all share its class, inside the brick grid, 0 for
  // mixed bricks (brick_radius_kernel); the raycast crosses such a cube at
  // once.  radius_scratch holds the passes' run and square radii.
  DeviceArray<uint8_t> brick_radius;
  DeviceArray<uint8_t> radius_scratch;
  DeviceArray<uint32_t> band_bits;       // band integration: blocks the bands cross
  // band-march raycast (BasicBandBitmap, occupancy.hpp:240-278): block bits
  // in z-major order (32 z-blocks per word), raw and 3^3-dilated; rebuilt
  // after every integration.
  DeviceArray<uint32_t> band_raw, band_map;
  // sparse storage: per block b (x-major), 1 while the blocks b + {0,1}^3 are
  // all unallocated (every trilinear stencil based in b is then nullopt)
  DeviceArray<uint8_t> null_bricks;
  // Sparse storage (BlockRep, block_rep.hpp:26-110): the voxel-block hash
  // (block -> slot, kf_common.cuh block_table_lookup) of 2^k >= 2 x capacity
  // entries, `sparse_capacity` slots in the pools.
  DeviceArray<unsigned long long> block_table;
  DeviceArray<uint32_t> slot_block;      // block of each allocated slot
  DeviceArray<unsigned long long> allocated;  // [0] attempts so far (overflow included), [1] this frame's base
  DeviceArray<uint32_t> new_bits, word_prefix, cta_prefix;
  uint64_t sparse_capacity = 0;
  // Block culling of the full sweep
  DeviceArray<float> depth_tiles;        // max depth per 8x8 pixel tile, then coarser levels
  DeviceArray<uint32_t> block_list;
  DeviceArray<unsigned> block_count;
  uint32_t tile_levels = 0, tile_w[12] = {}, tile_h[12] = {}, tile_off[12] = {};
  // integration pixel table (float4 per pixel: depth, lambda, weight, color)
  DeviceArray<float4> pixel_table;
  DeviceArray<uint16_t> own_depth;     // upload target when no pyramid supplies one
  DeviceArray<uint32_t> own_color;
  DeviceArray<float> own_normals;
  DeviceArray<uint32_t> frame_color;   // colour of the frame being processed
  // cached map buffers per extent (device_pipeline.cu:133-136)
  struct Maps {
    DeviceArray<float> points, normals;
    DeviceArray<uint32_t> colors;
  };
  std::map<std::pair<uint32_t, uint32_t>, Maps> maps;
  cudaStream_t stream = nullptr;
  DeviceArray<unsigned long long> counters;  // [0] voxel updates, [1] colour updates
  cudaEvent_t kernel_start = nullptr, kernel_stop = nullptr;  // borrowed
  // whole-frame graphs keyed by (width, height, iterations, first, colour, fork)
  // fork: the frame's inputs on a side branch (standalone frames; batch
  // members run concurrently already and keep one branch)
  struct GraphKey {
    uint32_t w, h, it0, it1, it2, it3, first, color, fork, cooperative;
    bool operator<(const GraphKey& o) const {
      const uint32_t a[10] = {w, h, it0, it1, it2, it3, first, color, fork, cooperative};
      const uint32_t b[10] = {o.w, o.h, o.it0, o.it1, o.it2, o.it3, o.first, o.color, o.fork, o.cooperative};
      for (int i = 0; i < 10; ++i) {
        if (a[i] != b[i]) return a[i] < b[i];
      }
      return false;
    }
  };
  struct FrameGraph {
    cudaGraph_t graph = nullptr;     // kept for batches (child graph nodes)
    cudaGraphExec_t exec = nullptr;
    uint32_t kernels = 0;  // kernel nodes of the captured frame
  };
  std::map<GraphKey, FrameGraph> graphs;
  uint64_t graph_epoch = 0;  // bumped whenever the frame graphs are dropped
  // Launch shapes the autotuner may change (none of them changes a result bit)
  uint32_t raycast_block_x = 16, raycast_block_y = 4;  // march CTA, at most 64 threads
  uint32_t integrate_ctas = 148 * 48;                 // fusion grid (grid-strided over listed blocks)
  bool concurrent = false;  // frames run beside other GPU work: per-step ICP launches (kf_pipeline_set_concurrent)
  uint32_t raycast_lanes[3] = {8, 4, 1};              // lanes per ray: <= 20,000 rays, <= 80,000, more
  uint32_t last_frame_kernels = 0;
  kf_pyramid* graph_pyramid = nullptr;
  kf_tracker* graph_tracker = nullptr;
  PinnedArray<IcpState> result_staging;
  PinnedArray<uint16_t> depth_staging;
  PinnedArray<uint32_t> color_staging;
  cudaEvent_t staging_done = nullptr;  // after the last upload from the staging buffers
  // kf_frame_submit's depth uploads: two pinned staging and device buffers
  // used in turn, copied on their own stream while earlier frames run
  PinnedArray<uint16_t> depth_pinned[2];
  DeviceArray<uint16_t> depth_upload[2];
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t uploaded[2] = {}, consumed[2] = {};
  int upload_turn = 0;
  // the frame graph's side branch (frame inputs beside the first model render)
  cudaStream_t side_stream = nullptr;
  cudaEvent_t fork_event = nullptr, pyramid_event = nullptr, inputs_event = nullptr;
  // kf_frame_submit: the results of frames in flight, oldest first
  static constexpr int kResultSlots = 8;
  PinnedArray<IcpState> result_ring;
  cudaEvent_t result_ready[kResultSlots] = {};
  uint8_t result_first[kResultSlots] = {};
  uint64_t results_pushed = 0, results_popped = 0;
  int frames_fused = 0;

  Maps& maps_for(uint32_t w, uint32_t h);
  void clear_graphs();
};

// Integration pixel table: depth meters (NaN if unusable), lambda, fusion
// weight and colour, one float4 per pixel.
void launch_pixel_table(const uint16_t* depth, const uint32_t* color, const float* normals,
                        uint32_t width, uint32_t height, Intr intrinsics,
                        const kf_integration_options& options, int rule, float4* table,
                        cudaStream_t stream);
// Dense full sweep.  `pose_state` (optional) overrides world_to_camera with
// the inverse of the tracked pose and skips fusion when tracking failed.
// With `inputs_ready` the steps of launch_integrate_inputs already ran.
void launch_integrate(Pipeline& p, const float4* table, uint32_t width, uint32_t height,
                      Intr intrinsics, Rigid world_to_camera, int has_color,
                      const IcpState* pose_state, cudaStream_t stream, bool inputs_ready = false);
// The integration steps that need only the frame's pixel table, not the pose:
// the depth-tile pyramid of the full sweep's block culling.
void launch_integrate_inputs(Pipeline& p, const float4* table, uint32_t width, uint32_t height,
                             cudaStream_t stream);
// Allocates and clears the per-block skip and culling buffers.
// C = A * B^T (+bias)(ReLU) on the tensor cores: A M x K, B N x K bf16
// row-major (leading dimensions lda, ldb), C M x N fp32 (ldc).  `error`
// (device int) is set when a tensor-core wait times out.  With a workspace
// (device floats) a GEMM of few output tiles and long K is split along K
// across CTAs (partials in the workspace, summed in split order).
void launch_gemm_bf16(const void* A, const void* B, float* C, int M, int N, int K, int lda, int ldb, int ldc,
                      const float* bias, int relu, int* error, cudaStream_t stream, float* workspace = nullptr,
                      size_t workspace_floats = 0);
// MarchingCubes::extract on the device (dense volumes); fills a host mesh.
void extract_mesh(Pipeline& p, float min_weight, kf_mesh& out);
void prepare_blocks(Pipeline& p, uint32_t width, uint32_t height, cudaStream_t stream);
// Clears the skip bits (a freshly filled volume: nothing observed).
void reset_blocks(Pipeline& p, cudaStream_t stream);
// Raycast into device maps.  `pose_state` (optional) supplies the
// camera_to_world from the tracker and skips the render after a failure.
// Rebuilds the band-march bitmap from the volume (BandRebuild, occupancy.hpp:229-238).
void launch_band_rebuild(Pipeline& p, cudaStream_t stream);
void launch_raycast(const Pipeline& p, const kf_raycast_camera& camera, float* points,
                    float* normals, uint32_t* colors, const IcpState* pose_state,
                    cudaStream_t stream);
void launch_fill_volume(Pipeline& p, cudaStream_t stream);
uint64_t count_observed(Pipeline& p);
// Sparse storage: every block unallocated again.
void reset_sparse(Pipeline& p, cudaStream_t stream);

}  // namespace kf

struct kf_pyramid {
  kf::Pyramid impl;
};
struct kf_tracker {
  kf::Tracker impl;
};
struct kf_pipeline {
  kf::Pipeline impl;
};
