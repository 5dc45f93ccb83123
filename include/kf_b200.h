/*
 * kf_b200.h - C ABI of the B200 (sm_100a) KinectFusion per-frame pipeline.
 *
 * Every entry point is extern "C", takes plain pointers, sizes and POD
 * structs, and returns a kf_status (0 = KF_OK).  kf_last_error() returns a
 * thread-local description of the last failure.  Device buffers are owned by
 * the library objects (pipelines, pyramids, trackers); caller buffers are
 * borrowed for the duration of a call only.
 *
 * Reference interfaces replaced (paths within maximsolodukhin/KinectFusion):
 *   Pipeline::device_available / create_device   include/kinectfusion/pipeline.hpp:154-158
 *                                                 (CPU stubs src/kinectfusion/pipeline.cpp:120-127)
 *   Pipeline::{integrate,raycast,track,observed_voxel_count,host_view,extract_mesh}
 *                                                 include/kinectfusion/pipeline.hpp:72-97
 *   PyramidSource::create_device / build / level  include/kinectfusion/depth_processing.hpp:422-463
 *   DepthUploader::create                          include/kinectfusion/tsdf_integration.hpp:108-109
 *   BasicDeviceCorrespondenceSweep::{run,run_loop} include/kinectfusion/icp_correspondence.hpp:363-369
 *   ProjectiveIcpTracker::estimate_pose(DeviceTrackingRequest)
 *                                                 include/kinectfusion/icp_optimizer.hpp:115-116
 */
#ifndef KF_B200_H
#define KF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KF_B200_ABI_VERSION 1

typedef int kf_status;
enum {
  KF_OK = 0,
  KF_ERR_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference (validation.hpp:9-13) */
  KF_ERR_CUDA = 2,             /* std::runtime_error from cuda::check (cuda/check.cuh:11-16) */
  KF_ERR_NO_DEVICE = 3,        /* create_device without a CUDA device */
  KF_ERR_OUT_OF_MEMORY = 4,
  KF_ERR_DEVICE_TIMEOUT = 5,   /* a bounded device-side wait gave up */
  KF_ERR_UNSUPPORTED = 6,      /* storage combination not offered (pipeline.cpp:104-118) */
  KF_ERR_IO = 7                /* file read, write or decode failure (std::runtime_error in read_png.cpp) */
};

/* Memory space of a caller buffer passed through the ABI. */
enum { KF_MEMORY_HOST = 0, KF_MEMORY_DEVICE = 1 };

/* Enumerations mirror include/kinectfusion/pipeline.hpp:24-26, raycasting.hpp:22,
 * tsdf_integration.hpp:28, trilinear.hpp:18-21, icp_correspondence.hpp:56. */
enum { KF_VOXEL_FLOAT = 0, KF_VOXEL_QUANTIZED = 1, KF_VOXEL_BF16 = 2 };
enum { KF_COLOR_FLOAT = 0, KF_COLOR_NONE = 1 };
enum { KF_STORAGE_DENSE = 0, KF_STORAGE_SPARSE = 1 };
enum { KF_RULE_CLASSIC = 0, KF_RULE_ANGLE_WEIGHTED = 1 };
enum { KF_INTEGRATION_FULL = 0, KF_INTEGRATION_BAND = 1 };
enum { KF_RAYCAST_MARCH = 0, KF_RAYCAST_BITMAP_MARCH = 1, KF_RAYCAST_BAND_MARCH = 2 };
enum { KF_CORNERS_SKIP_MISSING = 0, KF_CORNERS_REQUIRE_ALL = 1 };
enum { KF_DAMPING_NONE = 0, KF_DAMPING_IDENTITY = 1, KF_DAMPING_DIAGONAL = 2 };

/* IcpFailure (icp_optimizer.hpp:22-28) plus the two success kinds. */
enum {
  KF_ICP_MAX_ITERATIONS = 0,
  KF_ICP_CONVERGED = 1,
  KF_ICP_TOO_FEW_CORRESPONDENCES = 2,
  KF_ICP_SOLVE_FAILED = 3,
  KF_ICP_UPDATE_TOO_LARGE = 4,
  KF_ICP_UNCONSTRAINED_SYSTEM = 5,
  KF_ICP_INVALID_INPUT = 6,
  KF_ICP_NOT_RUN = 7
};

/* CameraIntrinsics (rgbd.hpp:26-74). */
typedef struct {
  float fx, fy, cx, cy;
} kf_intrinsics;

/* RigidTransform (vector.hpp:209-236): row-major rotation, then translation. */
typedef struct {
  float r[9];
  float t[3];
} kf_rigid;

/* DepthProcessingOptions (depth_processing.hpp:31-47). */
typedef struct {
  uint32_t levels;
  float depth_scale;
  float min_depth;
  float max_depth;
  float max_normal_depth_jump;
  float max_downsample_depth_jump;
  int32_t bilateral_filter;
  int32_t bilateral_radius;
  float bilateral_spatial_sigma;
  float bilateral_depth_sigma;
} kf_depth_options;

/* TsdfIntegrationOptions (tsdf_integration.hpp:31-50). */
typedef struct {
  float depth_scale;
  float observation_weight;
  float max_weight;
  float min_depth;
  float max_depth;
  int32_t projective_distance;
  int32_t distance_scaled_truncation;
  float truncation_distance_scale;
  int32_t mode; /* KF_INTEGRATION_* */
} kf_integration_options;

/* RaycastOptions (raycasting.hpp:66-78). */
typedef struct {
  float min_depth;
  float max_depth;
  float step_scale;
  int32_t corner_policy; /* KF_CORNERS_* */
  int32_t cell_gradient_normals;
  int32_t seed_from_previous;
} kf_raycast_options;

/* VolumeGeometry (volume.hpp:265-287). */
typedef struct {
  uint32_t res_x, res_y, res_z;
  float voxel_size;
  float origin[3];
  float truncation_distance;
} kf_volume_geometry;

/* PipelineConfig (pipeline.hpp:29-46) without the name and memory space. */
typedef struct {
  kf_volume_geometry volume;
  int32_t voxel;           /* KF_VOXEL_* */
  int32_t color;           /* KF_COLOR_* */
  int32_t storage;         /* KF_STORAGE_* */
  uint64_t sparse_block_capacity; /* 0 = block_count / 4 */
  int32_t tsdf_rule;       /* KF_RULE_* */
  kf_integration_options integration;
  kf_raycast_options raycast;
  int32_t raycast_backend; /* KF_RAYCAST_* */
} kf_pipeline_config;

/* One depth-camera observation (DepthFrameView, tsdf_integration.hpp:54-61).
 * depth: width*height uint16; color: RGBA8 packed uint32 or NULL; normals:
 * width*height*3 float (camera frame) or NULL.  `memory` says where all three
 * live. */
typedef struct {
  const uint16_t* depth;
  const uint32_t* color;
  const float* normals;
  uint32_t width, height;
  kf_intrinsics intrinsics;
  kf_rigid world_to_camera;
  int32_t memory; /* KF_MEMORY_* */
} kf_frame_view;

/* RaycastCamera (raycasting.hpp:80-90). */
typedef struct {
  kf_intrinsics intrinsics;
  uint32_t width, height;
  kf_rigid camera_to_world;
} kf_raycast_camera;

/* SurfaceMaps (volume.hpp:172-185): points/normals width*height*3 float
 * (world frame, NaN = no surface), colors width*height RGBA8. */
typedef struct {
  float* points;
  float* normals;
  uint32_t* colors;
  uint32_t width, height;
  int32_t memory; /* KF_MEMORY_* */
} kf_surface_maps;

/* One pyramid level as device views (PyramidLevel, depth_processing.hpp:412-416). */
typedef struct {
  const uint16_t* depth;  /* filtered (level 0) or downsampled depth */
  const float* vertices;  /* width*height*3, camera frame */
  const float* normals;   /* width*height*3 */
  uint32_t width, height;
  kf_intrinsics intrinsics;
} kf_level_view;

/* ProjectiveIcpOptions (icp_optimizer.hpp:80-101) + damping (icp_correspondence.hpp:56-98). */
typedef struct {
  uint64_t min_correspondences;
  float max_point_distance;
  float min_normal_dot;
  float min_update_translation;
  float min_update_rotation;
  float max_update_translation;
  float max_update_rotation;
  float min_system_eigenvalue;
  float max_condition_number;
  int32_t damping_mode; /* KF_DAMPING_* */
  float damping_lambda;
  int32_t adaptive_damping;
  float lambda_increase, lambda_decrease, min_lambda, max_lambda;
} kf_icp_options;

/* IcpOutcome + IcpDiagnostics (icp_optimizer.hpp:41-62).  pose is the
 * camera_to_world after the call (on failure: the last pose reached). */
typedef struct {
  kf_rigid pose;
  double pose_f64[12];
  int32_t status; /* KF_ICP_* */
  int32_t iterations;
  uint64_t correspondences;
  float mean_point_distance;
  float mean_squared_residual;
  float min_system_eigenvalue;
  float condition_number;
  float update_translation;
  float update_rotation;
  float damping_lambda;
  uint64_t rejected_steps;
} kf_icp_outcome;

/* Per-frame result of kf_frame_process. */
typedef struct {
  kf_rigid camera_to_world;
  int32_t tracked;      /* 1 when every level succeeded and the frame was fused */
  int32_t status[4];    /* per pyramid level, KF_ICP_* (index = level) */
  int32_t iterations[4];
  uint64_t correspondences[4];
  /* the world_to_camera the frame was integrated at: the FP64 inverse of the
   * tracked pose rounded to float (the reference inverts its float pose,
   * reconstruction.cpp:274; the two agree to rounding) */
  kf_rigid world_to_camera;
} kf_frame_result;

/* Welded triangle mesh (MarchingCubes::Mesh, marching_cubes.hpp:20-25). */
typedef struct {
  float* positions;   /* vertex_count*3 */
  float* normals;     /* vertex_count*3 */
  float* colors;      /* vertex_count*3, 0..255 */
  uint32_t* triangles;/* triangle_count*3 */
  uint64_t vertex_count;
  uint64_t triangle_count;
} kf_mesh;

typedef struct kf_pipeline kf_pipeline;
typedef struct kf_pyramid kf_pyramid;
typedef struct kf_tracker kf_tracker;

/* ---- library ---------------------------------------------------------- */
const char* kf_last_error(void);
int kf_abi_version(void);
/* Pipeline::device_available (pipeline.hpp:154). */
kf_status kf_device_available(int32_t* available);
/* Reference defaults of each options struct (the C++ default member values). */
void kf_default_depth_options(kf_depth_options* out);
void kf_default_integration_options(kf_integration_options* out);
void kf_default_raycast_options(kf_raycast_options* out);
void kf_default_icp_options(kf_icp_options* out);
void kf_default_pipeline_config(kf_pipeline_config* out);

/* ---- pyramid: PyramidSource::create_device (depth_processing.hpp:460-462) */
kf_status kf_pyramid_create(const kf_depth_options* options, kf_pyramid** out);
kf_status kf_pyramid_destroy(kf_pyramid* pyramid);
/* PyramidSource::build (depth_processing.hpp:434-435); returns the level count. */
kf_status kf_pyramid_build(kf_pyramid* pyramid, const uint16_t* depth, uint32_t width,
                           uint32_t height, kf_intrinsics intrinsics, int32_t memory,
                           uint32_t* level_count);
/* PyramidSource::level (depth_processing.hpp:437): device views, valid until the next build. */
kf_status kf_pyramid_level(const kf_pyramid* pyramid, uint32_t index, kf_level_view* out);
/* The unfiltered depth of the last build on the device (width*height u16,
 * valid until the next build): the upload PyramidSource::device_frame hands
 * to integration so the frame crosses to the device once
 * (depth_processing.hpp:451-453, depth_processing.cu:149-157). */
kf_status kf_pyramid_raw_depth(const kf_pyramid* pyramid, const uint16_t** depth);
/* Host copies of one level (any pointer may be NULL). */
kf_status kf_pyramid_download_level(const kf_pyramid* pyramid, uint32_t index, uint16_t* depth,
                                    float* vertices, float* normals);

/* ---- pipeline: Pipeline::create_device (pipeline.hpp:99-109, device_pipeline.cu:176-182) */
kf_status kf_pipeline_create(const kf_pipeline_config* config, kf_pipeline** out);
kf_status kf_pipeline_destroy(kf_pipeline* pipeline);
/* Refill the volume with unobserved voxels (BasicVolume construction fill). */
kf_status kf_pipeline_reset(kf_pipeline* pipeline);
/* The same refill queued on the pipeline's stream without waiting for it
 * (no reference counterpart: the reference starts a sequence by constructing
 * a pipeline).  Frames enqueued after it see the empty volume; a new sequence
 * starts without a host stall behind the previous one's frames in flight. */
kf_status kf_pipeline_reset_async(kf_pipeline* pipeline);
/* Pipeline::integrate (pipeline.hpp:75-79). */
kf_status kf_pipeline_integrate(kf_pipeline* pipeline, const kf_frame_view* frame);
/* Pipeline::raycast (pipeline.hpp:81): renders into `out` (host or device buffers). */
kf_status kf_pipeline_raycast(kf_pipeline* pipeline, const kf_raycast_camera* camera,
                              const kf_surface_maps* out);
/* Pipeline::observed_voxel_count (pipeline.hpp:87). */
kf_status kf_pipeline_observed_voxel_count(kf_pipeline* pipeline, uint64_t* count);
/* Pipeline::host_view (pipeline.hpp:90): dense float staging copy.  tsdf and
 * weight are voxel_count floats; color (voxel_count*4 floats) may be NULL. */
kf_status kf_pipeline_download_volume(kf_pipeline* pipeline, float* tsdf, float* weight,
                                      float* color);
/* Raw storage bytes of the volume (dense: voxel_count*voxel_bytes). */
kf_status kf_pipeline_download_raw(kf_pipeline* pipeline, void* voxels, size_t voxel_bytes,
                                   void* colors, size_t color_bytes);
/* Sparse storage: allocation attempts so far (BlockRep's `allocated`
 * counter, block_rep.cu:18-41, overflow included; allocated blocks =
 * min(attempts, capacity)) and the pool capacity in blocks.  Dense: 0, 0. */
kf_status kf_pipeline_block_stats(kf_pipeline* pipeline, uint64_t* attempts, uint64_t* capacity);
/* The 8^3 blocks the last integration visited (the culled or band-listed
 * blocks every voxel of which ran the projective test; no counterpart in the
 * reference, which visits every voxel). */
kf_status kf_pipeline_listed_blocks(kf_pipeline* pipeline, uint64_t* blocks);
/* Sparse storage: the block-slot grid (BlockRep::grid, block_rep.hpp:26-110),
 * one uint32 per 8^3 block in x-major block order, 0xFFFFFFFF = unallocated. */
kf_status kf_pipeline_download_block_grid(kf_pipeline* pipeline, uint32_t* grid, size_t count);
/* Dense storage: the march's skip structures as the last integration left
 * them (no counterpart in the reference, whose march reads the voxels).  Per
 * 8^3 brick, x-major brick order: its class (0 mixed, 1 every stencil based
 * in it nullopt, 2 every such stencil exactly 1.0) and the radius in bricks
 * (0-7) of the cube around it, inside the brick grid, whose bricks all share
 * its class (0 for mixed bricks).  Per brick layer z (brick * 8 + z) the
 * 16-byte stencil record of the 64 stencils based in it, bit y*8+x: words
 * 0-1 "not decided by the corner bits", words 2-3 "exactly 1.0" for a
 * decided stencil and "every observed corner exactly 1.0" for an undecided
 * one.  `bricks` = the brick count; `records` holds bricks * 32 words.
 * KF_ERR_INVALID_ARGUMENT for sparse storage or before the structures
 * exist. */
kf_status kf_pipeline_download_skip_structures(kf_pipeline* pipeline, uint8_t* brick_class, uint8_t* brick_radius,
                                               uint32_t* records, size_t bricks);
/* The sparse block pool: capacity blocks of 512 raw voxels (slot order, each
 * block's voxels z*64 + y*8 + x, the reference's SparseVolumeView pool layout,
 * block_rep.hpp:93-100); `bytes` = capacity * 512 * voxel bytes.  With the
 * block grid it is the whole sparse volume without a dense expansion (no
 * reference counterpart: the reference exposes it only as host_view's dense
 * staging copy). */
kf_status kf_pipeline_download_pool(kf_pipeline* pipeline, void* voxels, size_t bytes);
/* band-march backend: the dilated band bitmap the raycast reads
 * (BasicBandBitmap::view, occupancy.hpp:262-267), one bit per 8^3 block in
 * z-major order (((x * blocks_y) + y) * blocks_z + z), count =
 * ceil(blocks / 32) words. */
kf_status kf_pipeline_download_band_bitmap(kf_pipeline* pipeline, uint32_t* words, size_t count);

/* Pipeline::extract_mesh (pipeline.hpp:95) on the device; free with kf_mesh_free. */
kf_status kf_pipeline_extract_mesh(kf_pipeline* pipeline, float min_weight, kf_mesh* out);
void kf_mesh_free(kf_mesh* mesh);
/* Waits for the pipeline's stream. */
kf_status kf_pipeline_synchronize(kf_pipeline* pipeline);
/* The pipeline's CUDA stream (a cudaStream_t) for callers that order or time
 * their own work against it. */
kf_status kf_pipeline_stream(kf_pipeline* pipeline, void** stream);
/* Two cudaEvent_t handles (or NULL) recorded on the pipeline's stream right
 * before and after each standalone integration kernel launch. */
kf_status kf_pipeline_set_kernel_events(kf_pipeline* pipeline, void* start, void* stop);
/* Cumulative fused voxel updates and colour updates since creation/reset
 * (the unit of the voxel-updates/s metric). */
kf_status kf_pipeline_update_counts(kf_pipeline* pipeline, uint64_t* voxel_updates,
                                    uint64_t* color_updates);

/* ---- comparator: Comparator::compare (comparison.hpp:30-38, comparison.cpp:12-81)
 * Deviations of a pipeline-set member against the set's reference member,
 * computed on the device (the reference downloads both volumes first).
 * Counts and maxima are exact; a mean is a double sum of the float
 * deviations over the compared count, cast to float (Deviation). */
typedef struct {
  uint64_t compared_voxels; /* observed (weight > 0) in both volumes */
  uint64_t only_primary;
  uint64_t only_reference;
  float max_distance_delta; /* |tsdf delta| */
  float mean_distance_delta;
  float max_weight_delta;
} kf_volume_comparison;   /* VolumeComparison (comparison.hpp:21-28) */

typedef struct {
  uint64_t compared_pixels; /* point and normal finite in both maps */
  uint64_t only_primary;
  uint64_t only_reference;
  float max_point_distance;
  float mean_point_distance;
  float max_normal_angle;   /* radians, atan2(|n x n'|, n . n') of the normalised normals */
  float mean_normal_angle;
} kf_surface_maps_comparison; /* SurfaceMapsComparison (comparison.hpp:11-19) */

/* Comparator::compare(ConstHostVolumeView, ConstHostVolumeView) over two
 * pipelines' volumes in place; voxel formats and storages may differ, the
 * geometries must match (KF_ERR_INVALID_ARGUMENT otherwise). */
kf_status kf_compare_volumes(kf_pipeline* primary, kf_pipeline* reference, kf_volume_comparison* out);
/* Comparator::compare(SurfaceMaps, SurfaceMaps); each side in host or device
 * memory (colors are not read and may be NULL); extents must match. */
kf_status kf_compare_surface_maps(const kf_surface_maps* primary, const kf_surface_maps* reference,
                                  kf_surface_maps_comparison* out);

/* ---- tensor-core GEMM of the learned warm-start (no counterpart in the
 * reference): c[m x n] (fp32) = a[m x k] * b[n x k]^T (+ bias[n]) (ReLU when
 * relu != 0), a and b bf16 row-major on the device, k a multiple of 8, all
 * three 16-byte aligned; stream is a cudaStream_t (NULL: the default
 * stream).  Runs on tcgen05 (sm_100a); a product of few 128-row output tiles
 * and long k is split along k over more CTAs (partials in a device workspace
 * the library allocates on first need and keeps, summed in a fixed order).
 * Waits for the product; concurrent calls from several threads take turns. */
kf_status kf_gemm_bf16(const void* a, const void* b, float* c, int32_t m, int32_t n, int32_t k,
                       const float* bias, int32_t relu, void* stream);

/* ---- launch shapes and the autotuner (no counterpart in the reference) ----
 * Shapes that leave every output bit unchanged: the march kernel's CTA
 * (raycast_block_x * raycast_block_y <= 64 threads), the fusion grid, and
 * the lanes that march each ray together (1, 2, 4, 8, 16 or 32; a warp then
 * holds 32 down to 1 rays) for renders of at most 20,000 rays, at most 80,000 rays,
 * and more.  Small renders have too few rays to fill the GPU one lane per
 * ray; with several lanes a ray takes up to that many samples per round. */
typedef struct {
  uint32_t raycast_block_x, raycast_block_y;
  uint32_t integrate_ctas;
  uint32_t raycast_lanes[3];
} kf_launch_shapes;
kf_status kf_pipeline_get_launch_shapes(kf_pipeline* pipeline, kf_launch_shapes* shapes);
kf_status kf_pipeline_set_launch_shapes(kf_pipeline* pipeline, const kf_launch_shapes* shapes);
/* Declares whether the pipeline's frames run beside other GPU work (the
 * members of a pipeline set, several sequences on their own streams; no
 * reference counterpart).  A pipeline alone (the default, concurrent = 0)
 * runs each ICP level as one cooperative launch, which needs all its CTAs
 * resident at once; a concurrent one records each level as per-step launches
 * that can share the GPU.  Results are bit-identical either way. */
kf_status kf_pipeline_set_concurrent(kf_pipeline* pipeline, int32_t concurrent);
/* Times the candidate shapes on a scratch pipeline of the same configuration
 * over `count` consecutive device-resident width x height depth frames (the
 * first fused, the rest tracked), applies the fastest to `pipeline` and
 * returns it (and its time for frames 1..count-1 in best_ms, may be NULL). */
kf_status kf_pipeline_autotune(kf_pipeline* pipeline, const uint16_t* frames, uint32_t count,
                               uint32_t width, uint32_t height, kf_intrinsics intrinsics,
                               kf_launch_shapes* chosen, float* best_ms);

/* ---- tracker: ProjectiveIcpTracker::estimate_pose(DeviceTrackingRequest)
 * (icp_optimizer.hpp:115-116, icp_optimizer.cpp:58-76) with the device solve. */
kf_status kf_tracker_create(const kf_icp_options* options, kf_tracker** out);
kf_status kf_tracker_destroy(kf_tracker* tracker);
/* Test hook of the bounded device waits (no reference counterpart).  Each
 * ICP level runs as one cooperative kernel whose CTAs meet at a grid barrier
 * once per Gauss-Newton step; every wait there gives up after 250 ms.  This
 * arms the tracker so that the barrier of its next level never completes
 * (its start count is set beyond any count the arrivals reach): the waits
 * run out, the frame
 * is marked failed (no integration), and the call that reads the result
 * returns KF_ERR_DEVICE_TIMEOUT and clears the barrier, after which the
 * tracker runs normally.  Call it with no work of the tracker in flight. */
kf_status kf_tracker_stall_next_level(kf_tracker* tracker);
/* Renders the model at `camera` and tracks `live` against it for `iterations`
 * Gauss-Newton steps starting from camera->camera_to_world
 * (Pipeline::track, pipeline.hpp:84-85 + IcpConsumer, reconstruction.cpp:63-67). */
kf_status kf_pipeline_track(kf_pipeline* pipeline, kf_tracker* tracker,
                            const kf_raycast_camera* camera, const kf_level_view* live,
                            uint32_t iterations, kf_icp_outcome* outcome);
/* The model render of Pipeline::track (pipeline.hpp:83-85,
 * device_pipeline.cu:133-136): the volume raycast at `camera` into the
 * pipeline's cached device maps of that extent; `out` receives their device
 * views (KF_MEMORY_DEVICE), valid until the next render of the same extent. */
kf_status kf_pipeline_render_model(kf_pipeline* pipeline, const kf_raycast_camera* camera,
                                   kf_surface_maps* out);
/* The whole-level device Gauss-Newton loop over given device maps
 * (BasicDeviceCorrespondenceSweep::run_loop, icp_correspondence.hpp:366-369,
 * icp_correspondence.cu:397-439): `iterations` steps from
 * initial_camera_to_world against the model rendered with model_intrinsics
 * at model_world_to_camera's inverse, with the tracker's options, one host
 * sync at the end.  sums (29 floats, may be NULL) receives the normal
 * equations of the last step. */
kf_status kf_icp_level(kf_tracker* tracker, const kf_level_view* live, const float* model_points,
                       const float* model_normals, uint32_t model_width, uint32_t model_height,
                       kf_intrinsics model_intrinsics, const kf_rigid* model_world_to_camera,
                       const kf_rigid* initial_camera_to_world, uint32_t iterations, kf_icp_outcome* outcome,
                       float* sums);
/* One correspondence sweep (BasicDeviceCorrespondenceSweep::run,
 * icp_correspondence.cu:572-597): fills sums[29] (21 JtJ + 6 Jtr + distance
 * sum + squared residual sum) and the match count.  Device views. */
kf_status kf_icp_normal_equations(kf_tracker* tracker, const kf_level_view* live,
                                  const float* model_points, const float* model_normals,
                                  uint32_t model_width, uint32_t model_height,
                                  kf_intrinsics model_intrinsics, const kf_rigid* camera,
                                  const kf_rigid* model_world_to_camera, float* sums,
                                  uint64_t* count);

/* The same sweep without any allocation (no counterpart in the reference).
 * For callers that must not allocate device memory: plug-ins whose host
 * application owns every byte of the GPU through its own memory pool (a
 * cudaMalloc of theirs would bypass the pool's budget and can fail or evict
 * the host's data), hosts that forbid cudaMalloc after start-up, and real-time
 * loops that stay off the allocator because cudaMalloc may synchronise the
 * device and stall the loop.  No tracker object is needed, and the per-CTA
 * partial sums live in a fixed device array (about 150 KB, present on every
 * GPU that loads the library until the process exits).  Live images of at
 * most 1,228,800 pixels (1200 CTAs of 1024 pixels) are accepted; larger ones
 * return KF_ERR_INVALID_ARGUMENT.  The first call on each device looks up the
 * array's address; make that first call before any stream capture.  Every
 * call shares the array: calls that overlap on the GPU (for example from two
 * host threads) race.  The call is synchronous: it runs on the legacy default
 * stream with blocking copies and returns after the results are copied to
 * `sums` and `count`. */
kf_status kf_icp_normal_equations_static(const kf_level_view* live, const float* model_points,
                                         const float* model_normals, uint32_t model_width,
                                         uint32_t model_height, kf_intrinsics model_intrinsics,
                                         const kf_rigid* camera, const kf_rigid* model_world_to_camera,
                                         float max_point_distance, float min_normal_dot, float* sums,
                                         uint64_t* count);

/* ---- whole frame (Reconstruction::process_frame, reconstruction.cpp:184-216)
 * pyramid -> per level (raycast at the current estimate, ICP) -> integrate at
 * the tracked pose, as one CUDA graph with one host sync.  depth is
 * width*height uint16 in `memory`; color may be NULL.  `pose` is the
 * camera_to_world the frame starts from and receives the result.  When
 * `first_frame` is set the frame is fused at `pose` without tracking
 * (Reconstruction::initialize, reconstruction.cpp:143-182).  Host inputs in
 * page-locked memory are copied to the device straight from the caller's
 * buffers; pageable ones through the pipeline's pinned staging. */
kf_status kf_frame_process(kf_pipeline* pipeline, kf_pyramid* pyramid, kf_tracker* tracker,
                           const uint16_t* depth, const uint32_t* color, uint32_t width,
                           uint32_t height, kf_intrinsics intrinsics, int32_t memory,
                           const uint32_t* iterations_per_level, int32_t first_frame,
                           kf_rigid* pose, kf_frame_result* result);
/* Same, without the host sync: the pose stays on the device, result may be
 * read later with kf_frame_result_fetch. */
kf_status kf_frame_enqueue(kf_pipeline* pipeline, kf_pyramid* pyramid, kf_tracker* tracker,
                           const uint16_t* depth, const uint32_t* color, uint32_t width,
                           uint32_t height, kf_intrinsics intrinsics, int32_t memory,
                           const uint32_t* iterations_per_level, int32_t first_frame);
kf_status kf_frame_result_fetch(kf_pipeline* pipeline, kf_frame_result* result);
/* Frames in flight, for loops that read every frame's result but need not
 * wait for it before sending the next frame (the reference's loop waits,
 * reconstruction.cpp:184-216): kf_frame_submit is kf_frame_enqueue plus a
 * copy of the frame's result into a queue of eight; host inputs are staged
 * while earlier frames still run.  kf_frame_result_next waits for the oldest
 * queued frame only and returns its result; submitting a ninth frame before
 * reading one is KF_ERR_INVALID_ARGUMENT. */
kf_status kf_frame_submit(kf_pipeline* pipeline, kf_pyramid* pyramid, kf_tracker* tracker,
                          const uint16_t* depth, const uint32_t* color, uint32_t width,
                          uint32_t height, kf_intrinsics intrinsics, int32_t memory,
                          const uint32_t* iterations_per_level, int32_t first_frame);
kf_status kf_frame_result_next(kf_pipeline* pipeline, kf_frame_result* result);
/* Kernel launches in one frame graph: the kernel nodes of the graph that the
 * last kf_frame_enqueue / kf_frame_process launched (this library's kernels;
 * copies, memsets and event records are not kernels).  No counterpart in the
 * reference, which launches frame by frame from the host. */
kf_status kf_frame_kernel_count(kf_pipeline* pipeline, uint32_t* kernels);

/* ---- batches of independent sequences (no counterpart in the reference) ----
 * Members are (pipeline, pyramid, tracker) triples of different volumes
 * (resolutions and storages may differ).  kf_batch_step runs one frame of
 * every member whose depth pointer is non-null as ONE graph launch: each
 * member's frame graph (the one kf_frame_enqueue would launch) is a branch
 * of the step's graph, so the members run concurrently.  Colour is not
 * batched.  first_frame (may be NULL) has one flag per member.  The step is
 * ordered after each active member's earlier work and before its later
 * work; kf_frame_result_fetch reads a member's result as usual. */
typedef struct kf_batch kf_batch;
kf_status kf_batch_create(kf_pipeline* const* pipelines, kf_pyramid* const* pyramids,
                          kf_tracker* const* trackers, uint32_t count, kf_batch** out);
kf_status kf_batch_destroy(kf_batch* batch);
kf_status kf_batch_step(kf_batch* batch, const uint16_t* const* depths, uint32_t width,
                        uint32_t height, const kf_intrinsics* intrinsics,
                        const uint32_t* iterations_per_level, const uint8_t* first_frame,
                        int32_t memory);
/* The stream the steps run on (a cudaStream_t). */
kf_status kf_batch_stream(kf_batch* batch, void** stream);
/* Kernel nodes of the last step's graph. */
kf_status kf_batch_kernel_count(kf_batch* batch, uint32_t* kernels);

/* ---- learned ICP warm start (no counterpart in the reference) ------------
 * A bf16 CNN on the tcgen05 tensor cores reads two 80x60 maps - the current
 * depth (8x8 block means) and the model rendered at the constant-velocity
 * pose - and proposes the twist from that pose to the tracked one.
 * Layers: four 3x3 stride-2 pad-1 convolutions (2-32-32-64-64, ReLU), then
 * 1280-256 (ReLU) and 256-6.  The parameters are one flat fp32 vector: per
 * layer the weights [out][in] then the bias, every tensor starting at a
 * multiple of 8 floats; convolution weights are [out][c*9 + ky*3 + kx], conv1
 * padded to 24 columns whose last 6 stay zero.  Inputs are NHWC bf16
 * [batch][60][80][2] (channel 0: current depth minus the mean predicted
 * depth; channel 1: 10 x (current - predicted) clamped to [-1, 1]; metres, 0
 * where invalid); outputs [batch][6] = (tx, ty, tz, wx, wy, wz) times
 * KF_WARM_START_TWIST_SCALE, applied as pose * exp: translation added in the
 * pose's frame, rotation by Rodrigues' formula.  Batches are multiples of 8. */
#define KF_WARM_START_TWIST_SCALE 50.0
typedef struct kf_learner kf_learner;
kf_status kf_learner_create(uint32_t batch_capacity, uint32_t seed, kf_learner** out);
kf_status kf_learner_destroy(kf_learner* learner);
kf_status kf_learner_param_count(kf_learner* learner, uint64_t* count);
kf_status kf_learner_get_params(kf_learner* learner, float* host);
kf_status kf_learner_set_params(kf_learner* learner, const float* host);
/* Forward pass of device inputs into device outputs [batch][6] (async). */
kf_status kf_learner_forward(kf_learner* learner, const void* inputs, uint32_t batch, float* out, void* stream);
/* Gradient of the batch mean of the squared error against device targets
 * [batch][6] into host_grads (param_count floats) and the loss into *loss
 * (both host, either may be NULL).  Synchronous. */
kf_status kf_learner_gradients(kf_learner* learner, const void* inputs, const float* targets, uint32_t batch,
                               float* host_grads, float* loss, void* stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on that loss; `loss` (a device
 * float, may be NULL) receives the loss before the step.  Async. */
kf_status kf_learner_train_step(kf_learner* learner, const void* inputs, const float* targets, uint32_t batch,
                                float learning_rate, float* loss, void* stream);
/* 1 when a tensor-core wait of an earlier async call timed out (synchronises). */
kf_status kf_learner_error(kf_learner* learner, int32_t* timed_out);

typedef struct kf_warm_start kf_warm_start;
typedef struct {
  kf_rigid start;          /* the pose ICP should start from */
  kf_rigid proposal;       /* predicted * exp(twist) */
  float twist[6];          /* unscaled */
  float cost_predicted, matches_predicted;
  float cost_proposal, matches_proposal;
  int32_t used_proposal;   /* 0: the constant-velocity pose was kept */
} kf_warm_start_result;
kf_status kf_warm_start_create(float depth_scale, kf_warm_start** out);
kf_status kf_warm_start_destroy(kf_warm_start* warm);
/* The net input of one 640x480 depth frame against the model rendered at
 * render_pose, into `input` (device, 9600 bf16, 16-byte aligned).  Ordered on
 * the pipeline's stream. */
kf_status kf_warm_start_input(kf_warm_start* warm, kf_pipeline* pipeline, const uint16_t* depth, uint32_t width,
                              uint32_t height, kf_intrinsics intrinsics, int32_t memory, const kf_rigid* render_pose,
                              void* input);
/* The start pose for the next frame: the net's proposal when its truncated
 * point-to-plane cost (80x60, against the model rendered at `predicted`, 5 cm
 * cap, unmatched pixels at the cap) is not above that of `predicted`, else
 * `predicted`.  Call before kf_frame_process of the same depth frame. */
kf_status kf_warm_start_propose(kf_warm_start* warm, kf_learner* learner, kf_pipeline* pipeline,
                                const uint16_t* depth, uint32_t width, uint32_t height, kf_intrinsics intrinsics,
                                int32_t memory, const kf_rigid* predicted, kf_warm_start_result* result);
/* The same step kept on the device, for loops that enqueue frames without a
 * host round trip (kf_frame_enqueue): ordered on the pipeline's stream, it
 * reads the tracker's pose (the previous frame's result), predicts the
 * constant-velocity pose from it and the pose the previous call read (the
 * pose itself on the first call after kf_warm_start_reset), and, with
 * use_net, runs the net and the fallback test; the chosen start is written
 * into the tracker as kf_frame_set_pose does.  Call it once before each
 * tracked frame; kf_warm_start_fetch (synchronises) reads the last step's
 * candidates, costs and choice. */
kf_status kf_warm_start_reset(kf_warm_start* warm);
kf_status kf_warm_start_enqueue(kf_warm_start* warm, kf_learner* learner, kf_pipeline* pipeline, kf_tracker* tracker,
                                const uint16_t* depth, uint32_t width, uint32_t height, kf_intrinsics intrinsics,
                                int32_t memory, int32_t use_net);
kf_status kf_warm_start_fetch(kf_warm_start* warm, kf_pipeline* pipeline, kf_warm_start_result* result);

/* ---- files around the loop (host code) ---------------------------------
 * PNG frames as a TUM RGB-D sequence stores them (read_png.cpp / write_png.cpp,
 * VirtualSensor, virtual_sensor.cpp:41-147) and binary PLY output
 * (FrameOutput, frame_output.cpp:76-181).  Failures return KF_ERR_IO. */
/* Size and pixel format of a PNG file (color_type, bit_depth may be NULL). */
kf_status kf_png_info(const char* path, uint32_t* width, uint32_t* height, int32_t* color_type, int32_t* bit_depth);
/* read_png<DepthImage>: the file must be 16-bit grayscale; raw values copied. */
kf_status kf_png_read_depth(const char* path, uint16_t* out, uint32_t width, uint32_t height);
/* read_png<ColorImage>: any 8/16-bit grey, grey+alpha, RGB, RGBA or 8-bit
 * palette image as RGBA8 packed R | G << 8 | B << 16 | A << 24. */
kf_status kf_png_read_color(const char* path, uint32_t* out, uint32_t width, uint32_t height);
kf_status kf_png_write_depth(const char* path, const uint16_t* depth, uint32_t width, uint32_t height);
kf_status kf_png_write_color(const char* path, const uint32_t* rgba, uint32_t width, uint32_t height);
/* FrameOutput::write_mesh: binary little-endian PLY, vertices (position,
 * normal, uchar colour clamped to [0, 255]) and triangles (host mesh). */
kf_status kf_mesh_write_ply(const char* path, const kf_mesh* mesh);
/* FrameOutput::write_raycast_point_cloud: every pixel whose point and
 * normal are finite (host maps, width*height*3 floats each, RGBA8 colours). */
kf_status kf_maps_write_ply(const char* path, const float* points, const float* normals, const uint32_t* colors,
                            uint32_t width, uint32_t height);

/* Sets the device-resident camera_to_world that the next enqueued frame
 * starts from (ordered on the pipeline's stream). */
kf_status kf_frame_set_pose(kf_pipeline* pipeline, kf_tracker* tracker, const kf_rigid* pose);

#ifdef __cplusplus
}
#endif

#endif /* KF_B200_H */
