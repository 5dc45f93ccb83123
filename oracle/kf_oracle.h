/*
 * kf_oracle.h - CPU restatement of maximsolodukhin/KinectFusion's host path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * sm_100a kernels in kinectfusion_b200/: tests, the smoke check and the CPU
 * baseline leg of bench.py may call it; the product path never does.
 *
 * This file restates the host algorithms function by function, in IEEE
 * single precision with the reference's operation order (built with
 * -ffp-contract=off, like an x86-64 build without FMA), citing the reference
 * file:line each function follows.  It is pinned two ways: against the
 * reference's own known-answer tests (test/tests.cpp), re-expressed in
 * tests/test_oracle_pins.py, and against the reference itself - its CPU
 * translation units compiled from source with an Eigen stand-in
 * (oracle/ref_build.sh -> oracle/_ref/libkf_ref.so) and compared on the same
 * inputs in tests/test_oracle_vs_reference.py.
 */
#ifndef KF_ORACLE_H
#define KF_ORACLE_H

#include <stdint.h>

#include "../include/kf_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Storage of one volume.  voxels: KF_VOXEL_FLOAT -> 2 floats per voxel
 * (tsdf, weight); QUANTIZED/BF16 -> one uint32 per voxel (low 16 bits
 * distance, high 16 bits weight).  colors: 4 floats per voxel or NULL.
 * Sparse volumes (grid != NULL) hold `capacity` 8^3 blocks in the pools and
 * a block-slot grid over the block extent (block_rep.hpp:26-110). */
typedef struct {
  kf_volume_geometry geometry;
  int32_t voxel;
  void* voxels;
  float* colors;
  uint32_t* grid;
  uint32_t* marked_frame;
  uint32_t* work_list;
  uint64_t capacity;
  uint64_t allocated;
  uint64_t work_count;
  uint32_t frame_stamp;
} kfo_volume;

/* Fresh unobserved volume contents (volume.hpp:115-117, BasicVolume fill). */
void kfo_volume_clear(kfo_volume* volume);
uint64_t kfo_observed_voxel_count(const kfo_volume* volume);
/* Decoded (tsdf, weight) of voxel (x, y, z); returns 0 when the voxel's
 * block is not allocated (sparse). */
int kfo_voxel_at(const kfo_volume* volume, uint32_t x, uint32_t y, uint32_t z, float* tsdf,
                 float* weight);

/* ---- depth processing (include/kinectfusion/depth_processing.hpp) ---- */
void kfo_bilateral(const uint16_t* depth, uint32_t width, uint32_t height,
                   const kf_depth_options* options, uint16_t* out);
void kfo_downsample(const uint16_t* depth, uint32_t width, uint32_t height,
                    const kf_depth_options* options, uint16_t* out);
void kfo_vertices(const uint16_t* depth, uint32_t width, uint32_t height, kf_intrinsics intrinsics,
                  const kf_depth_options* options, float* out);
void kfo_normals(const float* vertices, uint32_t width, uint32_t height,
                 const kf_depth_options* options, float* out);
kf_intrinsics kfo_scaled_intrinsics(kf_intrinsics intrinsics, uint32_t level);

/* ---- TSDF integration (include/kinectfusion/tsdf_integration.hpp) ---- */
void kfo_integrate(kfo_volume* volume, const kf_frame_view* frame,
                   const kf_integration_options* options, int32_t rule, int32_t threads);
/* Band mode over a dense volume (BandIntegrationSweep<kHost>, tsdf_integration.hpp:434-497). */
void kfo_integrate_band(kfo_volume* volume, const kf_frame_view* frame,
                        const kf_integration_options* options, int32_t rule);
/* Sparse allocation + listed-block integration (BlockRep<kHost>, block_rep.hpp:193-329). */
/* The device band sweep: the same walk at half-block steps. */
void kfo_integrate_band_device(kfo_volume* volume, const kf_frame_view* frame,
                               const kf_integration_options* options, int32_t rule);
/* The same integration in FP64 into (tsdf, weight) double pairs, x fastest. */
void kfo_integrate_f64(double* voxels, const kf_volume_geometry* geometry, const kf_frame_view* frame,
                       const kf_integration_options* options, int32_t rule, int32_t threads);
void kfo_integrate_sparse(kfo_volume* volume, const kf_frame_view* frame,
                          const kf_integration_options* options, int32_t rule);

/* ---- raycasting (include/kinectfusion/raycasting.hpp) ---- */
/* The band bitmap of a dense volume (BandRebuild<kHost>, occupancy.hpp:229-238):
 * raw and dilated words, kfo_band_word_count of each, z-major block bits. */
uint64_t kfo_band_word_count(const kfo_volume* volume);
void kfo_band_bitmap(const kfo_volume* volume, uint32_t* raw, uint32_t* dilated);
/* The band-march raycast (BandSkip over the dilated band words). */
void kfo_raycast_band(const kfo_volume* volume, const uint32_t* band_words, const kf_raycast_camera* camera,
                      const kf_raycast_options* options, float* points, float* normals, uint32_t* colors,
                      int32_t threads);
void kfo_raycast(const kfo_volume* volume, const kf_raycast_camera* camera,
                 const kf_raycast_options* options, float* points, float* normals,
                 uint32_t* colors, int32_t threads);

/* ---- projective ICP (icp_correspondence.hpp, icp_optimizer.cpp) ---- */
/* One correspondence sweep; sums[29] = 21 JtJ, 6 Jtr, distance sum, squared
 * residual sum, accumulated in float in pixel order. */
void kfo_icp_equations(const float* live_vertices, const float* live_normals, uint32_t live_width,
                       uint32_t live_height, const float* model_points, const float* model_normals,
                       uint32_t model_width, uint32_t model_height, kf_intrinsics model_intrinsics,
                       const kf_rigid* camera, const kf_rigid* model, float max_point_distance,
                       float min_normal_dot, float* sums, uint64_t* count);
/* The same sweep accumulated in double (the FP64 oracle reduction). */
void kfo_icp_equations_f64(const float* live_vertices, const float* live_normals,
                           uint32_t live_width, uint32_t live_height, const float* model_points,
                           const float* model_normals, uint32_t model_width, uint32_t model_height,
                           kf_intrinsics model_intrinsics, const kf_rigid* camera,
                           const kf_rigid* model, float max_point_distance, float min_normal_dot,
                           double* sums, uint64_t* count);
/* ProjectiveIcpTracker::estimate_with over host surfaces (icp_optimizer.cpp:208-302). */
void kfo_icp_estimate(const float* live_vertices, const float* live_normals, uint32_t live_width,
                      uint32_t live_height, const float* model_points, const float* model_normals,
                      uint32_t model_width, uint32_t model_height, kf_intrinsics model_intrinsics,
                      const kf_rigid* model_camera_to_world, const kf_rigid* initial_camera_to_world,
                      uint32_t iterations, const kf_icp_options* options, kf_icp_outcome* outcome);

/* Rigid helpers shared by the tests (vector.hpp:228-236). */
void kfo_rigid_inverse(const kf_rigid* in, kf_rigid* out);
void kfo_rigid_compose(const kf_rigid* a, const kf_rigid* b, kf_rigid* out);

/* ---- marching cubes (src/kinectfusion/marching_cubes.cpp:367-507) ---- */
kf_status kfo_marching_cubes(const kfo_volume* volume, float min_weight, kf_mesh* out);
void kfo_mesh_free(kf_mesh* mesh);
/* Triangle count of each of the 256 cube cases of the generated tables. */
void kfo_mc_case_triangle_counts(int32_t* counts);

#ifdef __cplusplus
}
#endif

#endif /* KF_ORACLE_H */
