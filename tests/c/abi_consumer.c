/* A plain C99 consumer of include/kf_b200.h: the header must compile as C
 * (no C++ types in the signatures) and the library must link and answer the
 * calls that need no GPU.  Built and run by tests/test_c_abi.py. */
#include <stdio.h>
#include <string.h>

#include "kf_b200.h"

int main(void) {
  kf_pipeline_config config;
  kf_depth_options depth;
  kf_icp_options icp;
  kf_volume_comparison volume_cmp;
  kf_surface_maps_comparison surface_cmp;
  kf_pipeline* pipeline = NULL;
  int32_t available = -1;
  memset(&volume_cmp, 0, sizeof volume_cmp);
  memset(&surface_cmp, 0, sizeof surface_cmp);
  if (kf_abi_version() != KF_B200_ABI_VERSION) return 1;
  kf_default_pipeline_config(&config);
  kf_default_depth_options(&depth);
  kf_default_icp_options(&icp);
  if (kf_device_available(&available) != KF_OK) return 2;
  /* null arguments are rejected before any device work */
  if (kf_pipeline_create(NULL, &pipeline) != KF_ERR_INVALID_ARGUMENT) return 3;
  if (kf_compare_volumes(NULL, NULL, &volume_cmp) != KF_ERR_INVALID_ARGUMENT) return 4;
  if (kf_compare_surface_maps(NULL, NULL, &surface_cmp) != KF_ERR_INVALID_ARGUMENT) return 5;
  if (kf_last_error() == NULL || kf_last_error()[0] == '\0') return 6;
  printf("%d %u %u %u %.3f %u %zu %zu\n", kf_abi_version(), config.volume.res_x, config.volume.res_y,
         config.volume.res_z, (double)config.volume.voxel_size, depth.levels, sizeof(kf_volume_comparison),
         sizeof(kf_surface_maps_comparison));
  return 0;
}
