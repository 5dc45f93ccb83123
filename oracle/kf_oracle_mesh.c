/*
 * kf_oracle_mesh.c - marching cubes of the oracle (filled in with the mesher).
 *
 * TEST INFRASTRUCTURE ONLY.
 */
#include <stdlib.h>
#include <string.h>

#include "kf_oracle.h"

kf_status kfo_marching_cubes(const kfo_volume* volume, float min_weight, kf_mesh* out) {
  (void)volume;
  (void)min_weight;
  memset(out, 0, sizeof(*out));
  return KF_ERR_UNSUPPORTED;
}

void kfo_mesh_free(kf_mesh* mesh) {
  free(mesh->positions);
  free(mesh->normals);
  free(mesh->colors);
  free(mesh->triangles);
  memset(mesh, 0, sizeof(*mesh));
}

void kfo_mc_case_triangle_counts(int32_t* counts) {
  for (int i = 0; i < 256; ++i) counts[i] = 0;
}
