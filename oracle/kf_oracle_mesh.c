/*
 * kf_oracle_mesh.c - mesh storage helpers of the oracle (the marching cubes
 * themselves are in kf_oracle.c, next to the sampler they use).
 *
 * TEST INFRASTRUCTURE ONLY.
 */
#include <stdlib.h>
#include <string.h>

#include "kf_oracle.h"
#include "kf_mc_tables.h"

void kfo_mesh_free(kf_mesh* mesh) {
  free(mesh->positions);
  free(mesh->normals);
  free(mesh->colors);
  free(mesh->triangles);
  memset(mesh, 0, sizeof(*mesh));
}

/* Triangles per sign case of the triangulation table. */
void kfo_mc_case_triangle_counts(int32_t* counts) {
  for (int i = 0; i < 256; ++i) {
    int n = 0;
    while (n < 5 && kMcTriangles[i][3 * n] >= 0) ++n;
    counts[i] = n;
  }
}
