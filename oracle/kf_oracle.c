/*
 * kf_oracle.c - CPU restatement of the reference host path (see kf_oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker, never the product.
 *
 * Arithmetic follows the reference's C++ expression order exactly; the file
 * must be compiled with -ffp-contract=off so that no multiply-add is fused
 * (oracle/Makefile).  Citations are file:line in maximsolodukhin/KinectFusion.
 */
#include "kf_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Vec3f / RigidTransform (include/kinectfusion/vector.hpp:21-236)           */
/* ------------------------------------------------------------------------ */
typedef struct {
  float x, y, z;
} v3;

static inline v3 v3m(float x, float y, float z) {
  v3 r = {x, y, z};
  return r;
}
static inline v3 v3add(v3 a, v3 b) { return v3m(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 v3sub(v3 a, v3 b) { return v3m(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 v3neg(v3 a) { return v3m(-a.x, -a.y, -a.z); }
static inline v3 v3mul(v3 a, float s) { return v3m(a.x * s, a.y * s, a.z * s); }
static inline v3 v3div(v3 a, float s) { return v3m(a.x / s, a.y / s, a.z / s); }
/* vector.hpp:140-143: (x*x' + y*y') + z*z' */
static inline float v3dot(v3 a, v3 b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }
static inline v3 v3cross(v3 a, v3 b) {
  return v3m((a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x));
}
static inline float v3norm(v3 a) { return sqrtf(v3dot(a, a)); }
/* Host branch of normalized (vector.hpp:164-175). */
static inline v3 v3normalized(v3 a) {
  const float length = v3norm(a);
  return length > 0.0f ? v3div(a, length) : v3m(0.0f, 0.0f, 0.0f);
}
static inline int v3finite(v3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
static inline v3 v3nan(void) { return v3m(NAN, NAN, NAN); }
static inline v3 v3load(const float* p) { return v3m(p[0], p[1], p[2]); }
static inline void v3store(float* p, v3 a) {
  p[0] = a.x;
  p[1] = a.y;
  p[2] = a.z;
}

/* Mat3f * Vec3f then + translation (vector.hpp:198-236). */
static inline v3 rot_apply(const kf_rigid* t, v3 p) {
  return v3m(v3dot(v3load(t->r), p), v3dot(v3load(t->r + 3), p), v3dot(v3load(t->r + 6), p));
}
static inline v3 rigid_apply(const kf_rigid* t, v3 p) {
  return v3add(rot_apply(t, p), v3load(t->t));
}

void kfo_rigid_inverse(const kf_rigid* in, kf_rigid* out) {
  /* vector.hpp:219-229: {R^T, -(R^T t)} */
  kf_rigid r;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      r.r[i * 3 + j] = in->r[j * 3 + i];
    }
  }
  const v3 t = v3load(in->t);
  const v3 rt = v3m(v3dot(v3load(r.r), t), v3dot(v3load(r.r + 3), t), v3dot(v3load(r.r + 6), t));
  v3store(r.t, v3neg(rt));
  *out = r;
}

/* 4x4 product a*b of rigid matrices, summed over k = 0..3 in order like a
 * column-major 4x4 float product (bottom row 0 0 0 1). */
void kfo_rigid_compose(const kf_rigid* a, const kf_rigid* b, kf_rigid* out) {
  float A[4][4], B[4][4], C[4][4];
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      A[i][j] = a->r[i * 3 + j];
      B[i][j] = b->r[i * 3 + j];
    }
    A[i][3] = a->t[i];
    B[i][3] = b->t[i];
  }
  for (int j = 0; j < 4; ++j) {
    A[3][j] = (j == 3) ? 1.0f : 0.0f;
    B[3][j] = (j == 3) ? 1.0f : 0.0f;
  }
  for (int i = 0; i < 4; ++i) {
    for (int j = 0; j < 4; ++j) {
      float s = A[i][0] * B[0][j];
      s = s + A[i][1] * B[1][j];
      s = s + A[i][2] * B[2][j];
      s = s + A[i][3] * B[3][j];
      C[i][j] = s;
    }
  }
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      out->r[i * 3 + j] = C[i][j];
    }
    out->t[i] = C[i][3];
  }
}

/* ------------------------------------------------------------------------ */
/* Sensor conventions (rgbd.hpp:36-137)                                      */
/* ------------------------------------------------------------------------ */
/* depth_in_range (rgbd.hpp:122-133); returns 0 for a missing sample. */
static inline int depth_in_range(uint16_t raw, float scale, float min_d, float max_d, float* m) {
  if (raw == 0) {
    return 0;
  }
  const float meters = (float)raw / scale;
  if (meters < min_d || meters > max_d) {
    return 0;
  }
  *m = meters;
  return 1;
}

/* CameraIntrinsics::project (rgbd.hpp:40-44). */
static inline void project(kf_intrinsics k, v3 p, float* px, float* py) {
  *px = ((k.fx * p.x) / p.z) + k.cx;
  *py = ((k.fy * p.y) / p.z) + k.cy;
}

/* CameraIntrinsics::back_project (rgbd.hpp:52-56). */
static inline v3 back_project(kf_intrinsics k, float px, float py, float depth) {
  return v3m(((px - k.cx) * depth) / k.fx, ((py - k.cy) * depth) / k.fy, depth);
}

/* CameraIntrinsics::scaled (rgbd.hpp:66-70). */
kf_intrinsics kfo_scaled_intrinsics(kf_intrinsics k, uint32_t level) {
  const float scale = 1.0f / (float)(1u << level);
  kf_intrinsics r = {k.fx * scale, k.fy * scale, k.cx * scale, k.cy * scale};
  return r;
}

/* pixel_from_color (rgbd.hpp:88-98): truncating byte conversion, alpha 255. */
static inline uint32_t pixel_from_color(v3 c) {
  const float lo = 0.0f, hi = 255.0f;
  const float r = c.x < lo ? lo : (hi < c.x ? hi : c.x);
  const float g = c.y < lo ? lo : (hi < c.y ? hi : c.y);
  const float b = c.z < lo ? lo : (hi < c.z ? hi : c.z);
  return (uint32_t)r | ((uint32_t)g << 8) | ((uint32_t)b << 16) | (0xFFu << 24);
}

/* color_from_pixel (rgbd.hpp:102-107). */
static inline v3 color_from_pixel(uint32_t p) {
  return v3m((float)(p & 0xFFu), (float)((p >> 8) & 0xFFu), (float)((p >> 16) & 0xFFu));
}

/* ------------------------------------------------------------------------ */
/* Depth processing (depth_processing.hpp:54-284)                            */
/* ------------------------------------------------------------------------ */
void kfo_bilateral(const uint16_t* depth, uint32_t width, uint32_t height,
                   const kf_depth_options* o, uint16_t* out) {
  /* DepthProcessor<kHost>::bilateral_filter (depth_processing.cpp:98-108). */
  if (!o->bilateral_filter || o->bilateral_radius == 0) {
    memcpy(out, depth, (size_t)width * height * sizeof(uint16_t));
    return;
  }
  const float spatial_scale = -0.5f / (o->bilateral_spatial_sigma * o->bilateral_spatial_sigma);
  const float range_scale = -0.5f / (o->bilateral_depth_sigma * o->bilateral_depth_sigma);
  const int radius = o->bilateral_radius;
  const int w = (int)width, h = (int)height;
#pragma omp parallel for schedule(static)
  for (int row = 0; row < h; ++row) {
    for (int col = 0; col < w; ++col) {
      /* BilateralFilter::operator() (depth_processing.hpp:71-115) */
      float center;
      uint16_t result = 0;
      if (depth_in_range(depth[(size_t)row * w + col], o->depth_scale, o->min_depth, o->max_depth,
                         &center)) {
        const int x_begin = col - radius > 0 ? col - radius : 0;
        const int y_begin = row - radius > 0 ? row - radius : 0;
        const int x_end = col + radius < w - 1 ? col + radius : w - 1;
        const int y_end = row + radius < h - 1 ? row + radius : h - 1;
        float weighted_sum = 0.0f;
        float weight_sum = 0.0f;
        for (int y = y_begin; y <= y_end; ++y) {
          for (int x = x_begin; x <= x_end; ++x) {
            const uint16_t raw = depth[(size_t)y * w + x];
            float sample;
            if (!depth_in_range(raw, o->depth_scale, o->min_depth, o->max_depth, &sample)) {
              continue;
            }
            const float d2 = (float)(((x - col) * (x - col)) + ((y - row) * (y - row)));
            const float dd = sample - center;
            /* std::exp(float) in the reference is the C library's expf, which
             * differs from the correctly rounded value by one ulp for about
             * 1e-4 of the arguments; the oracle takes the correctly rounded
             * value (exp in double, rounded once), as the device does. */
            const float arg = (d2 * spatial_scale) + (dd * dd * range_scale);
            const float weight = (float)exp((double)arg);
            weighted_sum += weight * (float)raw;
            weight_sum += weight;
          }
        }
        if (weight_sum > 0.0f) {
          result = (uint16_t)lroundf(weighted_sum / weight_sum);
        }
      }
      out[(size_t)row * w + col] = result;
    }
  }
}

void kfo_downsample(const uint16_t* depth, uint32_t width, uint32_t height,
                    const kf_depth_options* o, uint16_t* out) {
  /* BlockDownsample::operator() (depth_processing.hpp:153-187) */
  const uint32_t ow = width / 2, oh = height / 2;
  for (uint32_t row = 0; row < oh; ++row) {
    for (uint32_t col = 0; col < ow; ++col) {
      uint32_t sum = 0, count = 0;
      uint16_t lo = 0xFFFF, hi = 0;
      for (uint32_t dy = 0; dy < 2; ++dy) {
        for (uint32_t dx = 0; dx < 2; ++dx) {
          const uint16_t s = depth[(size_t)(row * 2 + dy) * width + (col * 2 + dx)];
          if (s == 0) {
            continue;
          }
          sum += s;
          ++count;
          lo = s < lo ? s : lo;
          hi = hi < s ? s : hi;
        }
      }
      uint16_t result = 0;
      if (count != 0) {
        const float max_m = (float)hi / o->depth_scale;
        const float min_m = (float)lo / o->depth_scale;
        if (!(max_m - min_m > o->max_downsample_depth_jump)) {
          result = (uint16_t)((sum + (count / 2u)) / count);
        }
      }
      out[(size_t)row * ow + col] = result;
    }
  }
}

void kfo_vertices(const uint16_t* depth, uint32_t width, uint32_t height, kf_intrinsics k,
                  const kf_depth_options* o, float* out) {
  /* VertexProjection::operator() (depth_processing.hpp:215-226) with the
   * identity camera pose (depth_processing.cu:104-108). */
  for (uint32_t row = 0; row < height; ++row) {
    for (uint32_t col = 0; col < width; ++col) {
      float d;
      v3 v = v3nan();
      if (depth_in_range(depth[(size_t)row * width + col], o->depth_scale, o->min_depth,
                         o->max_depth, &d)) {
        v = back_project(k, (float)col, (float)row, d);
      }
      v3store(out + ((size_t)row * width + col) * 3, v);
    }
  }
}

void kfo_normals(const float* vertices, uint32_t width, uint32_t height, const kf_depth_options* o,
                 float* out) {
  /* NormalEstimation::operator() (depth_processing.hpp:251-279) */
  for (uint32_t row = 0; row < height; ++row) {
    for (uint32_t col = 0; col < width; ++col) {
      v3 n = v3nan();
      if (col != 0 && row != 0 && col + 1 < width && row + 1 < height) {
        const v3 c = v3load(vertices + ((size_t)row * width + col) * 3);
        const v3 l = v3load(vertices + ((size_t)row * width + col - 1) * 3);
        const v3 r = v3load(vertices + ((size_t)row * width + col + 1) * 3);
        const v3 t = v3load(vertices + ((size_t)(row - 1) * width + col) * 3);
        const v3 b = v3load(vertices + ((size_t)(row + 1) * width + col) * 3);
        const v3 s = v3add(v3add(v3add(v3add(c, l), r), t), b);
        if (v3finite(s) && !(fabsf(r.z - l.z) > o->max_normal_depth_jump ||
                             fabsf(b.z - t.z) > o->max_normal_depth_jump)) {
          const v3 nn = v3cross(v3sub(b, t), v3sub(r, l));
          const float length = v3norm(nn);
          if (length > 0.0f) {
            n = v3div(nn, length);
          }
        }
      }
      v3store(out + ((size_t)row * width + col) * 3, n);
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Voxel codecs (volume.hpp:25-193)                                          */
/* ------------------------------------------------------------------------ */
#define Q_SCALE 32767.0f
#define Q_INV_SCALE (1.0f / 32767.0f)
#define W_SCALE 256.0f
#define W_INV_SCALE (1.0f / 256.0f)
#define W_MAX (65535.0f / 256.0f)

static inline float clampf(float v, float lo, float hi) {
  if (v < lo) return lo;
  if (hi < v) return hi;
  return v;
}

static inline uint16_t bf16_encode(float t) {
  const float c = clampf(t, -1.0f, 1.0f);
  uint32_t bits;
  memcpy(&bits, &c, 4);
  return (uint16_t)((bits + 0x7FFFu + ((bits >> 16) & 1u)) >> 16);
}
static inline float bf16_decode(uint16_t raw) {
  const uint32_t bits = (uint32_t)raw << 16;
  float f;
  memcpy(&f, &bits, 4);
  return f;
}
static inline uint16_t qweight_encode(float w) { return (uint16_t)(clampf(w, 0.0f, W_MAX) * W_SCALE); }
static inline float qweight_decode(uint16_t raw) { return (float)raw * W_INV_SCALE; }
static inline int16_t qtsdf_encode(float t) { return (int16_t)(clampf(t, -1.0f, 1.0f) * Q_SCALE); }
static inline float qtsdf_decode(int16_t raw) { return (float)raw * Q_INV_SCALE; }

typedef struct {
  float tsdf, weight;
  int observed, finite;
} decoded_voxel;

static inline decoded_voxel decode_voxel(int32_t kind, const void* base, size_t index) {
  decoded_voxel d;
  if (kind == KF_VOXEL_FLOAT) {
    const float* f = (const float*)base + index * 2;
    d.tsdf = f[0];
    d.weight = f[1];
    d.observed = d.weight > 0.0f;
    d.finite = isfinite(d.tsdf);
  } else {
    const uint32_t raw = ((const uint32_t*)base)[index];
    const uint16_t draw = (uint16_t)(raw & 0xFFFFu);
    const uint16_t wraw = (uint16_t)(raw >> 16);
    d.tsdf = kind == KF_VOXEL_QUANTIZED ? qtsdf_decode((int16_t)draw) : bf16_decode(draw);
    d.weight = qweight_decode(wraw);
    d.observed = wraw != 0;
    d.finite = 1;
  }
  return d;
}

/* BasicVoxel::fused (volume.hpp:137-146) */
static inline void fuse_voxel(int32_t kind, void* base, size_t index, float observed, float ow,
                              float max_weight) {
  const decoded_voxel d = decode_voxel(kind, base, index);
  const float avg = ((d.tsdf * d.weight) + (observed * ow)) / (d.weight + ow);
  const float sum_w = d.weight + ow;
  const float w = max_weight < sum_w ? max_weight : sum_w;
  if (kind == KF_VOXEL_FLOAT) {
    float* f = (float*)base + index * 2;
    f[0] = avg;
    f[1] = w;
  } else {
    const uint16_t draw =
        kind == KF_VOXEL_QUANTIZED ? (uint16_t)qtsdf_encode(avg) : bf16_encode(avg);
    ((uint32_t*)base)[index] = (uint32_t)draw | ((uint32_t)qweight_encode(w) << 16);
  }
}

static uint32_t unobserved_raw(int32_t kind) {
  const uint16_t d = kind == KF_VOXEL_QUANTIZED ? (uint16_t)qtsdf_encode(1.0f) : bf16_encode(1.0f);
  return (uint32_t)d;
}

static inline int is_sparse(const kfo_volume* v) { return v->grid != NULL; }

static inline uint64_t blocks_along(uint32_t voxels) { return (voxels + 7u) / 8u; }

/* Storage index of voxel (x, y, z), or -1 when its block is unallocated. */
static inline int64_t storage_index(const kfo_volume* v, uint64_t x, uint64_t y, uint64_t z) {
  const kf_volume_geometry* g = &v->geometry;
  if (!is_sparse(v)) {
    return (int64_t)((z * g->res_y + y) * g->res_x + x);
  }
  const uint64_t bx = blocks_along(g->res_x), by = blocks_along(g->res_y);
  const uint64_t block = ((z / 8) * by + (y / 8)) * bx + (x / 8);
  const uint32_t slot = v->grid[block];
  if (slot == 0xFFFFFFFFu) {
    return -1;
  }
  return (int64_t)((uint64_t)slot * 512u + (((z % 8) * 8 + (y % 8)) * 8 + (x % 8)));
}

static uint64_t storage_voxel_count(const kfo_volume* v) {
  const kf_volume_geometry* g = &v->geometry;
  if (!is_sparse(v)) {
    return (uint64_t)g->res_x * g->res_y * g->res_z;
  }
  return v->capacity * 512u;
}

void kfo_volume_clear(kfo_volume* v) {
  const uint64_t n = storage_voxel_count(v);
  if (v->voxel == KF_VOXEL_FLOAT) {
    float* f = (float*)v->voxels;
    for (uint64_t i = 0; i < n; ++i) {
      f[2 * i] = 1.0f;
      f[2 * i + 1] = 0.0f;
    }
  } else {
    const uint32_t raw = unobserved_raw(v->voxel);
    uint32_t* u = (uint32_t*)v->voxels;
    for (uint64_t i = 0; i < n; ++i) {
      u[i] = raw;
    }
  }
  if (v->colors) {
    memset(v->colors, 0, n * 4 * sizeof(float));
  }
  if (is_sparse(v)) {
    const kf_volume_geometry* g = &v->geometry;
    const uint64_t blocks = blocks_along(g->res_x) * blocks_along(g->res_y) * blocks_along(g->res_z);
    for (uint64_t b = 0; b < blocks; ++b) {
      v->grid[b] = 0xFFFFFFFFu;
      if (v->marked_frame) v->marked_frame[b] = 0;
    }
    v->allocated = 0;
    v->work_count = 0;
    v->frame_stamp = 1;
  }
}

uint64_t kfo_observed_voxel_count(const kfo_volume* v) {
  /* VolumeReduction<kHost>::observed_voxel_count (volume.hpp:409-421) and
   * BlockRep::observed_voxel_count (block_rep.hpp:212-222). */
  uint64_t used = storage_voxel_count(v);
  if (is_sparse(v)) {
    const uint64_t a = v->allocated < v->capacity ? v->allocated : v->capacity;
    used = a * 512u;
  }
  uint64_t count = 0;
  for (uint64_t i = 0; i < used; ++i) {
    const decoded_voxel d = decode_voxel(v->voxel, v->voxels, i);
    if (is_sparse(v) ? d.observed : d.weight > 0.0f) {
      ++count;
    }
  }
  return count;
}

int kfo_voxel_at(const kfo_volume* v, uint32_t x, uint32_t y, uint32_t z, float* tsdf,
                 float* weight) {
  const int64_t i = storage_index(v, x, y, z);
  if (i < 0) {
    return 0;
  }
  const decoded_voxel d = decode_voxel(v->voxel, v->voxels, (size_t)i);
  *tsdf = d.tsdf;
  *weight = d.weight;
  return 1;
}

/* ------------------------------------------------------------------------ */
/* TSDF integration (tsdf_integration.hpp:127-342)                           */
/* ------------------------------------------------------------------------ */
typedef struct {
  const kf_frame_view* frame;
  const kf_integration_options* o;
  int32_t rule;
} icontext;

/* VolumeGeometry::cell_center (volume.hpp:276-283). */
static inline v3 cell_center(const kf_volume_geometry* g, uint64_t x, uint64_t y, uint64_t z) {
  const v3 start = v3m((float)x, (float)y, (float)z);
  const v3 c = v3mul(v3add(start, v3m(0.5f, 0.5f, 0.5f)), g->voxel_size);
  return v3add(v3m(g->origin[0], g->origin[1], g->origin[2]), c);
}

static inline float truncation_for(const kf_integration_options* o, float base, float depth) {
  if (o->distance_scaled_truncation) {
    return base + (o->truncation_distance_scale * depth);
  }
  return base;
}

/* IntegrationContext::observe + rule weight + fuse for one voxel
 * (tsdf_integration.hpp:183-263, 287-342). */
static inline void update_voxel(const kfo_volume* v, const icontext* ctx, uint64_t x, uint64_t y,
                                uint64_t z) {
  const kf_frame_view* f = ctx->frame;
  const kf_integration_options* o = ctx->o;
  const kf_volume_geometry* g = &v->geometry;
  const v3 cp = rigid_apply(&f->world_to_camera, cell_center(g, x, y, z));
  if (cp.z <= 0.0f) {
    return;
  }
  float px, py;
  project(f->intrinsics, cp, &px, &py);
  const long rx = lroundf(px), ry = lroundf(py);
  if (rx < 0 || ry < 0) {
    return;
  }
  if ((unsigned long)rx >= f->width || (unsigned long)ry >= f->height) {
    return;
  }
  const size_t pix = (size_t)ry * f->width + (size_t)rx;
  float surface_depth;
  if (!depth_in_range(f->depth[pix], o->depth_scale, o->min_depth, o->max_depth, &surface_depth)) {
    return;
  }
  const v3 ray = back_project(f->intrinsics, (float)rx, (float)ry, 1.0f);
  const float lambda = v3norm(ray);
  if (!v3finite(ray) || lambda == 0.0f) {
    return;
  }
  const float truncation = truncation_for(o, g->truncation_distance, surface_depth);
  const float sdf =
      o->projective_distance ? surface_depth - (v3norm(cp) / lambda) : surface_depth - cp.z;
  if (sdf < -truncation) {
    return;
  }
  const float tsdf = clampf(sdf / truncation, -1.0f, 1.0f);
  const int integrate_color = sdf <= truncation * 0.5f;

  float weight = o->observation_weight;
  if (ctx->rule == KF_RULE_ANGLE_WEIGHTED && f->normals != NULL) {
    const v3 n = v3load(f->normals + pix * 3);
    if (v3finite(n)) {
      const v3 view = v3neg(v3normalized(ray));
      const float d = v3dot(v3normalized(n), view);
      const float cos_theta = 0.0f < d ? d : 0.0f;
      weight *= cos_theta / surface_depth;
    }
  }
  if (weight <= 0.0f) {
    return;
  }
  const int64_t index = storage_index(v, x, y, z);
  fuse_voxel(v->voxel, v->voxels, (size_t)index, tsdf, weight, o->max_weight);
  if (v->colors != NULL && f->color != NULL && integrate_color) {
    /* ColorVoxel::fused (volume.hpp:160-170) */
    const v3 c = color_from_pixel(f->color[pix]);
    float* cv = v->colors + (size_t)index * 4;
    const v3 old = v3load(cv);
    const float w = cv[3];
    const v3 avg = v3div(v3add(v3mul(old, w), v3mul(c, weight)), w + weight);
    const float sum_w = w + weight;
    v3store(cv, avg);
    cv[3] = o->max_weight < sum_w ? o->max_weight : sum_w;
  }
}

void kfo_integrate(kfo_volume* v, const kf_frame_view* frame, const kf_integration_options* o,
                   int32_t rule, int32_t threads) {
  /* IntegrationSweep<kHost>::run (tsdf_integration.hpp:356-370). */
  const icontext ctx = {frame, o, rule};
  const kf_volume_geometry* g = &v->geometry;
  (void)threads;
#ifdef _OPENMP
  const int nt = threads > 0 ? threads : 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
#endif
  for (int64_t z = 0; z < (int64_t)g->res_z; ++z) {
    for (uint64_t y = 0; y < g->res_y; ++y) {
      for (uint64_t x = 0; x < g->res_x; ++x) {
        update_voxel(v, &ctx, x, y, (uint64_t)z);
      }
    }
  }
}

/* TruncationBandWalk::visit_pixel (tsdf_integration.hpp:384-428) */
typedef void (*visit_block_fn)(void* user, uint64_t block);

static void band_walk(const kf_frame_view* f, const kf_integration_options* o,
                      const kf_volume_geometry* g, float step, visit_block_fn visit, void* user) {
  kf_rigid camera_to_world;
  kfo_rigid_inverse(&f->world_to_camera, &camera_to_world);
  const uint64_t bx = blocks_along(g->res_x), by = blocks_along(g->res_y);
  for (uint32_t row = 0; row < f->height; ++row) {
    for (uint32_t col = 0; col < f->width; ++col) {
      float measured;
      if (!depth_in_range(f->depth[(size_t)row * f->width + col], o->depth_scale, o->min_depth,
                          o->max_depth, &measured)) {
        continue;
      }
      const float band = truncation_for(o, g->truncation_distance, measured);
      const float inv_voxel = 1.0f / g->voxel_size;
      const int samples = (int)((2.0f * band) / step) + 1;
      uint64_t previous = ~(uint64_t)0;
      for (int s = 0; s <= samples; ++s) {
        const float depth = (measured - band) + ((float)s * step);
        const v3 world =
            rigid_apply(&camera_to_world, back_project(f->intrinsics, (float)col, (float)row, depth));
        const v3 grid = v3mul(v3sub(world, v3m(g->origin[0], g->origin[1], g->origin[2])), inv_voxel);
        if (!(grid.x >= 0.0f && grid.y >= 0.0f && grid.z >= 0.0f && grid.x < (float)g->res_x &&
              grid.y < (float)g->res_y && grid.z < (float)g->res_z)) {
          continue;
        }
        const uint64_t ix = (uint64_t)grid.x, iy = (uint64_t)grid.y, iz = (uint64_t)grid.z;
        const uint64_t index = ((iz / 8) * by + (iy / 8)) * bx + (ix / 8);
        if (index == previous) {
          continue;
        }
        previous = index;
        visit(user, index);
      }
    }
  }
}

static void integrate_block(const kfo_volume* v, const icontext* ctx, uint64_t block) {
  /* BlockVoxels (grid.hpp:226-279): the block clamped to the resolution. */
  const kf_volume_geometry* g = &v->geometry;
  const uint64_t bx = blocks_along(g->res_x), by = blocks_along(g->res_y);
  const uint64_t x0 = (block % bx) * 8, y0 = ((block / bx) % by) * 8, z0 = (block / (bx * by)) * 8;
  for (uint64_t z = z0; z < z0 + 8 && z < g->res_z; ++z) {
    for (uint64_t y = y0; y < y0 + 8 && y < g->res_y; ++y) {
      for (uint64_t x = x0; x < x0 + 8 && x < g->res_x; ++x) {
        update_voxel(v, ctx, x, y, z);
      }
    }
  }
}

static void set_bit(void* user, uint64_t block) {
  uint32_t* bitmap = (uint32_t*)user;
  bitmap[block / 32] |= 1u << (block % 32);
}

static void integrate_band_with_step(kfo_volume* v, const kf_frame_view* frame,
                                     const kf_integration_options* o, int32_t rule, float step) {
  const kf_volume_geometry* g = &v->geometry;
  const uint64_t blocks = blocks_along(g->res_x) * blocks_along(g->res_y) * blocks_along(g->res_z);
  const uint64_t words = (blocks + 31) / 32;
  uint32_t* bitmap = (uint32_t*)calloc(words, sizeof(uint32_t));
  band_walk(frame, o, g, step, set_bit, bitmap);
  const icontext ctx = {frame, o, rule};
  for (uint64_t w = 0; w < words; ++w) {
    uint32_t word = bitmap[w];
    while (word) {
      const int bit = __builtin_ctz(word);
      word &= word - 1u;
      integrate_block(v, &ctx, w * 32 + (uint64_t)bit);
    }
  }
  free(bitmap);
}

void kfo_integrate_band(kfo_volume* v, const kf_frame_view* frame,
                        const kf_integration_options* o, int32_t rule) {
  /* BandIntegrationSweep<kHost>::run (tsdf_integration.hpp:439-471): the
   * host walks at voxel-size steps. */
  integrate_band_with_step(v, frame, o, rule, v->geometry.voxel_size);
}

void kfo_integrate_band_device(kfo_volume* v, const kf_frame_view* frame,
                               const kf_integration_options* o, int32_t rule) {
  /* BandIntegrationSweep<kDevice>::run (tsdf_integration.cu:240-291): the
   * device walks at half-block steps (band_walk.cuh:41-55,
   * TruncationBandWalk::half_block_step, tsdf_integration.hpp:379-382). */
  integrate_band_with_step(v, frame, o, rule, 0.5f * 8.0f * v->geometry.voxel_size);
}

static void sparse_allocate(void* user, uint64_t block) {
  /* BlockRep<kHost>::allocate (block_rep.hpp:291-308) */
  kfo_volume* v = (kfo_volume*)user;
  if (v->grid[block] != 0xFFFFFFFFu) {
    if (v->marked_frame[block] != v->frame_stamp) {
      v->marked_frame[block] = v->frame_stamp;
      v->work_list[v->work_count++] = (uint32_t)block;
    }
    return;
  }
  if (v->allocated >= v->capacity) {
    ++v->allocated;
    return;
  }
  const uint64_t slot = v->allocated++;
  v->grid[block] = (uint32_t)slot;
  v->marked_frame[block] = v->frame_stamp;
  v->work_list[v->work_count++] = (uint32_t)block;
}

void kfo_integrate_sparse(kfo_volume* v, const kf_frame_view* frame,
                          const kf_integration_options* o, int32_t rule) {
  /* BlockRep<kHost>::integrate (block_rep.hpp:224-236) */
  const kf_volume_geometry* g = &v->geometry;
  ++v->frame_stamp;
  v->work_count = 0;
  band_walk(frame, o, g, 4.0f * g->voxel_size, sparse_allocate, v);
  const icontext ctx = {frame, o, rule};
  for (uint64_t i = 0; i < v->work_count; ++i) {
    integrate_block(v, &ctx, v->work_list[i]);
  }
}

/* ------------------------------------------------------------------------ */
/* Trilinear sampling (trilinear.hpp:85-269, volume_sampler.hpp:36-255)      */
/* ------------------------------------------------------------------------ */
typedef struct {
  const kfo_volume* v;
  float inv_voxel;
} sampler;

static inline int grid_contains(const kf_volume_geometry* g, v3 p) {
  return p.x >= 0.0f && p.y >= 0.0f && p.z >= 0.0f && p.x < (float)g->res_x &&
         p.y < (float)g->res_y && p.z < (float)g->res_z;
}

static inline v3 grid_coords(const sampler* s, v3 p) {
  const kf_volume_geometry* g = &s->v->geometry;
  return v3mul(v3sub(p, v3m(g->origin[0], g->origin[1], g->origin[2])), s->inv_voxel);
}

/* Corner storage index, clipped to the resolution; -1 = missing. */
static inline int64_t corner_index(const kfo_volume* v, int bx, int by, int bz) {
  const kf_volume_geometry* g = &v->geometry;
  if (bx < 0 || by < 0 || bz < 0 || (uint32_t)bx >= g->res_x || (uint32_t)by >= g->res_y ||
      (uint32_t)bz >= g->res_z) {
    return -1;
  }
  return storage_index(v, (uint64_t)bx, (uint64_t)by, (uint64_t)bz);
}

static inline float axis_weight(float fraction, int offset) {
  return offset == 0 ? 1.0f - fraction : fraction;
}

/* TrilinearSampler::tsdf + blend_tsdf; returns 0 for nullopt. */
static int sample_tsdf(const sampler* s, v3 point, int32_t policy, float* out) {
  const kf_volume_geometry* g = &s->v->geometry;
  const v3 grid = grid_coords(s, point);
  if (!grid_contains(g, grid)) {
    return 0;
  }
  const v3 gg = v3sub(grid, v3m(0.5f, 0.5f, 0.5f));
  const v3 fl = v3m(floorf(gg.x), floorf(gg.y), floorf(gg.z));
  const int bx = (int)fl.x, by = (int)fl.y, bz = (int)fl.z;
  const v3 fr = v3sub(gg, fl);
  float accumulated = 0.0f, weight_sum = 0.0f;
  int valid = 0;
  for (int oz = 0; oz <= 1; ++oz) {
    for (int oy = 0; oy <= 1; ++oy) {
      for (int ox = 0; ox <= 1; ++ox) {
        const int64_t i = corner_index(s->v, bx + ox, by + oy, bz + oz);
        if (i < 0) continue;
        const decoded_voxel d = decode_voxel(s->v->voxel, s->v->voxels, (size_t)i);
        if (!d.observed || !d.finite) continue;
        const float w = axis_weight(fr.x, ox) * axis_weight(fr.y, oy) * axis_weight(fr.z, oz);
        accumulated += w * d.tsdf;
        weight_sum += w;
        ++valid;
      }
    }
  }
  if (policy == KF_CORNERS_REQUIRE_ALL && valid < 8) {
    return 0;
  }
  if (weight_sum <= 1.0e-6f) {
    return 0;
  }
  const float distance = accumulated / weight_sum;
  if (!isfinite(distance)) {
    return 0;
  }
  *out = distance;
  return 1;
}

/* TrilinearSampler::color + blend_color. */
static int sample_color(const sampler* s, v3 point, v3* out) {
  const kf_volume_geometry* g = &s->v->geometry;
  if (s->v->colors == NULL) {
    return 0;
  }
  const v3 grid = grid_coords(s, point);
  if (!grid_contains(g, grid)) {
    return 0;
  }
  const v3 gg = v3sub(grid, v3m(0.5f, 0.5f, 0.5f));
  const v3 fl = v3m(floorf(gg.x), floorf(gg.y), floorf(gg.z));
  const int bx = (int)fl.x, by = (int)fl.y, bz = (int)fl.z;
  const v3 fr = v3sub(gg, fl);
  v3 acc = v3m(0.0f, 0.0f, 0.0f);
  float ws = 0.0f;
  for (int oz = 0; oz <= 1; ++oz) {
    for (int oy = 0; oy <= 1; ++oy) {
      for (int ox = 0; ox <= 1; ++ox) {
        const int64_t i = corner_index(s->v, bx + ox, by + oy, bz + oz);
        if (i < 0) continue;
        const float* c = s->v->colors + (size_t)i * 4;
        if (c[3] <= 0.0f) continue;
        const float w = axis_weight(fr.x, ox) * axis_weight(fr.y, oy) * axis_weight(fr.z, oz);
        acc = v3add(acc, v3mul(v3load(c), w));
        ws += w;
      }
    }
  }
  if (ws <= 1.0e-6f) {
    return 0;
  }
  *out = v3div(acc, ws);
  return 1;
}

/* trilinear::central_normal (trilinear.hpp:243-266) */
static int central_normal(const sampler* s, v3 p, int32_t policy, v3* out) {
  const float vs = s->v->geometry.voxel_size;
  float gradient[3];
  for (int axis = 0; axis < 3; ++axis) {
    const v3 dir = v3m(axis == 0 ? 1.0f : 0.0f, axis == 1 ? 1.0f : 0.0f, axis == 2 ? 1.0f : 0.0f);
    const v3 offset = v3mul(dir, vs);
    float plus, minus;
    if (!sample_tsdf(s, v3add(p, offset), policy, &plus)) return 0;
    if (!sample_tsdf(s, v3sub(p, offset), policy, &minus)) return 0;
    gradient[axis] = plus - minus;
  }
  const v3 d = v3m(gradient[0], gradient[1], gradient[2]);
  const float length = v3norm(d);
  if (length <= 0.0f) return 0;
  *out = v3div(d, length);
  return 1;
}

/* TrilinearSampler::cell_normal (volume_sampler.hpp:189-239) */
static int cell_normal(const sampler* s, v3 p, v3* out) {
  const kf_volume_geometry* g = &s->v->geometry;
  const v3 grid = grid_coords(s, p);
  if (!grid_contains(g, grid)) return 0;
  const v3 gg = v3sub(grid, v3m(0.5f, 0.5f, 0.5f));
  const v3 fl = v3m(floorf(gg.x), floorf(gg.y), floorf(gg.z));
  const int bx = (int)fl.x, by = (int)fl.y, bz = (int)fl.z;
  const v3 f = v3sub(gg, fl);
  float c[2][2][2];
  for (int oz = 0; oz <= 1; ++oz) {
    for (int oy = 0; oy <= 1; ++oy) {
      for (int ox = 0; ox <= 1; ++ox) {
        const int64_t i = corner_index(s->v, bx + ox, by + oy, bz + oz);
        if (i < 0) return central_normal(s, p, KF_CORNERS_SKIP_MISSING, out);
        const decoded_voxel d = decode_voxel(s->v->voxel, s->v->voxels, (size_t)i);
        if (!d.observed || !d.finite) return central_normal(s, p, KF_CORNERS_SKIP_MISSING, out);
        c[oz][oy][ox] = d.tsdf;
      }
    }
  }
  /* trilinear::cell_gradient (trilinear.hpp:205-238): lerp(l, h, m) = l + m*(h-l) */
#define LERP(l, h, m) ((l) + ((m) * ((h) - (l))))
  const float gx = LERP(LERP(c[0][0][1] - c[0][0][0], c[0][1][1] - c[0][1][0], f.y),
                        LERP(c[1][0][1] - c[1][0][0], c[1][1][1] - c[1][1][0], f.y), f.z);
  const float gy = LERP(LERP(c[0][1][0] - c[0][0][0], c[0][1][1] - c[0][0][1], f.x),
                        LERP(c[1][1][0] - c[1][0][0], c[1][1][1] - c[1][0][1], f.x), f.z);
  const float gz = LERP(LERP(c[1][0][0] - c[0][0][0], c[1][0][1] - c[0][0][1], f.x),
                        LERP(c[1][1][0] - c[0][1][0], c[1][1][1] - c[0][1][1], f.x), f.y);
#undef LERP
  const v3 gr = v3m(gx, gy, gz);
  const float length = v3norm(gr);
  if (length <= 0.0f) return 0;
  *out = v3div(gr, length);
  return 1;
}

/* ------------------------------------------------------------------------ */
/* Band bitmap (occupancy.hpp:105-121, 150-278) and BandSkip                  */
/* (empty_space_skip.hpp:19-153, 196-287)                                      */
/* ------------------------------------------------------------------------ */
#define KFO_BAND_EPSILON (1.0f / 64.0f) /* kBandEpsilon, occupancy.hpp:148 */
#define KFO_INF 1.0e30f                 /* BlockMarch::kInfinity */

typedef struct {
  const uint32_t* words;
  uint64_t bx, by, bz;
} band_view;

static inline void band_extent(const kfo_volume* v, uint64_t* bx, uint64_t* by, uint64_t* bz) {
  /* BlockGrid::for_resolution (grid.hpp:27-33) */
  *bx = (v->geometry.res_x + 7u) / 8u;
  *by = (v->geometry.res_y + 7u) / 8u;
  *bz = (v->geometry.res_z + 7u) / 8u;
}

/* BandView::block_index (occupancy.hpp:179-182): z-major, 32 z-blocks per word. */
static inline uint64_t band_index(uint64_t by, uint64_t bz, uint64_t x, uint64_t y, uint64_t z) {
  return ((x * by) + y) * bz + z;
}

static inline int band_test(const band_view* b, uint64_t x, uint64_t y, uint64_t z) {
  const uint64_t i = band_index(b->by, b->bz, x, y, z);
  return (int)((b->words[i / 32u] >> (i % 32u)) & 1u);
}

uint64_t kfo_band_word_count(const kfo_volume* v) {
  uint64_t bx, by, bz;
  band_extent(v, &bx, &by, &bz);
  return (bx * by * bz + 31u) / 32u;
}

void kfo_band_bitmap(const kfo_volume* v, uint32_t* raw, uint32_t* dilated) {
  /* BlockBitmapOps::rebuild (occupancy.hpp:105-121) with BandFilter
   * (occupancy.hpp:150-153, 166-171): a block is in the band when any voxel
   * is observed with tsdf < 1 - kBandEpsilon; the view is the 3^3 dilation
   * (neighborhood_occupied, occupancy.hpp:69-94). */
  uint64_t bx, by, bz;
  band_extent(v, &bx, &by, &bz);
  const uint64_t words = (bx * by * bz + 31u) / 32u;
  memset(raw, 0, words * sizeof(uint32_t));
  memset(dilated, 0, words * sizeof(uint32_t));
  const kf_volume_geometry* g = &v->geometry;
  for (uint32_t z = 0; z < g->res_z; ++z) {
    for (uint32_t y = 0; y < g->res_y; ++y) {
      for (uint32_t x = 0; x < g->res_x; ++x) {
        const int64_t i = storage_index(v, x, y, z);
        if (i < 0) continue;
        const decoded_voxel d = decode_voxel(v->voxel, v->voxels, (size_t)i);
        if (d.observed && d.tsdf < (1.0f - KFO_BAND_EPSILON)) {
          const uint64_t b = band_index(by, bz, x / 8u, y / 8u, z / 8u);
          raw[b / 32u] |= 1u << (b % 32u);
        }
      }
    }
  }
  const band_view rv = {raw, bx, by, bz};
  for (uint64_t x = 0; x < bx; ++x) {
    for (uint64_t y = 0; y < by; ++y) {
      for (uint64_t z = 0; z < bz; ++z) {
        int hit = 0;
        for (int oz = -1; oz <= 1 && !hit; ++oz) {
          for (int oy = -1; oy <= 1 && !hit; ++oy) {
            for (int ox = -1; ox <= 1 && !hit; ++ox) {
              const int64_t nx = (int64_t)x + ox, ny = (int64_t)y + oy, nz = (int64_t)z + oz;
              if (nx < 0 || ny < 0 || nz < 0 || (uint64_t)nx >= bx || (uint64_t)ny >= by || (uint64_t)nz >= bz) {
                continue;
              }
              hit = band_test(&rv, (uint64_t)nx, (uint64_t)ny, (uint64_t)nz);
            }
          }
        }
        if (hit) {
          const uint64_t b = band_index(by, bz, x, y, z);
          dilated[b / 32u] |= 1u << (b % 32u);
        }
      }
    }
  }
}

/* compat::min / compat::max (cuda_compat.hpp:75-86) */
static inline float cmin(float lhs, float rhs) { return rhs < lhs ? rhs : lhs; }
static inline float cmax(float lhs, float rhs) { return lhs < rhs ? rhs : lhs; }

/* BlockMarch (empty_space_skip.hpp:19-153): one ray in one volume. */
typedef struct {
  const kf_volume_geometry* g;
  float block_size;
  v3 origin, dir;
} block_march;

static inline float axis_exit(float origin, float direction, float low, float high) {
  return ((direction >= 0.0f ? high : low) - origin) / direction;
}

static float bm_block_exit(const block_march* m, uint64_t bx, uint64_t by, uint64_t bz) {
  const float lx = m->g->origin[0] + ((float)bx * m->block_size);
  const float ly = m->g->origin[1] + ((float)by * m->block_size);
  const float lz = m->g->origin[2] + ((float)bz * m->block_size);
  const float hx = lx + (1.0f * m->block_size), hy = ly + (1.0f * m->block_size), hz = lz + (1.0f * m->block_size);
  return cmin(axis_exit(m->origin.x, m->dir.x, lx, hx),
              cmin(axis_exit(m->origin.y, m->dir.y, ly, hy), axis_exit(m->origin.z, m->dir.z, lz, hz)));
}

static float bm_column_exit(const block_march* m, uint64_t bx, uint64_t by) {
  const float lx = m->g->origin[0] + ((float)bx * m->block_size);
  const float ly = m->g->origin[1] + ((float)by * m->block_size);
  float exit = KFO_INF;
  if (m->dir.x != 0.0f) exit = cmin(exit, axis_exit(m->origin.x, m->dir.x, lx, lx + m->block_size));
  if (m->dir.y != 0.0f) exit = cmin(exit, axis_exit(m->origin.y, m->dir.y, ly, ly + m->block_size));
  return exit;
}

static float bm_z_entry(const block_march* m, uint64_t bz) {
  const float side = m->dir.z >= 0.0f ? 0.0f : 1.0f;
  const float plane = m->g->origin[2] + (((float)bz + side) * m->block_size);
  return (plane - m->origin.z) / m->dir.z;
}

static void bm_slab(float origin, float direction, float low, float high, float* entry, float* exit) {
  if (direction == 0.0f) {
    if (origin < low || origin > high) *entry = KFO_INF;
    return;
  }
  const float t_low = (low - origin) / direction;
  const float t_high = (high - origin) / direction;
  *entry = cmax(*entry, cmin(t_low, t_high));
  *exit = cmin(*exit, cmax(t_low, t_high));
}

static float bm_volume_entry(const block_march* m) {
  const kf_volume_geometry* g = m->g;
  float entry = 0.0f, exit = KFO_INF;
  bm_slab(m->origin.x, m->dir.x, g->origin[0], g->origin[0] + ((float)g->res_x * g->voxel_size), &entry, &exit);
  bm_slab(m->origin.y, m->dir.y, g->origin[1], g->origin[1] + ((float)g->res_y * g->voxel_size), &entry, &exit);
  bm_slab(m->origin.z, m->dir.z, g->origin[2], g->origin[2] + ((float)g->res_z * g->voxel_size), &entry, &exit);
  return entry <= exit ? entry : KFO_INF;
}

/* find_set_at_or_after / find_set_at_or_before (empty_space_skip.hpp:196-217) */
static inline int set_at_or_after(uint32_t word, unsigned offset) {
  const uint32_t masked = word & ~((1u << offset) - 1u);
  return masked == 0u ? -1 : __builtin_ctz(masked);
}
static inline int set_at_or_before(uint32_t word, unsigned offset) {
  const uint32_t masked = word & (offset >= 31u ? ~0u : ((1u << (offset + 1u)) - 1u));
  return masked == 0u ? -1 : 31 - __builtin_clz(masked);
}

/* BandSkip::word_scan_z (empty_space_skip.hpp:266-284) */
static float band_word_scan_z(const band_view* b, const block_march* m, uint64_t x, uint64_t y, uint64_t z) {
  const uint64_t index = band_index(b->by, b->bz, x, y, z);
  const uint32_t word = b->words[index / 32u];
  const unsigned offset = (unsigned)(index % 32u);
  const int forward = m->dir.z >= 0.0f;
  const int found = forward ? set_at_or_after(word, offset) : set_at_or_before(word, offset);
  uint64_t target_z;
  if (found >= 0) {
    target_z = z + (uint64_t)found - offset;
  } else {
    target_z = forward ? z + (32u - offset) : z - (offset < z ? offset : z);
  }
  return cmin(bm_z_entry(m, target_z), bm_column_exit(m, x, y));
}

/* BandSkip::advance (empty_space_skip.hpp:225-262) */
static float band_advance(const band_view* b, const kf_volume_geometry* g, v3 origin, v3 dir, float ray_length,
                          float base_step, float max_depth) {
  const block_march m = {g, 8.0f * g->voxel_size, origin, dir};
  const float nudge = 0.25f * g->voxel_size;
  const int z_major = fabsf(dir.z) >= fabsf(dir.x) && fabsf(dir.z) >= fabsf(dir.y) && (b->bz % 32u) == 0u;
  while (ray_length <= max_depth) {
    const v3 point = v3add(origin, v3mul(dir, ray_length));
    const v3 grid = v3m((point.x - g->origin[0]) / g->voxel_size, (point.y - g->origin[1]) / g->voxel_size,
                        (point.z - g->origin[2]) / g->voxel_size);
    if (!grid_contains(g, grid)) {
      const float entry = bm_volume_entry(&m);
      if (entry >= KFO_INF || entry > max_depth) {
        return max_depth + base_step;
      }
      ray_length = cmax(ray_length + base_step, entry + nudge);
      continue;
    }
    const uint64_t x = (uint64_t)grid.x / 8u, y = (uint64_t)grid.y / 8u, z = (uint64_t)grid.z / 8u;
    if (band_test(b, x, y, z)) {
      return ray_length;
    }
    float target = KFO_INF;
    if (z_major) target = band_word_scan_z(b, &m, x, y, z);
    if (target >= KFO_INF) target = bm_block_exit(&m, x, y, z);
    ray_length = cmax(ray_length + base_step, target + nudge);
  }
  return ray_length;
}

/* ------------------------------------------------------------------------ */
/* Raycasting (raycasting.hpp:116-245)                                       */
/* ------------------------------------------------------------------------ */
/* `band` selects BandSkip (the band-march backend); NULL is the plain march
 * (NoSkip), whose output the bitmap-march backend reproduces bit for bit. */
static void render_pixel(const sampler* s, const band_view* band, const kf_raycast_camera* cam,
                         const kf_raycast_options* o, uint32_t col, uint32_t row, float* points,
                         float* normals, uint32_t* colors) {
  const size_t pix = (size_t)row * cam->width + col;
  const kf_rigid* pose = &cam->camera_to_world;
  const v3 translation = v3load(pose->t);
  float seed = o->min_depth;
  if (o->seed_from_previous) {
    const v3 previous = v3load(points + pix * 3);
    if (v3finite(previous) && v3dot(previous, previous) > 0.0f) {
      const float previous_depth = v3norm(v3sub(previous, translation));
      const float truncated = previous_depth - 2.0f * s->v->geometry.truncation_distance;
      seed = o->min_depth < truncated ? truncated : o->min_depth;
    }
  }
  v3store(points + pix * 3, v3nan());
  v3store(normals + pix * 3, v3nan());
  colors[pix] = 0;

  const v3 translated = back_project(cam->intrinsics, (float)col, (float)row, 1.0f);
  const v3 direction = rot_apply(pose, translated);
  const float dn = v3norm(direction);
  if (dn <= 0.0f) {
    return;
  }
  const v3 dir = v3div(direction, dn);

  /* find_zero_crossing (raycasting.hpp:165-211) */
  const float trunc = s->v->geometry.truncation_distance;
  const float base_step = s->v->geometry.voxel_size * o->step_scale;
  int have_prev = 0;
  float prev_tsdf = 0.0f;
  v3 prev_point = v3m(0, 0, 0);
  float ray_length = seed;
  int found = 0;
  v3 surface = v3m(0, 0, 0);
  while (ray_length <= o->max_depth) {
    if (band != NULL) {
      const float advanced =
          band_advance(band, &s->v->geometry, translation, dir, ray_length, base_step, o->max_depth);
      if (advanced != ray_length) {
        have_prev = 0; /* the skipped samples were all nullopt */
        ray_length = advanced;
        if (ray_length > o->max_depth) {
          break;
        }
      }
    }
    const v3 point = v3add(translation, v3mul(dir, ray_length));
    float tsdf;
    if (!sample_tsdf(s, point, o->corner_policy, &tsdf)) {
      have_prev = 0;
      ray_length += base_step;
      continue;
    }
    if (have_prev && prev_tsdf > 0.0f && tsdf <= 0.0f) {
      const float gap = prev_tsdf - tsdf;
      const float alpha = gap != 0.0f ? prev_tsdf / gap : 0.0f;
      surface = v3add(prev_point, v3mul(v3sub(point, prev_point), alpha));
      found = 1;
      break;
    }
    if (have_prev && prev_tsdf < 0.0f && tsdf > 0.0f) {
      break;
    }
    have_prev = 1;
    prev_tsdf = tsdf;
    prev_point = point;
    const float precomp = tsdf * trunc * o->step_scale;
    const float step = base_step < precomp ? precomp : base_step;
    ray_length += tsdf > 0.0f ? step : base_step;
  }
  if (!found) {
    return;
  }
  /* write_surface_sample (raycasting.hpp:215-245) */
  v3 normal;
  int has_normal = o->cell_gradient_normals ? cell_normal(s, surface, &normal)
                                            : central_normal(s, surface, o->corner_policy, &normal);
  if (!has_normal) {
    return;
  }
  v3store(points + pix * 3, surface);
  v3store(normals + pix * 3, normal);
  if (s->v->colors != NULL) {
    v3 c;
    if (sample_color(s, surface, &c)) {
      colors[pix] = pixel_from_color(c);
    }
  } else {
    const v3 view = v3normalized(v3sub(translation, surface));
    const float d = v3dot(normal, view);
    const float intensity = 255.0f * (0.0f < d ? d : 0.0f);
    colors[pix] = pixel_from_color(v3m(intensity, intensity, intensity));
  }
}

void kfo_raycast(const kfo_volume* v, const kf_raycast_camera* cam, const kf_raycast_options* o,
                 float* points, float* normals, uint32_t* colors, int32_t threads) {
  /* Raycaster::render (raycasting.hpp:277-301) */
  const sampler s = {v, 1.0f / v->geometry.voxel_size};
  (void)threads;
#ifdef _OPENMP
  const int nt = threads > 0 ? threads : 1;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
#endif
  for (int64_t row = 0; row < (int64_t)cam->height; ++row) {
    for (uint32_t col = 0; col < cam->width; ++col) {
      render_pixel(&s, NULL, cam, o, col, (uint32_t)row, points, normals, colors);
    }
  }
}

void kfo_raycast_band(const kfo_volume* v, const uint32_t* band_words, const kf_raycast_camera* cam,
                      const kf_raycast_options* o, float* points, float* normals, uint32_t* colors,
                      int32_t threads) {
  /* Raycaster::render with EmptySpaceIndex::visit -> BandSkip
   * (raycasting.hpp:22-60, 165-211) over the dilated band bitmap. */
  const sampler s = {v, 1.0f / v->geometry.voxel_size};
  band_view b;
  b.words = band_words;
  band_extent(v, &b.bx, &b.by, &b.bz);
  (void)threads;
#ifdef _OPENMP
  const int nt = threads > 0 ? threads : 1;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
#endif
  for (int64_t row = 0; row < (int64_t)cam->height; ++row) {
    for (uint32_t col = 0; col < cam->width; ++col) {
      render_pixel(&s, &b, cam, o, col, (uint32_t)row, points, normals, colors);
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Projective ICP (icp_correspondence.hpp:38-301, icp_optimizer.cpp)         */
/* ------------------------------------------------------------------------ */
typedef struct {
  float j[6];
  float residual;
  float distance;
} correspondence;

/* CorrespondenceSearch::match (icp_correspondence.hpp:244-294). */
static int icp_match(const float* lv, const float* ln, const float* mp, const float* mn,
                     uint32_t mw, uint32_t mh, kf_intrinsics k, const kf_rigid* camera,
                     const kf_rigid* model, float max_d, float min_dot, correspondence* out) {
  const v3 live_vertex = v3load(lv);
  const v3 live_normal = v3load(ln);
  if (!v3finite(live_vertex) || !v3finite(live_normal)) return 0;
  const v3 source = rigid_apply(camera, live_vertex);
  const v3 sim = rigid_apply(model, source);
  if (!v3finite(sim) || sim.z <= 0.0f) return 0;
  float px, py;
  project(k, sim, &px, &py);
  const long mx = lroundf(px), my = lroundf(py);
  if (mx < 0 || my < 0) return 0;
  if ((unsigned long)mx >= mw || (unsigned long)my >= mh) return 0;
  const size_t mi = (size_t)my * mw + (size_t)mx;
  const v3 model_vertex = v3load(mp + mi * 3);
  const v3 model_normal = v3load(mn + mi * 3);
  if (!v3finite(model_vertex) || !v3finite(model_normal)) return 0;
  const v3 source_normal = v3normalized(rot_apply(camera, live_normal));
  const float distance = v3norm(v3sub(source, model_vertex));
  if (distance > max_d) return 0;
  if (v3dot(source_normal, model_normal) < min_dot) return 0;
  /* IcpCorrespondence::from_match (icp_correspondence.hpp:44-52) */
  const v3 rot = v3cross(source, model_normal);
  out->j[0] = rot.x;
  out->j[1] = rot.y;
  out->j[2] = rot.z;
  out->j[3] = model_normal.x;
  out->j[4] = model_normal.y;
  out->j[5] = model_normal.z;
  out->residual = v3dot(model_normal, v3sub(model_vertex, source));
  out->distance = distance;
  return 1;
}

void kfo_icp_equations(const float* lv, const float* ln, uint32_t lw, uint32_t lh, const float* mp,
                       const float* mn, uint32_t mw, uint32_t mh, kf_intrinsics k,
                       const kf_rigid* camera, const kf_rigid* model, float max_d, float min_dot,
                       float* sums, uint64_t* count) {
  /* ProjectiveIcpTracker::find_correspondences (icp_optimizer.cpp:304-317)
   * with IcpNormalEquations::accumulate (icp_correspondence.hpp:111-129). */
  for (int i = 0; i < 29; ++i) sums[i] = 0.0f;
  uint64_t n = 0;
  for (uint32_t y = 0; y < lh; ++y) {
    for (uint32_t x = 0; x < lw; ++x) {
      correspondence c;
      const size_t p = (size_t)y * lw + x;
      if (!icp_match(lv + p * 3, ln + p * 3, mp, mn, mw, mh, k, camera, model, max_d, min_dot, &c)) {
        continue;
      }
      int e = 0;
      for (int r = 0; r < 6; ++r) {
        for (int col = r; col < 6; ++col) {
          sums[e] += c.j[r] * c.j[col];
          ++e;
        }
      }
      for (int r = 0; r < 6; ++r) sums[21 + r] += c.j[r] * c.residual;
      sums[27] += c.distance;
      sums[28] += c.residual * c.residual;
      ++n;
    }
  }
  *count = n;
}

void kfo_icp_equations_f64(const float* lv, const float* ln, uint32_t lw, uint32_t lh,
                           const float* mp, const float* mn, uint32_t mw, uint32_t mh,
                           kf_intrinsics k, const kf_rigid* camera, const kf_rigid* model,
                           float max_d, float min_dot, double* sums, uint64_t* count) {
  for (int i = 0; i < 29; ++i) sums[i] = 0.0;
  uint64_t n = 0;
  for (uint32_t y = 0; y < lh; ++y) {
    for (uint32_t x = 0; x < lw; ++x) {
      correspondence c;
      const size_t p = (size_t)y * lw + x;
      if (!icp_match(lv + p * 3, ln + p * 3, mp, mn, mw, mh, k, camera, model, max_d, min_dot, &c)) {
        continue;
      }
      int e = 0;
      for (int r = 0; r < 6; ++r) {
        for (int col = r; col < 6; ++col) {
          sums[e] += (double)c.j[r] * (double)c.j[col];
          ++e;
        }
      }
      for (int r = 0; r < 6; ++r) sums[21 + r] += (double)c.j[r] * (double)c.residual;
      sums[27] += (double)c.distance;
      sums[28] += (double)c.residual * (double)c.residual;
      ++n;
    }
  }
  *count = n;
}

/* Symmetric eigenvalues of a 6x6 matrix by cyclic Jacobi rotations (double). */
static int jacobi_eigenvalues6(const double in[6][6], double eig[6]) {
  double a[6][6];
  memcpy(a, in, sizeof(a));
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < 6; ++p)
      for (int q = p + 1; q < 6; ++q) off += a[p][q] * a[p][q];
    if (off < 1e-300) break;
    for (int p = 0; p < 6; ++p) {
      for (int q = p + 1; q < 6; ++q) {
        if (a[p][q] == 0.0) continue;
        const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0);
        const double sn = t * c;
        for (int k = 0; k < 6; ++k) {
          const double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - sn * akq;
          a[k][q] = sn * akp + c * akq;
        }
        for (int k = 0; k < 6; ++k) {
          const double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - sn * aqk;
          a[q][k] = sn * apk + c * aqk;
        }
      }
    }
  }
  for (int i = 0; i < 6; ++i) {
    eig[i] = a[i][i];
    if (!isfinite(eig[i])) return 0;
  }
  return 1;
}

typedef struct {
  int stable;
  float min_eigenvalue;
  float condition_number;
} stability;

/* ProjectiveIcpTracker::check_system_stability (icp_optimizer.cpp:319-347). */
static stability check_stability(const float* sums, uint64_t count, const kf_icp_options* o) {
  stability s = {0, 0.0f, 0.0f};
  if (count < o->min_correspondences) return s;
  double m[6][6];
  int e = 0;
  for (int r = 0; r < 6; ++r) {
    for (int c = r; c < 6; ++c) {
      m[r][c] = sums[e];
      m[c][r] = sums[e];
      ++e;
    }
  }
  double eig[6];
  if (!jacobi_eigenvalues6(m, eig)) return s;
  double lo = eig[0], hi = eig[0];
  for (int i = 1; i < 6; ++i) {
    lo = eig[i] < lo ? eig[i] : lo;
    hi = eig[i] > hi ? eig[i] : hi;
  }
  const float mn = (float)lo, mx = (float)hi;
  if (mn <= 0.0f || mx <= 0.0f) {
    s.min_eigenvalue = mn;
    return s;
  }
  s.condition_number = mx / mn;
  s.min_eigenvalue = mn;
  s.stable = mn >= o->min_system_eigenvalue && s.condition_number <= o->max_condition_number;
  return s;
}

/* LDL^T solve with symmetric diagonal pivoting, in float. */
static void ldlt_solve6(const float A[6][6], const float b[6], float x[6]) {
  float a[6][6];
  int perm[6];
  memcpy(a, A, sizeof(a));
  for (int i = 0; i < 6; ++i) perm[i] = i;
  float d[6];
  float L[6][6] = {{0}};
  for (int k = 0; k < 6; ++k) {
    int piv = k;
    float best = fabsf(a[k][k]);
    for (int i = k + 1; i < 6; ++i) {
      if (fabsf(a[i][i]) > best) {
        best = fabsf(a[i][i]);
        piv = i;
      }
    }
    if (piv != k) {
      for (int i = 0; i < 6; ++i) {
        const float t = a[k][i];
        a[k][i] = a[piv][i];
        a[piv][i] = t;
      }
      for (int i = 0; i < 6; ++i) {
        const float t = a[i][k];
        a[i][k] = a[i][piv];
        a[i][piv] = t;
      }
      for (int i = 0; i < k; ++i) {
        const float t = L[k][i];
        L[k][i] = L[piv][i];
        L[piv][i] = t;
      }
      const int t = perm[k];
      perm[k] = perm[piv];
      perm[piv] = t;
    }
    d[k] = a[k][k];
    L[k][k] = 1.0f;
    for (int i = k + 1; i < 6; ++i) {
      L[i][k] = d[k] != 0.0f ? a[i][k] / d[k] : 0.0f;
    }
    for (int i = k + 1; i < 6; ++i) {
      for (int j = k + 1; j < 6; ++j) {
        a[i][j] = a[i][j] - L[i][k] * d[k] * L[j][k];
      }
    }
  }
  float y[6];
  for (int i = 0; i < 6; ++i) {
    float s = b[perm[i]];
    for (int j = 0; j < i; ++j) s -= L[i][j] * y[j];
    y[i] = s;
  }
  /* Zero pivots (an exactly rank-deficient system, e.g. a single plane)
   * take a zero component, the minimum-norm convention of an LDL^T solve
   * with diagonal pivoting (Eigen's LDLT::solve behaves this way). */
  for (int i = 0; i < 6; ++i) y[i] = fabsf(d[i]) > FLT_MIN ? y[i] / d[i] : 0.0f;
  float z[6];
  for (int i = 5; i >= 0; --i) {
    float s = y[i];
    for (int j = i + 1; j < 6; ++j) s -= L[j][i] * z[j];
    z[i] = s;
  }
  for (int i = 0; i < 6; ++i) x[perm[i]] = z[i];
}

typedef struct {
  kf_rigid transform;
  float update_translation;
  float update_rotation;
  float lambda;
  int solved;
} increment;

/* ProjectiveIcpTracker::increment_from_solution (icp_optimizer.cpp:349-365):
 * Rodrigues R = c I + s [u]x + (1 - c) u u^T. */
static increment increment_from_solution(const float sol[6]) {
  increment inc;
  memset(&inc, 0, sizeof(inc));
  const v3 aa = v3m(sol[0], sol[1], sol[2]);
  const v3 tr = v3m(sol[3], sol[4], sol[5]);
  const float angle = v3norm(aa);
  float R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (angle > 1.0e-12f) {
    const v3 u = v3div(aa, angle);
    const float s = sinf(angle), c = cosf(angle), oc = 1.0f - c;
    R[0] = c + u.x * u.x * oc;
    R[1] = u.x * u.y * oc - u.z * s;
    R[2] = u.x * u.z * oc + u.y * s;
    R[3] = u.y * u.x * oc + u.z * s;
    R[4] = c + u.y * u.y * oc;
    R[5] = u.y * u.z * oc - u.x * s;
    R[6] = u.z * u.x * oc - u.y * s;
    R[7] = u.z * u.y * oc + u.x * s;
    R[8] = c + u.z * u.z * oc;
  }
  memcpy(inc.transform.r, R, sizeof(R));
  v3store(inc.transform.t, tr);
  inc.update_translation = v3norm(tr);
  inc.update_rotation = angle;
  inc.solved = 1;
  return inc;
}

static int within_caps(const increment* i, const kf_icp_options* o) {
  return i->update_translation <= o->max_update_translation &&
         i->update_rotation <= o->max_update_rotation;
}

static float damping_offset(const kf_icp_options* o, float diag, float scale) {
  if (o->damping_mode == KF_DAMPING_IDENTITY) return scale;
  if (o->damping_mode == KF_DAMPING_DIAGONAL) return scale * diag;
  return 0.0f;
}

static float grow(const kf_icp_options* o, float l) {
  const float v = l * o->lambda_increase;
  return v < o->max_lambda ? v : o->max_lambda;
}
static float shrink(const kf_icp_options* o, float l) {
  const float v = l * o->lambda_decrease;
  return o->min_lambda < v ? v : o->min_lambda;
}

/* ProjectiveIcpTracker::solve_increment (icp_optimizer.cpp:370-402). */
static increment solve_increment(const float* sums, uint64_t count, float lambda,
                                 const kf_icp_options* o) {
  increment last;
  memset(&last, 0, sizeof(last));
  if (count < o->min_correspondences) return last;
  float base[6][6], rhs[6];
  int e = 0;
  for (int r = 0; r < 6; ++r) {
    for (int c = r; c < 6; ++c) {
      base[r][c] = sums[e];
      base[c][r] = sums[e];
      ++e;
    }
  }
  for (int r = 0; r < 6; ++r) rhs[r] = sums[21 + r];
  const int active = o->damping_mode != KF_DAMPING_NONE;
  const unsigned attempts = active ? 8u : 1u;
  float scale = lambda;
  for (unsigned a = 0; a < attempts; ++a) {
    float damped[6][6];
    memcpy(damped, base, sizeof(damped));
    for (int r = 0; r < 6; ++r) {
      const int diag_index = (r * 6) - (r * (r + 1) / 2) + r;
      damped[r][r] += damping_offset(o, sums[diag_index], scale);
    }
    float sol[6];
    ldlt_solve6(damped, rhs, sol);
    int finite = 1;
    for (int i = 0; i < 6; ++i) finite &= isfinite(sol[i]) != 0;
    if (finite) {
      last = increment_from_solution(sol);
      last.lambda = scale;
      if (!active || within_caps(&last, o)) return last;
    }
    scale = grow(o, scale);
  }
  return last;
}

void kfo_icp_estimate(const float* lv, const float* ln, uint32_t lw, uint32_t lh, const float* mp,
                      const float* mn, uint32_t mw, uint32_t mh, kf_intrinsics k,
                      const kf_rigid* model_camera_to_world, const kf_rigid* initial,
                      uint32_t iterations, const kf_icp_options* o, kf_icp_outcome* out) {
  /* ProjectiveIcpTracker::estimate_with (icp_optimizer.cpp:208-302) */
  memset(out, 0, sizeof(*out));
  kf_rigid pose = *initial;
  kf_rigid model;
  kfo_rigid_inverse(model_camera_to_world, &model);
  const int active = o->damping_mode != KF_DAMPING_NONE;
  const int adaptive = active && o->adaptive_damping;
  float lambda = o->damping_lambda;
  float best_cost = 0.0f;
  kf_rigid best_pose = pose;
  float best_sums[29] = {0};
  uint64_t best_count = 0;
  int have_best = 0;
  out->status = KF_ICP_MAX_ITERATIONS;
  for (uint32_t it = 0; it < iterations; ++it) {
    float sums[29];
    uint64_t count;
    kfo_icp_equations(lv, ln, lw, lh, mp, mn, mw, mh, k, &pose, &model, o->max_point_distance,
                      o->min_normal_dot, sums, &count);
    out->iterations = (int32_t)(it + 1);
    out->correspondences = count;
    if (count > 0) out->mean_point_distance = sums[27] / (float)count;
    if (count < o->min_correspondences) {
      out->status = KF_ICP_TOO_FEW_CORRESPONDENCES;
      break;
    }
    out->mean_squared_residual = count == 0 ? 0.0f : sums[28] / (float)count;
    int accepted = 1;
    if (adaptive) {
      const float cost = sums[28] / (float)count;
      accepted = !have_best || cost <= best_cost;
      if (accepted) {
        have_best = 1;
        best_cost = cost;
        best_pose = pose;
        memcpy(best_sums, sums, sizeof(sums));
        best_count = count;
        lambda = shrink(o, lambda);
      } else {
        ++out->rejected_steps;
        pose = best_pose;
        memcpy(sums, best_sums, sizeof(sums));
        count = best_count;
        lambda = grow(o, lambda);
      }
    }
    const stability st = check_stability(sums, count, o);
    out->min_system_eigenvalue = st.min_eigenvalue;
    out->condition_number = st.condition_number;
    if (!st.stable && !active) {
      out->status = KF_ICP_UNCONSTRAINED_SYSTEM;
      break;
    }
    const increment inc = solve_increment(sums, count, lambda, o);
    if (!inc.solved) {
      out->status = KF_ICP_SOLVE_FAILED;
      break;
    }
    lambda = inc.lambda;
    out->damping_lambda = lambda;
    out->update_translation = inc.update_translation;
    out->update_rotation = inc.update_rotation;
    if (!within_caps(&inc, o)) {
      out->status = KF_ICP_UPDATE_TOO_LARGE;
      break;
    }
    kf_rigid next;
    kfo_rigid_compose(&inc.transform, &pose, &next);
    pose = next;
    if (accepted && inc.update_translation < o->min_update_translation &&
        inc.update_rotation < o->min_update_rotation) {
      out->status = KF_ICP_CONVERGED;
      break;
    }
  }
  out->pose = pose;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) out->pose_f64[i * 4 + j] = pose.r[i * 3 + j];
    out->pose_f64[i * 4 + 3] = pose.t[i];
  }
}

/* ------------------------------------------------------------------------ */
/* Marching cubes (MarchingCubes::extract / MeshBuilder,                    */
/* marching_cubes.cpp:311-485) with this project's triangulation table      */
/* (kf_mc_tables.h); every other step follows the reference.               */
/* ------------------------------------------------------------------------ */
#include "kf_mc_tables.h"

typedef struct {
  uint64_t* keys;
  uint32_t* values;
  uint64_t capacity; /* power of two */
  uint64_t count;
} weld_map;

static uint64_t weld_hash(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  return k;
}

static void weld_grow(weld_map* m) {
  const uint64_t old_cap = m->capacity;
  uint64_t* old_keys = m->keys;
  uint32_t* old_values = m->values;
  m->capacity = old_cap ? old_cap * 2 : 1024;
  m->keys = (uint64_t*)malloc(m->capacity * sizeof(uint64_t));
  m->values = (uint32_t*)malloc(m->capacity * sizeof(uint32_t));
  for (uint64_t i = 0; i < m->capacity; ++i) m->keys[i] = UINT64_MAX;
  for (uint64_t i = 0; i < old_cap; ++i) {
    if (old_keys[i] == UINT64_MAX) continue;
    uint64_t h = weld_hash(old_keys[i]) & (m->capacity - 1);
    while (m->keys[h] != UINT64_MAX) h = (h + 1) & (m->capacity - 1);
    m->keys[h] = old_keys[i];
    m->values[h] = old_values[i];
  }
  free(old_keys);
  free(old_values);
}

/* Returns the slot for `key`; *found tells whether it already held a vertex. */
static uint64_t weld_slot(weld_map* m, uint64_t key, int* found) {
  if ((m->count + 1) * 2 > m->capacity) weld_grow(m);
  uint64_t h = weld_hash(key) & (m->capacity - 1);
  while (m->keys[h] != UINT64_MAX) {
    if (m->keys[h] == key) {
      *found = 1;
      return h;
    }
    h = (h + 1) & (m->capacity - 1);
  }
  *found = 0;
  m->keys[h] = key;
  ++m->count;
  return h;
}

typedef struct {
  const kfo_volume* v;
  sampler s;
  float min_weight;
  weld_map weld;
  float *pos, *nrm, *col;
  uint64_t nv, cap_v;
  uint32_t* tri;
  uint64_t nt, cap_t;
} mesh_builder;

/* MeshBuilder::vertex_on_edge (marching_cubes.cpp:403-437) */
static uint32_t vertex_on_edge(mesh_builder* b, uint64_t x, uint64_t y, uint64_t z, const float values[8], int edge) {
  const kf_volume_geometry* g = &b->v->geometry;
  const int near = kMcEdge[edge][0], far = kMcEdge[edge][1], axis = kMcEdge[edge][2];
  const uint64_t nx = x + kMcCorner[near][0], ny = y + kMcCorner[near][1], nz = z + kMcCorner[near][2];
  const uint64_t key = ((nz * g->res_y + ny) * g->res_x + nx) * 3u + (uint64_t)axis;
  int found;
  const uint64_t slot = weld_slot(&b->weld, key, &found);
  if (found) return b->weld.values[slot];
  const uint32_t index = (uint32_t)b->nv;
  b->weld.values[slot] = index;
  const float near_value = values[near], far_value = values[far];
  const v3 near_point = cell_center(g, nx, ny, nz);
  const v3 far_point = cell_center(g, x + kMcCorner[far][0], y + kMcCorner[far][1], z + kMcCorner[far][2]);
  const float fraction = -near_value / (far_value - near_value);
  const v3 position = v3add(near_point, v3mul(v3sub(far_point, near_point), fraction));
  v3 normal = v3m(0.0f, 0.0f, 0.0f);
  if (!central_normal(&b->s, position, KF_CORNERS_SKIP_MISSING, &normal)) normal = v3m(0.0f, 0.0f, 0.0f);
  v3 color;
  if (!sample_color(&b->s, position, &color)) color = v3m(255.0f, 255.0f, 255.0f);
  if (b->nv == b->cap_v) {
    b->cap_v = b->cap_v ? b->cap_v * 2 : 1024;
    b->pos = (float*)realloc(b->pos, b->cap_v * 3 * sizeof(float));
    b->nrm = (float*)realloc(b->nrm, b->cap_v * 3 * sizeof(float));
    b->col = (float*)realloc(b->col, b->cap_v * 3 * sizeof(float));
  }
  v3store(b->pos + b->nv * 3, position);
  v3store(b->nrm + b->nv * 3, normal);
  v3store(b->col + b->nv * 3, color);
  ++b->nv;
  return index;
}

/* MeshBuilder::add_cell (marching_cubes.cpp:369-400); a corner that is
 * missing, unobserved, non-finite or lighter than min_weight skips the cell */
static void add_cell(mesh_builder* b, uint64_t x, uint64_t y, uint64_t z) {
  float values[8];
  unsigned cube = 0;
  for (int c = 0; c < 8; ++c) {
    const int64_t i = storage_index(b->v, x + kMcCorner[c][0], y + kMcCorner[c][1], z + kMcCorner[c][2]);
    if (i < 0) return;
    const decoded_voxel d = decode_voxel(b->v->voxel, b->v->voxels, (size_t)i);
    if (!d.observed || !d.finite || d.weight < b->min_weight) return;
    values[c] = d.tsdf;
    if (values[c] < 0.0f) cube |= 1u << c;
  }
  if (kMcEdgeMask[cube] == 0) return;
  for (int k = 0; kMcTriangles[cube][k] >= 0; k += 3) {
    const uint32_t a = vertex_on_edge(b, x, y, z, values, kMcTriangles[cube][k]);
    const uint32_t bb = vertex_on_edge(b, x, y, z, values, kMcTriangles[cube][k + 1]);
    const uint32_t c = vertex_on_edge(b, x, y, z, values, kMcTriangles[cube][k + 2]);
    if (b->nt == b->cap_t) {
      b->cap_t = b->cap_t ? b->cap_t * 2 : 1024;
      b->tri = (uint32_t*)realloc(b->tri, b->cap_t * 3 * sizeof(uint32_t));
    }
    b->tri[b->nt * 3] = a;
    b->tri[b->nt * 3 + 1] = bb;
    b->tri[b->nt * 3 + 2] = c;
    ++b->nt;
  }
}

/* MeshBuilder::fill_missing_normals (marching_cubes.cpp:441-456): a vertex
 * without a gradient normal takes the normalised sum of its face normals. */
static void fill_missing_normals(mesh_builder* b) {
  uint8_t* missing = (uint8_t*)calloc(b->nv ? b->nv : 1, 1);
  float* acc = (float*)calloc((b->nv ? b->nv : 1) * 3, sizeof(float));
  for (uint64_t i = 0; i < b->nv; ++i) {
    missing[i] = b->nrm[i * 3] == 0.0f && b->nrm[i * 3 + 1] == 0.0f && b->nrm[i * 3 + 2] == 0.0f;
  }
  for (uint64_t t = 0; t < b->nt; ++t) {
    const uint32_t* tr = b->tri + t * 3;
    const v3 p0 = v3load(b->pos + (size_t)tr[0] * 3), p1 = v3load(b->pos + (size_t)tr[1] * 3),
             p2 = v3load(b->pos + (size_t)tr[2] * 3);
    const v3 face = v3cross(v3sub(p1, p0), v3sub(p2, p0));
    for (int k = 0; k < 3; ++k) {
      if (!missing[tr[k]]) continue;
      v3store(acc + (size_t)tr[k] * 3, v3add(v3load(acc + (size_t)tr[k] * 3), face));
    }
  }
  for (uint64_t i = 0; i < b->nv; ++i) {
    if (missing[i]) v3store(b->nrm + i * 3, v3normalized(v3load(acc + i * 3)));
  }
  free(missing);
  free(acc);
}

kf_status kfo_marching_cubes(const kfo_volume* volume, float min_weight, kf_mesh* out) {
  memset(out, 0, sizeof(*out));
  const kf_volume_geometry* g = &volume->geometry;
  if (g->res_x < 2 || g->res_y < 2 || g->res_z < 2) return KF_OK;
  mesh_builder b;
  memset(&b, 0, sizeof(b));
  b.v = volume;
  b.s.v = volume;
  b.s.inv_voxel = 1.0f / g->voxel_size;
  b.min_weight = min_weight;
  const uint64_t cx = g->res_x - 1, cy = g->res_y - 1, cz = g->res_z - 1;
  if (!is_sparse(volume)) {
    for (uint64_t z = 0; z < cz; ++z)
      for (uint64_t y = 0; y < cy; ++y)
        for (uint64_t x = 0; x < cx; ++x) add_cell(&b, x, y, z);
  } else {
    /* only allocated blocks can hold the zero crossing (marching_cubes.cpp:475-485) */
    const uint64_t bx = blocks_along(g->res_x), by = blocks_along(g->res_y), bz = blocks_along(g->res_z);
    for (uint64_t block = 0; block < bx * by * bz; ++block) {
      if (volume->grid[block] == 0xFFFFFFFFu) continue;
      const uint64_t x0 = (block % bx) * 8, y0 = ((block / bx) % by) * 8, z0 = (block / (bx * by)) * 8;
      for (uint64_t z = z0; z < z0 + 8 && z < cz; ++z)
        for (uint64_t y = y0; y < y0 + 8 && y < cy; ++y)
          for (uint64_t x = x0; x < x0 + 8 && x < cx; ++x) add_cell(&b, x, y, z);
    }
  }
  fill_missing_normals(&b);
  free(b.weld.keys);
  free(b.weld.values);
  out->positions = b.pos;
  out->normals = b.nrm;
  out->colors = b.col;
  out->triangles = b.tri;
  out->vertex_count = b.nv;
  out->triangle_count = b.nt;
  return KF_OK;
}

/* ------------------------------------------------------------------------ */
/* FP64 integration: IntegrationContext::observe + BasicVoxel::fused        */
/* (tsdf_integration.hpp:183-263, volume.hpp:137-146) in double, into a      */
/* (tsdf, weight) double pair per voxel, x fastest.  The reference point     */
/* for the FP32/int16/bf16 volumes' error statements.                        */
/* ------------------------------------------------------------------------ */
void kfo_integrate_f64(double* voxels, const kf_volume_geometry* g, const kf_frame_view* f,
                       const kf_integration_options* o, int32_t rule, int32_t threads) {
  const double R[9] = {f->world_to_camera.r[0], f->world_to_camera.r[1], f->world_to_camera.r[2],
                       f->world_to_camera.r[3], f->world_to_camera.r[4], f->world_to_camera.r[5],
                       f->world_to_camera.r[6], f->world_to_camera.r[7], f->world_to_camera.r[8]};
  const double T[3] = {f->world_to_camera.t[0], f->world_to_camera.t[1], f->world_to_camera.t[2]};
  const double fx = f->intrinsics.fx, fy = f->intrinsics.fy, cx = f->intrinsics.cx, cy = f->intrinsics.cy;
  (void)threads;
#ifdef _OPENMP
  const int nt = threads > 0 ? threads : 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
#endif
  for (int64_t z = 0; z < (int64_t)g->res_z; ++z) {
    for (uint64_t y = 0; y < g->res_y; ++y) {
      for (uint64_t x = 0; x < g->res_x; ++x) {
        const double c[3] = {g->origin[0] + ((double)x + 0.5) * g->voxel_size,
                             g->origin[1] + ((double)y + 0.5) * g->voxel_size,
                             g->origin[2] + ((double)z + 0.5) * g->voxel_size};
        double cp[3];
        for (int i = 0; i < 3; ++i) cp[i] = R[i * 3] * c[0] + R[i * 3 + 1] * c[1] + R[i * 3 + 2] * c[2] + T[i];
        if (cp[2] <= 0.0) continue;
        const long rx = lround(fx * cp[0] / cp[2] + cx), ry = lround(fy * cp[1] / cp[2] + cy);
        if (rx < 0 || ry < 0 || (unsigned long)rx >= f->width || (unsigned long)ry >= f->height) continue;
        const size_t pix = (size_t)ry * f->width + (size_t)rx;
        const uint16_t raw = f->depth[pix];
        if (raw == 0) continue;
        const double measured = (double)raw / o->depth_scale;
        if (measured < o->min_depth || measured > o->max_depth) continue;
        const double ray[3] = {((double)rx - cx) / fx, ((double)ry - cy) / fy, 1.0};
        const double lambda = sqrt(ray[0] * ray[0] + ray[1] * ray[1] + 1.0);
        const double trunc = o->distance_scaled_truncation
                                 ? (double)g->truncation_distance + o->truncation_distance_scale * measured
                                 : (double)g->truncation_distance;
        const double dist = sqrt(cp[0] * cp[0] + cp[1] * cp[1] + cp[2] * cp[2]);
        const double sdf = o->projective_distance ? measured - dist / lambda : measured - cp[2];
        if (sdf < -trunc) continue;
        const double tsdf = sdf / trunc > 1.0 ? 1.0 : (sdf / trunc < -1.0 ? -1.0 : sdf / trunc);
        double weight = o->observation_weight;
        if (rule == KF_RULE_ANGLE_WEIGHTED && f->normals != NULL) {
          const float* n = f->normals + pix * 3;
          if (isfinite(n[0]) && isfinite(n[1]) && isfinite(n[2])) {
            const double nn = sqrt((double)n[0] * n[0] + (double)n[1] * n[1] + (double)n[2] * n[2]);
            const double d = -((double)n[0] * ray[0] + (double)n[1] * ray[1] + (double)n[2] * ray[2]) / (nn * lambda);
            weight *= (d > 0.0 ? d : 0.0) / measured;
          }
        }
        if (weight <= 0.0) continue;
        double* vx = voxels + ((z * g->res_y + y) * g->res_x + x) * 2;
        const double w0 = vx[1];
        vx[0] = (vx[0] * w0 + tsdf * weight) / (w0 + weight);
        vx[1] = o->max_weight < w0 + weight ? o->max_weight : w0 + weight;
      }
    }
  }
}
