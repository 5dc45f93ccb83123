// kf_icp.cu - projective point-to-plane ICP on the device.
//
// One cooperative launch per pyramid level (icp_level_kernel; the three
// levels of a frame are nodes of its CUDA graph).  Each Gauss-Newton step:
//  1. every CTA associates its live pixels with the model render
//     (CorrespondenceSearch::match, icp_correspondence.hpp:244-294) and
//     accumulates the 29 float sums of IcpNormalEquations::accumulate
//     (icp_correspondence.hpp:111-129) per thread;
//  2. reduces them per warp with register shuffles and per CTA through
//     shared memory in a fixed order, writing one partial slot per CTA;
//  3. meets the other CTAs at a bounded grid barrier, combines every slot in
//     CTA order with Kahan-compensated FP32 sums, and runs the Gauss-Newton/
//     LM step of ProjectiveIcpTracker::estimate_with (icp_optimizer.cpp:
//     208-302) in FP64 on its own copy of the tracker state: stability veto,
//     damped LDL^T solve, Rodrigues increment, pose composition and the
//     convergence test.  The loop leaves at the first step whose status is
//     not running (the reference's device loop stops the same way,
//     icp_correspondence.cu:68-78).
// icp_iteration_kernel is one sweep of the same association, slots and
// combine (kf_icp_normal_equations).  The reference reduces with FP32 atomics
// (non-deterministic, icp_correspondence.cu:131-145); this reduction is
// deterministic.
#include <atomic>
#include <cmath>
#include <cstddef>

#include "kf_internal.h"

namespace kf {
namespace {

__device__ __forceinline__ Rigid rigid_load(const float* c) {
  return Rigid{{c[0], c[1], c[2]}, {c[3], c[4], c[5]}, {c[6], c[7], c[8]}, {c[9], c[10], c[11]}};
}

// The model half of CorrespondenceSearch::match and
// IcpCorrespondence::from_match (icp_correspondence.hpp:270-294, 52-74):
// `source` is the live vertex in world coordinates, (mv, mn) the model
// point and normal the live pixel projects to.
__device__ __forceinline__ bool finish_match(f3 source, f3 ln, f3 mv, f3 mn, const Rigid& cam, float max_d,
                                             float min_dot, float* j, float& residual, float& distance) {
  if (!finite3(mv) || !finite3(mn)) return false;
  const f3 sn = normalized(rotate(cam, ln));
  distance = norm(source - mv);
  if (distance > max_d) return false;
  if (dot(sn, mn) < min_dot) return false;
  const f3 rot = cross(source, mn);
  j[0] = rot.x;
  j[1] = rot.y;
  j[2] = rot.z;
  j[3] = mn.x;
  j[4] = mn.y;
  j[5] = mn.z;
  residual = dot(mn, mv - source);
  return true;
}

// CorrespondenceSearch::match + IcpCorrespondence::from_match.
__device__ __forceinline__ bool match(const IcpLevelArgs& a, const Rigid& cam, const Rigid& model,
                                      float max_d, float min_dot, uint32_t x, uint32_t y, float* j,
                                      float& residual, float& distance) {
  const size_t p = static_cast<size_t>(y) * a.live_width + x;
  const f3 lv = ldg3(a.live_vertices + p * 3);
  const f3 ln = ldg3(a.live_normals + p * 3);
  if (!finite3(lv) || !finite3(ln)) return false;
  const f3 source = apply(cam, lv);
  const f3 sim = apply(model, source);
  if (!finite3(sim) || sim.z <= 0.0f) return false;
  float px, py;
  project(a.model_intrinsics, sim, px, py);
  const long mx = lroundf(px), my = lroundf(py);
  if (mx < 0 || my < 0 || mx >= static_cast<long>(a.model_width) || my >= static_cast<long>(a.model_height)) {
    return false;
  }
  const size_t mi = static_cast<size_t>(my) * a.model_width + static_cast<size_t>(mx);
  return finish_match(source, ln, ldg3(a.model_points + mi * 3), ldg3(a.model_normals + mi * 3), cam, max_d,
                      min_dot, j, residual, distance);
}

// ---- FP64 6x6 linear algebra ------------------------------------------------
// Every loop has constant bounds and is unrolled, so the matrices live in
// registers (the solve runs on one thread of the last CTA).
// Cholesky A = L L^T; false on a non-positive pivot.  rinv[c] = 1 / L[c][c].
__device__ __forceinline__ bool cholesky6(const double (&a)[6][6], double (&l)[6][6], double (&rinv)[6]) {
  bool ok = true;
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    double d = a[c][c];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      if (k < c) d -= l[c][k] * l[c][k];
    }
    ok = ok && (d > 0.0);
    const double lc = sqrt(fmax(d, 1e-300));
    l[c][c] = lc;
    rinv[c] = 1.0 / lc;
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      if (r <= c) {
        if (r < c) l[r][c] = 0.0;
        continue;
      }
      double s = a[r][c];
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        if (k < c) s -= l[r][k] * l[c][k];
      }
      l[r][c] = s * rinv[c];
    }
  }
  return ok;
}

// L^-1 of a lower triangular factor (no divisions: rinv holds 1 / L[c][c]).
__device__ __forceinline__ void lower_inverse6(const double (&l)[6][6], const double (&rinv)[6], double (&inv)[6][6]) {
#pragma unroll
  for (int c = 0; c < 6; ++c) {
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      if (r < c) {
        inv[r][c] = 0.0;
        continue;
      }
      double s = (r == c) ? 1.0 : 0.0;
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        if (k >= c && k < r) s -= l[r][k] * inv[k][c];
      }
      inv[r][c] = s * rinv[r];
    }
  }
}

// x = A^-1 b = L^-T (L^-1 b).
__device__ __forceinline__ void inverse_solve6(const double (&inv)[6][6], const double (&b)[6], double (&x)[6]) {
  double y[6];
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      if (k <= r) s += inv[r][k] * b[k];
    }
    y[r] = s;
  }
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      if (k >= r) s += inv[k][r] * y[k];
    }
    x[r] = s;
  }
}

// The same three steps on the packed lower triangle (element (r, c), c <= r,
// at tri(r, c)), in place: the factor overwrites the matrix and the inverse
// overwrites the factor.  Each element takes cholesky6's, lower_inverse6's
// and inverse_solve6's operations in their order (the upper zeros only ever
// add exact zeros there), so the results are theirs bit for bit; a third of
// the registers keeps the one-thread step free of local-memory spills.
__host__ __device__ constexpr int tri(int r, int c) { return r * (r + 1) / 2 + c; }

__device__ __forceinline__ bool cholesky_packed(double (&m)[21], double (&rinv)[6]) {
  bool ok = true;
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    double d = m[tri(c, c)];
#pragma unroll
    for (int k = 0; k < c; ++k) d -= m[tri(c, k)] * m[tri(c, k)];
    ok = ok && (d > 0.0);
    const double lc = sqrt(fmax(d, 1e-300));
    m[tri(c, c)] = lc;
    rinv[c] = 1.0 / lc;
#pragma unroll
    for (int r = c + 1; r < 6; ++r) {
      double s = m[tri(r, c)];
#pragma unroll
      for (int k = 0; k < c; ++k) s -= m[tri(r, k)] * m[tri(c, k)];
      m[tri(r, c)] = s * rinv[c];
    }
  }
  return ok;
}

// Column by column, rows downward: inv[r][c] reads the factor's row r from
// column c on (not yet overwritten) and the inverse's column c above row r.
__device__ __forceinline__ void lower_inverse_packed(double (&m)[21], const double (&rinv)[6]) {
#pragma unroll
  for (int c = 0; c < 6; ++c) {
#pragma unroll
    for (int r = c; r < 6; ++r) {
      double s = (r == c) ? 1.0 : 0.0;
#pragma unroll
      for (int k = c; k < r; ++k) s -= m[tri(r, k)] * m[tri(k, c)];
      m[tri(r, c)] = s * rinv[r];
    }
  }
}

__device__ __forceinline__ void inverse_solve_packed(const double (&inv)[21], const double (&b)[6], double (&x)[6]) {
  double y[6];
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k <= r; ++k) s += inv[tri(r, k)] * b[k];
    y[r] = s;
  }
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    double s = 0.0;
#pragma unroll
    for (int k = r; k < 6; ++k) s += inv[tri(k, r)] * y[k];
    x[r] = s;
  }
}

// Element (r, c) of the normal matrix from the 29 sums (its upper triangle,
// row-major, then the right-hand side and the residual terms).
__device__ __forceinline__ double normal_entry(const float* sums, int r, int c) {
  const int i = r < c ? r : c, j = r < c ? c : r;
  return static_cast<double>(sums[i * 6 - i * (i - 1) / 2 + (j - i)]);
}

// LDL^T solve with symmetric diagonal pivoting (largest remaining diagonal
// first).  An exactly zero pivot (a rank-deficient system such as a single
// plane) takes a zero solution component, the minimum-norm convention of the
// reference's LDLT solve (icp_optimizer.cpp:391).
__device__ void ldlt_solve6(const double (&in)[6][6], const double (&b)[6], double (&x)[6]) {
  double a[6][6], l[6][6], d[6];
  int perm[6];
  for (int i = 0; i < 6; ++i) {
    perm[i] = i;
    for (int j = 0; j < 6; ++j) {
      a[i][j] = in[i][j];
      l[i][j] = 0.0;
    }
  }
  for (int k = 0; k < 6; ++k) {
    int piv = k;
    double best = fabs(a[k][k]);
    for (int i = k + 1; i < 6; ++i) {
      if (fabs(a[i][i]) > best) {
        best = fabs(a[i][i]);
        piv = i;
      }
    }
    if (piv != k) {
      for (int i = 0; i < 6; ++i) {
        const double t = a[k][i];
        a[k][i] = a[piv][i];
        a[piv][i] = t;
      }
      for (int i = 0; i < 6; ++i) {
        const double t = a[i][k];
        a[i][k] = a[i][piv];
        a[i][piv] = t;
      }
      for (int i = 0; i < k; ++i) {
        const double t = l[k][i];
        l[k][i] = l[piv][i];
        l[piv][i] = t;
      }
      const int t = perm[k];
      perm[k] = perm[piv];
      perm[piv] = t;
    }
    d[k] = a[k][k];
    l[k][k] = 1.0;
    for (int i = k + 1; i < 6; ++i) l[i][k] = d[k] != 0.0 ? a[i][k] / d[k] : 0.0;
    for (int i = k + 1; i < 6; ++i)
      for (int j = k + 1; j < 6; ++j) a[i][j] -= l[i][k] * d[k] * l[j][k];
  }
  double y[6], z[6];
  for (int i = 0; i < 6; ++i) {
    double s = b[perm[i]];
    for (int j = 0; j < i; ++j) s -= l[i][j] * y[j];
    y[i] = s;
  }
  for (int i = 0; i < 6; ++i) y[i] = fabs(d[i]) > 1.17549435e-38 ? y[i] / d[i] : 0.0;
  for (int i = 5; i >= 0; --i) {
    double s = y[i];
    for (int j = i + 1; j < 6; ++j) s -= l[j][i] * z[j];
    z[i] = s;
  }
  for (int i = 0; i < 6; ++i) x[perm[i]] = z[i];
}

// Symmetric eigenvalues by cyclic Jacobi rotations.
__device__ bool jacobi6(const double (&in)[6][6], double (&eig)[6]) {
  double a[6][6];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) a[i][j] = in[i][j];
  for (int sweep = 0; sweep < 50; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int p = 0; p < 6; ++p) {
      diag += a[p][p] * a[p][p];
      for (int q = p + 1; q < 6; ++q) off += a[p][q] * a[p][q];
    }
    if (off <= 1e-30 * diag || off == 0.0) break;
    for (int p = 0; p < 6; ++p) {
      for (int q = p + 1; q < 6; ++q) {
        if (a[p][q] == 0.0) continue;
        const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0);
        const double s = t * c;
        for (int k = 0; k < 6; ++k) {
          const double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 6; ++k) {
          const double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
      }
    }
  }
  for (int i = 0; i < 6; ++i) {
    eig[i] = a[i][i];
    if (!isfinite(eig[i])) return false;
  }
  return true;
}

struct Stability {
  bool stable;
  float min_eigenvalue;
  float condition_number;
};

// check_system_stability (icp_optimizer.cpp:319-347).  The common
// well-conditioned case is decided without eigenvalues: with A = L L^T,
// s = ||L^-1||_F^2 >= ||A^-1||_2, so lambda_min >= 1/s and
// lambda_max / lambda_min <= ||A||_F * s; when both bounds meet the limits
// the system is stable.  Any other case computes the spectrum.  `m`
// receives L^-1 (packed) when A factorises.
__device__ Stability stability(const float* sums, const IcpParams& p, bool want_values, double (&m)[21],
                               bool& chol_ok) {
  Stability s{false, 0.0f, 0.0f};
  double fro = 0.0;  // ||A||_F^2 over the full matrix, row-major
#pragma unroll
  for (int i = 0; i < 6; ++i) {
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      const double v = normal_entry(sums, i, j);
      fro += v * v;
    }
  }
#pragma unroll
  for (int r = 0; r < 6; ++r) {
#pragma unroll
    for (int c = 0; c <= r; ++c) m[tri(r, c)] = normal_entry(sums, r, c);
  }
  double rinv[6];
  chol_ok = cholesky_packed(m, rinv);
  if (chol_ok) lower_inverse_packed(m, rinv);
  if (!want_values && chol_ok) {
    double inv2 = 0.0;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
#pragma unroll
      for (int j = 0; j <= i; ++j) inv2 += m[tri(i, j)] * m[tri(i, j)];
    }
    if (1.0 >= static_cast<double>(p.min_system_eigenvalue) * inv2 &&
        sqrt(fro) * inv2 <= static_cast<double>(p.max_condition_number)) {
      s.stable = true;
      return s;
    }
  }
  double a[6][6];
  for (int r = 0; r < 6; ++r)
    for (int c = 0; c < 6; ++c) a[r][c] = normal_entry(sums, r, c);
  double eig[6];
  if (!jacobi6(a, eig)) return s;
  double lo = eig[0], hi = eig[0];
  for (int i = 1; i < 6; ++i) {
    lo = fmin(lo, eig[i]);
    hi = fmax(hi, eig[i]);
  }
  const float mn = static_cast<float>(lo), mx = static_cast<float>(hi);
  s.min_eigenvalue = mn;
  if (mn <= 0.0f || mx <= 0.0f) return s;
  s.condition_number = mx / mn;
  s.stable = mn >= p.min_system_eigenvalue && s.condition_number <= p.max_condition_number;
  return s;
}

__device__ float grow(const IcpParams& p, float l) { return fminf(l * p.lambda_increase, p.max_lambda); }
__device__ float shrink(const IcpParams& p, float l) { return fmaxf(l * p.lambda_decrease, p.min_lambda); }

struct Increment {
  double r[9];
  double t[3];
  float update_translation, update_rotation, lambda;
  bool solved;
};

// increment_from_solution (icp_optimizer.cpp:349-365) in FP64:
// R = c I + s [u]x + (1 - c) u u^T.
__device__ void increment_from(const double (&x)[6], Increment& inc) {
  const double angle = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  for (int i = 0; i < 9; ++i) inc.r[i] = (i % 4 == 0) ? 1.0 : 0.0;
  if (angle > 1.0e-12) {
    const double ux = x[0] / angle, uy = x[1] / angle, uz = x[2] / angle;
    double s, c;
    sincos(angle, &s, &c);
    const double oc = 1.0 - c;
    inc.r[0] = c + ux * ux * oc;
    inc.r[1] = ux * uy * oc - uz * s;
    inc.r[2] = ux * uz * oc + uy * s;
    inc.r[3] = uy * ux * oc + uz * s;
    inc.r[4] = c + uy * uy * oc;
    inc.r[5] = uy * uz * oc - ux * s;
    inc.r[6] = uz * ux * oc - uy * s;
    inc.r[7] = uz * uy * oc + ux * s;
    inc.r[8] = c + uz * uz * oc;
  }
  inc.t[0] = x[3];
  inc.t[1] = x[4];
  inc.t[2] = x[5];
  inc.update_translation = static_cast<float>(sqrt(x[3] * x[3] + x[4] * x[4] + x[5] * x[5]));
  inc.update_rotation = static_cast<float>(angle);
  inc.solved = true;
}

__device__ bool within_caps(const Increment& inc, const IcpParams& p) {
  return inc.update_translation <= p.max_update_translation && inc.update_rotation <= p.max_update_rotation;
}

// solve_increment (icp_optimizer.cpp:370-402) in FP64: a Cholesky solve for
// positive definite systems, the pivoted LDL^T for the rank-deficient ones.
// Undamped: one attempt, with the inverse factor of the stability test
// (`inv`, packed) when the system factorised.
__device__ Increment solve_increment(const float* sums, float lambda, const IcpParams& p, const double (&inv)[21],
                                     bool chol_ok) {
  Increment last;
  last.solved = false;
  last.update_translation = last.update_rotation = last.lambda = 0.0f;
  double rhs[6];
  for (int r = 0; r < 6; ++r) rhs[r] = static_cast<double>(sums[21 + r]);
  if (p.damping_mode == KF_DAMPING_NONE) {
    double x[6];
    if (chol_ok) {
      inverse_solve_packed(inv, rhs, x);
    } else {
      double a[6][6];
      for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) a[r][c] = normal_entry(sums, r, c);
      ldlt_solve6(a, rhs, x);
    }
    bool finite = true;
    for (int i = 0; i < 6; ++i) finite = finite && isfinite(x[i]);
    if (finite) {
      increment_from(x, last);
      last.lambda = lambda;
    }
    return last;
  }
  double base[6][6];
  for (int r = 0; r < 6; ++r)
    for (int c = 0; c < 6; ++c) base[r][c] = normal_entry(sums, r, c);
  float scale = lambda;
  for (int attempt = 0; attempt < 8; ++attempt) {
    double damped[6][6], x[6];
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) damped[i][j] = base[i][j];
    for (int r = 0; r < 6; ++r) {
      double off = 0.0;
      if (p.damping_mode == KF_DAMPING_IDENTITY) off = scale;
      if (p.damping_mode == KF_DAMPING_DIAGONAL) off = static_cast<double>(scale) * base[r][r];
      damped[r][r] += off;
    }
    double l[6][6], rinv[6], dinv[6][6];
    if (cholesky6(damped, l, rinv)) {
      lower_inverse6(l, rinv, dinv);
      inverse_solve6(dinv, rhs, x);
    } else {
      ldlt_solve6(damped, rhs, x);
    }
    bool finite = true;
    for (int i = 0; i < 6; ++i) finite = finite && isfinite(x[i]);
    if (finite) {
      increment_from(x, last);
      last.lambda = scale;
      if (within_caps(last, p)) return last;
    }
    scale = grow(p, scale);
  }
  return last;
}

// Rigid inverse in FP64, rounded to float ({R^T, -R^T t}).
__device__ void write_float_inverse(const double* pose, float* out) {
  // pose is a row-major 3x4 matrix [R | t]
  double rt[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) rt[i * 3 + j] = pose[j * 4 + i];
  const double t[3] = {pose[3], pose[7], pose[11]};
  for (int i = 0; i < 3; ++i) {
    out[i * 3 + 0] = static_cast<float>(rt[i * 3 + 0]);
    out[i * 3 + 1] = static_cast<float>(rt[i * 3 + 1]);
    out[i * 3 + 2] = static_cast<float>(rt[i * 3 + 2]);
    out[9 + i] = static_cast<float>(-(rt[i * 3 + 0] * t[0] + rt[i * 3 + 1] * t[1] + rt[i * 3 + 2] * t[2]));
  }
}

// float kf_rigid layout: r[9] row-major then t[3].  The FP64 pose is a
// row-major 3x4 matrix.
__device__ void pose_to_rigid_floats(const double* pose, float* out) {
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) out[i * 3 + j] = static_cast<float>(pose[i * 4 + j]);
    out[9 + i] = static_cast<float>(pose[i * 4 + 3]);
  }
}

// One Gauss-Newton / LM step of estimate_with on the combined sums.
__device__ __noinline__ void gauss_newton_step(IcpState* st, const float* sums_in, unsigned long long count_in,
                                  const IcpParams& p, bool want_values) {
  const float* sums = sums_in;
  unsigned long long count = count_in;
  st->iterations += 1;
  st->correspondences = count;
  if (count > 0) st->mean_point_distance = sums[27] / static_cast<float>(count);
  if (count < p.min_correspondences) {
    st->status = KF_ICP_TOO_FEW_CORRESPONDENCES;
    return;
  }
  st->mean_squared_residual = sums[28] / static_cast<float>(count);
  const bool active = p.damping_mode != KF_DAMPING_NONE;
  bool accepted = true;
  if (p.adaptive && active) {
    const float cost = sums[28] / static_cast<float>(count);
    accepted = !st->have_best || cost <= st->best_cost;
    if (accepted) {
      st->have_best = 1;
      st->best_cost = cost;
      for (int i = 0; i < 12; ++i) st->best_pose[i] = st->pose[i];
      for (int i = 0; i < kIcpSums; ++i) st->best_sums[i] = sums[i];
      st->best_count = count;
      st->lambda = shrink(p, st->lambda);
    } else {
      st->rejected_steps += 1;
      for (int i = 0; i < 12; ++i) st->pose[i] = st->best_pose[i];
      sums = st->best_sums;
      count = st->best_count;
      st->lambda = grow(p, st->lambda);
    }
  }
  double inv[21];
  bool chol_ok = false;
  const Stability stab = stability(sums, p, want_values, inv, chol_ok);
  st->min_system_eigenvalue = stab.min_eigenvalue;
  st->condition_number = stab.condition_number;
  if (!stab.stable && !active) {
    st->status = KF_ICP_UNCONSTRAINED_SYSTEM;
    return;
  }
  const Increment inc = solve_increment(sums, st->lambda, p, inv, chol_ok);
  if (!inc.solved) {
    st->status = KF_ICP_SOLVE_FAILED;
    return;
  }
  st->lambda = inc.lambda;
  st->damping_lambda = inc.lambda;
  st->update_translation = inc.update_translation;
  st->update_rotation = inc.update_rotation;
  if (!within_caps(inc, p)) {
    st->status = KF_ICP_UPDATE_TOO_LARGE;
    return;
  }
  // pose = increment * pose (icp_optimizer.cpp:286)
  double next[12];
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      next[i * 4 + j] = inc.r[i * 3 + 0] * st->pose[0 * 4 + j] + inc.r[i * 3 + 1] * st->pose[1 * 4 + j] +
                        inc.r[i * 3 + 2] * st->pose[2 * 4 + j];
    }
    next[i * 4 + 3] = inc.r[i * 3 + 0] * st->pose[3] + inc.r[i * 3 + 1] * st->pose[7] +
                      inc.r[i * 3 + 2] * st->pose[11] + inc.t[i];
  }
  for (int i = 0; i < 12; ++i) st->pose[i] = next[i];
  pose_to_rigid_floats(st->pose, st->camera);
  if (accepted && inc.update_translation < p.min_update_translation &&
      inc.update_rotation < p.min_update_rotation) {
    st->status = KF_ICP_CONVERGED;
  }
}

// One CTA's share of a correspondence sweep: CTA `cta` of `ctas` associates
// its pixels (Pix per thread and grid step) and writes its partial slot - the
// 29 sums and, as integer bits in slot kIcpSums, the matched pixel count.
template <int Pix>
__device__ __forceinline__ void sweep_cta(const IcpLevelArgs& a, const Rigid& cam, const Rigid& model,
                                          const IcpParams& p, unsigned cta, unsigned ctas, float* __restrict__ slot,
                                          float (&s_warp)[kIcpBlock / 32][kIcpSlot]) {
  // acc[0..28]: the 29 sums, acc[29]: matched pixels, acc[30..31]: padding
  float acc[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) acc[i] = 0.0f;
  const uint32_t pixels = a.live_width * a.live_height;
  const uint32_t stride = ctas * kIcpBlock;
  for (uint32_t first = cta * kIcpBlock + threadIdx.x; first < pixels; first += stride * Pix) {
    // Pix pixels per thread, each step of the association issued for all of
    // them before the next, so their memory latencies overlap
    f3 src[Pix], lnr[Pix];
    long mi[Pix];
#pragma unroll
    for (int q = 0; q < Pix; ++q) {
      const uint32_t pix = first + q * stride;
      mi[q] = -1;
      src[q] = lnr[q] = make(0.0f, 0.0f, 0.0f);
      if (pix < pixels) {
        const f3 lv = ldg3(a.live_vertices + static_cast<size_t>(pix) * 3);
        const f3 ln = ldg3(a.live_normals + static_cast<size_t>(pix) * 3);
        if (finite3(lv) && finite3(ln)) {
          const f3 source = apply(cam, lv);
          const f3 sim = apply(model, source);
          if (finite3(sim) && sim.z > 0.0f) {
            float px, py;
            project(a.model_intrinsics, sim, px, py);
            const long mx = lroundf(px), my = lroundf(py);
            if (mx >= 0 && my >= 0 && mx < static_cast<long>(a.model_width) &&
                my < static_cast<long>(a.model_height)) {
              mi[q] = my * static_cast<long>(a.model_width) + mx;
              src[q] = source;
              lnr[q] = ln;
            }
          }
        }
      }
    }
    f3 mv[Pix], mn[Pix];
#pragma unroll
    for (int q = 0; q < Pix; ++q) {
      mv[q] = mn[q] = make(kNaN, kNaN, kNaN);
      if (mi[q] >= 0) {
        mv[q] = ldg3(a.model_points + static_cast<size_t>(mi[q]) * 3);
        mn[q] = ldg3(a.model_normals + static_cast<size_t>(mi[q]) * 3);
      }
    }
#pragma unroll
    for (int q = 0; q < Pix; ++q) {
      float j[6], residual, distance;
      if (mi[q] < 0 || !finish_match(src[q], lnr[q], mv[q], mn[q], cam, p.max_point_distance, p.min_normal_dot, j,
                                     residual, distance)) {
        continue;
      }
      int e = 0;
#pragma unroll
      for (int r = 0; r < 6; ++r) {
#pragma unroll
        for (int c = r; c < 6; ++c) {
          acc[e] += j[r] * j[c];
          ++e;
        }
      }
#pragma unroll
      for (int r = 0; r < 6; ++r) acc[21 + r] += j[r] * residual;
      acc[27] += distance;
      acc[28] += residual * residual;
      acc[29] += 1.0f;
    }
  }
  // Warp: recursive halving, 31 shuffles; lane L ends with the warp's sum of
  // value L (a fixed order).
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 16; k >= 1; k >>= 1) {
    const bool upper = (lane & k) != 0;
#pragma unroll
    for (int i = 0; i < k; ++i) {
      const float give = upper ? acc[i] : acc[i + k];
      const float keep = upper ? acc[i + k] : acc[i];
      acc[i] = keep + __shfl_xor_sync(0xFFFFFFFFu, give, k);
    }
  }
  s_warp[warp][lane] = acc[0];
  __syncthreads();
  if (threadIdx.x < kIcpSlot) {
    float sum = 0.0f;
    for (int w = 0; w < kIcpBlock / 32; ++w) sum += s_warp[w][threadIdx.x];
    // the count travels as integer bits in slot kIcpSums
    slot[threadIdx.x] = threadIdx.x == kIcpSums ? __uint_as_float(static_cast<unsigned>(sum)) : sum;
    __threadfence();
  }
}

// Shared memory of the combine: the eight segment sums and compensations.
struct CombineShared {
  float seg_sum[kIcpSegments][kIcpSlot];
  float seg_comp[kIcpSegments][kIcpSlot];
  float total[kIcpSlot];
  unsigned long long count;
};

// Deterministic Kahan-compensated combine of `ctas` partial slots, by all
// threads of the CTA: warp g (segment g of kIcpSegments) lane i (sum i)
// loads value i of slots g, g + kIcpSegments, ... - every load in flight at
// once, each warp's loads one coalesced row per slot - and compensates over
// them in slot order; then the segment results of each sum are combined in
// segment order.  Ends with c.total / c.count valid after a barrier.
__device__ __forceinline__ void combine_slots(const float* __restrict__ slots, unsigned ctas, CombineShared& c) {
  static_assert(kIcpBlock == kIcpSegments * 32 && kIcpSlot == 32, "one warp per segment, one lane per slot value");
  constexpr unsigned kPerSegment = (kIcpMaxGrid + kIcpSegments - 1) / kIcpSegments;
  const unsigned i = threadIdx.x & 31u, g = threadIdx.x >> 5;
  float v[kPerSegment];
#pragma unroll
  for (unsigned u = 0; u < kPerSegment; ++u) {
    const unsigned b = g + kIcpSegments * u;
    v[u] = b < ctas ? __ldcg(slots + b * kIcpSlot + i) : 0.0f;
  }
  if (i < kIcpSums) {
    float sum = 0.0f, comp = 0.0f;
#pragma unroll
    for (unsigned u = 0; u < kPerSegment; ++u) {
      if (g + kIcpSegments * u >= ctas) break;
      const float y = v[u] - comp;
      const float t = sum + y;
      comp = (t - sum) - y;
      sum = t;
    }
    c.seg_sum[g][i] = sum;
    c.seg_comp[g][i] = comp;
  } else if (i == kIcpSums) {
    unsigned n = 0;
#pragma unroll
    for (unsigned u = 0; u < kPerSegment; ++u) {
      if (g + kIcpSegments * u >= ctas) break;
      n += __float_as_uint(v[u]);
    }
    c.seg_sum[g][i] = __uint_as_float(n);
  }
  __syncthreads();
  if (threadIdx.x < kIcpSums) {
    float sum = 0.0f, comp = 0.0f;
    for (unsigned g2 = 0; g2 < kIcpSegments; ++g2) {
      const float y = (c.seg_sum[g2][threadIdx.x] - c.seg_comp[g2][threadIdx.x]) - comp;
      const float t = sum + y;
      comp = (t - sum) - y;
      sum = t;
    }
    c.total[threadIdx.x] = sum;
  } else if (threadIdx.x == kIcpSums) {
    unsigned long long n = 0;
    for (unsigned g2 = 0; g2 < kIcpSegments; ++g2) n += __float_as_uint(c.seg_sum[g2][kIcpSums]);
    c.count = n;
  }
  __syncthreads();
}

// One sweep per launch, one CTA per SM, Pix live pixels per thread and
// grid step; the last CTA to arrive (an atomic ticket, no waiting) combines
// the slots into the state's sums and count and, with Solve, takes the
// Gauss-Newton step - icp_level_kernel's step, one launch per step (the
// frame graphs of a batch, whose members' levels must share the GPU).
template <bool Solve, int Pix>
__global__ void __launch_bounds__(kIcpBlock, 1)
    icp_iteration_kernel(IcpLevelArgs a, IcpState* __restrict__ st, float* __restrict__ partials, IcpParams p,
                         int want_values) {
  __shared__ int s_flag;
  __shared__ float s_warp[kIcpBlock / 32][kIcpSlot];
  __shared__ CombineShared s_combine;
  if (threadIdx.x == 0) s_flag = (st->status != kIcpRunning);
  __syncthreads();
  if (s_flag) return;
  sweep_cta<Pix>(a, rigid_load(st->camera), rigid_load(st->model), p, blockIdx.x, gridDim.x,
                 partials + blockIdx.x * kIcpSlot, s_warp);
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned ticket = atomicAdd(&st->arrived, 1u);
    s_flag = (ticket == gridDim.x - 1) ? 1 : 0;
  }
  __syncthreads();
  if (!s_flag) return;
  __threadfence();
  combine_slots(partials, gridDim.x, s_combine);
  if (threadIdx.x == 0) {
    st->arrived = 0;
    for (int i = 0; i < kIcpSums; ++i) st->sums[i] = s_combine.total[i];
    st->count = s_combine.count;
    if (Solve) gauss_newton_step(st, s_combine.total, s_combine.count, p, want_values != 0);
  }
}

// ProjectiveIcpTracker's level start (icp_optimizer.cpp:208-230): counters
// and damping reset, status running unless a previous level of the frame
// failed, the float camera and the model world_to_camera from the pose.
__device__ void level_begin(IcpState* st, float damping_lambda) {
  st->arrived = 0;
  st->iterations = 0;
  st->have_best = 0;
  st->lambda = damping_lambda;
  st->rejected_steps = 0;
  st->correspondences = 0;
  st->mean_point_distance = 0.0f;
  st->mean_squared_residual = 0.0f;
  st->min_system_eigenvalue = 0.0f;
  st->condition_number = 0.0f;
  st->update_translation = 0.0f;
  st->update_rotation = 0.0f;
  st->damping_lambda = 0.0f;
  if (st->failed) {
    st->status = KF_ICP_NOT_RUN;
    return;
  }
  st->status = kIcpRunning;
  pose_to_rigid_floats(st->pose, st->camera);
  write_float_inverse(st->pose, st->model);
}

// The level's outcome: a loop that ran out of steps is MAX_ITERATIONS; a
// status other than that or CONVERGED fails the frame (later levels skip).
// level >= 0 records the per-level results of the frame.
__device__ void level_end(IcpState* st, int level) {
  if (st->status == kIcpRunning) st->status = KF_ICP_MAX_ITERATIONS;
  if (level >= 0 && level < 4) {
    st->level_status[level] = st->status;
    st->level_iterations[level] = st->iterations;
    st->level_correspondences[level] = st->correspondences;
  }
  if (st->status != KF_ICP_MAX_ITERATIONS && st->status != KF_ICP_CONVERGED) st->failed = 1;
  pose_to_rigid_floats(st->pose, st->camera);
  write_float_inverse(st->pose, st->world_to_camera);
}

__device__ __forceinline__ unsigned load_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// A grid-barrier wait gives up after 250 ms (the sweep it waits for takes
// microseconds), or after kBarrierPolls polls should the timer not advance
// (the first kBarrierSpinPolls polls back to back, the rest about 100 ns
// apart).
constexpr unsigned long long kBarrierWaitNs = 250000000ull;
constexpr uint32_t kBarrierPolls = 1u << 24;
constexpr uint32_t kBarrierSpinPolls = 4096u;

__device__ __forceinline__ unsigned long long load_acquire64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Counting grid barrier, called by thread 0 of every CTA of a cooperative
// launch (all CTAs resident, so every arrival comes): barrier `index` of a
// launch whose arrivals started at `base` completes once the count reaches
// base + (index + 1) * ctas.  An arrival is one fire-and-forget add after a
// fence; the count only grows, so nothing is cleared between barriers.  A
// wait that runs out of time, or sees another CTA's give-up, marks the
// barrier broken and returns false; the kernel then returns and the host
// reports KF_ERR_DEVICE_TIMEOUT (and clears the barrier).
__device__ bool grid_barrier(IcpBarrier* b, unsigned long long base, uint32_t index, unsigned ctas) {
  const unsigned long long target = base + (static_cast<unsigned long long>(index) + 1ull) * ctas;
  __threadfence();
  atomicAdd(&b->count, 1ull);
  const unsigned long long start = global_ns();
  for (uint32_t poll = 0; poll < kBarrierPolls; ++poll) {
    if (load_acquire64(&b->count) >= target) {
      __threadfence();
      return true;
    }
    if ((poll & 63u) == 63u) {
      if (load_acquire(&b->broken) != 0u) return false;
      if (global_ns() - start > kBarrierWaitNs) break;
    }
    // the waits are microseconds: poll back to back at first, then sleep
    if (poll >= kBarrierSpinPolls) __nanosleep(100);
  }
  atomicExch(&b->broken, 1u);
  return false;
}

// One whole ICP level in one cooperative launch
// (BasicDeviceCorrespondenceSweep::run_loop, icp_correspondence.cu:397-439,
// with the sweep of :216-343): with `begin`, the level start; then up to
// `iterations` Gauss-Newton steps, each a sweep by every CTA, a grid
// barrier, and the combine plus FP64 step run redundantly by every CTA on
// its own shared-memory copy of the tracker state (the same inputs in the
// same order, so every copy takes the same step and no second barrier is
// needed); then the level end, written back by CTA 0.  The partial slots
// alternate between two buffers by step parity: a CTA may write step i+1's
// slot while another still reads step i's.  Every CTA sees the same status
// and leaves the loop at the same step.  The sweep, the slot layout and the
// combine are icp_iteration_kernel's, so the steps are bit-identical to a
// launch per step at the same grid.
template <int Pix>
__global__ void __launch_bounds__(kIcpBlock, 1)
    icp_level_kernel(IcpLevelArgs a, IcpState* __restrict__ st, float* __restrict__ partials, IcpParams p,
                     uint32_t iterations, int level, int begin, int want_values) {
  __shared__ int s_flag;
  __shared__ float s_warp[kIcpBlock / 32][kIcpSlot];
  __shared__ CombineShared s_combine;
  __shared__ IcpState s_st;
  constexpr unsigned kWords = offsetof(IcpState, barrier) / sizeof(unsigned);
  static_assert(offsetof(IcpState, barrier) % sizeof(unsigned) == 0, "state words");
  {
    const unsigned* src = reinterpret_cast<const unsigned*>(st);
    unsigned* dst = reinterpret_cast<unsigned*>(&s_st);
    for (unsigned w = threadIdx.x; w < kWords; w += kIcpBlock) dst[w] = src[w];
  }
  __syncthreads();
  if (threadIdx.x == 0 && begin) level_begin(&s_st, p.damping_lambda);
  // where this launch's barrier arrivals start (set by the previous launch's
  // CTA 0 after its last barrier, when every CTA of that launch had arrived)
  const unsigned long long base = st->barrier.base;
  __syncthreads();
  const unsigned ctas = gridDim.x;
  uint32_t steps = 0;
  for (uint32_t it = 0; it < iterations; ++it) {
    if (s_st.status != kIcpRunning) break;
    float* slots = partials + (it & 1u) * (kIcpMaxGrid * kIcpSlot);
    sweep_cta<Pix>(a, rigid_load(s_st.camera), rigid_load(s_st.model), p, blockIdx.x, ctas,
                   slots + blockIdx.x * kIcpSlot, s_warp);
    __syncthreads();
    if (threadIdx.x == 0) {
      s_flag = grid_barrier(&st->barrier, base, it, ctas) ? 1 : 0;
      // a barrier that gave up fails the frame: later levels skip, the
      // integration does not run, and the host reports the timeout
      if (!s_flag) st->failed = 1;
    }
    __syncthreads();
    if (!s_flag) return;
    combine_slots(slots, ctas, s_combine);
    if (threadIdx.x == 0) {
      for (int i = 0; i < kIcpSums; ++i) s_st.sums[i] = s_combine.total[i];
      s_st.count = s_combine.count;
      gauss_newton_step(&s_st, s_combine.total, s_combine.count, p, want_values != 0);
    }
    __syncthreads();
    ++steps;
  }
  if (blockIdx.x != 0) return;
  if (threadIdx.x == 0) {
    level_end(&s_st, level);
    // every CTA read `base` before its first arrival, so after CTA 0's last
    // barrier nothing reads it any more
    if (steps != 0u) st->barrier.base = base + static_cast<unsigned long long>(steps) * ctas;
  }
  __syncthreads();
  const unsigned* src = reinterpret_cast<const unsigned*>(&s_st);
  unsigned* dst = reinterpret_cast<unsigned*>(st);
  for (unsigned w = threadIdx.x; w < kWords; w += kIcpBlock) dst[w] = src[w];
}

__global__ void icp_level_begin_kernel(IcpState* st, float damping_lambda) {
  if (threadIdx.x == 0) level_begin(st, damping_lambda);
}

__global__ void icp_level_end_kernel(IcpState* st, int level) {
  if (threadIdx.x == 0) level_end(st, level);
}

__global__ void icp_set_pose_kernel(IcpState* st, kf_rigid pose, int reset_frame) {
  if (threadIdx.x != 0) return;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) st->pose[i * 4 + j] = static_cast<double>(pose.r[i * 3 + j]);
    st->pose[i * 4 + 3] = static_cast<double>(pose.t[i]);
  }
  pose_to_rigid_floats(st->pose, st->camera);
  write_float_inverse(st->pose, st->world_to_camera);
  if (reset_frame) {
    st->failed = 0;
    st->status = KF_ICP_NOT_RUN;
    for (int l = 0; l < 4; ++l) {
      st->level_status[l] = KF_ICP_NOT_RUN;
      st->level_iterations[l] = 0;
      st->level_correspondences[l] = 0;
    }
  }
}

}  // namespace

IcpParams icp_params_from(const kf_icp_options& o) {
  IcpParams p;
  p.min_correspondences = o.min_correspondences;
  p.max_point_distance = o.max_point_distance;
  p.min_normal_dot = o.min_normal_dot;
  p.min_update_translation = o.min_update_translation;
  p.min_update_rotation = o.min_update_rotation;
  p.max_update_translation = o.max_update_translation;
  p.max_update_rotation = o.max_update_rotation;
  p.min_system_eigenvalue = o.min_system_eigenvalue;
  p.max_condition_number = o.max_condition_number;
  p.damping_mode = o.damping_mode;
  p.damping_lambda = o.damping_lambda;
  p.adaptive = o.adaptive_damping;
  p.lambda_increase = o.lambda_increase;
  p.lambda_decrease = o.lambda_decrease;
  p.min_lambda = o.min_lambda;
  p.max_lambda = o.max_lambda;
  return p;
}

unsigned icp_grid_for(uint32_t pixels) {
  const unsigned g = ceil_div(pixels, kIcpBlock * kIcpPixels);
  return g < static_cast<unsigned>(kIcpMaxGrid) ? (g == 0 ? 1 : g) : static_cast<unsigned>(kIcpMaxGrid);
}

namespace {

// Largest cooperative grid of icp_level_kernel per device (all CTAs
// resident at once), set by prepare_icp_kernels.
constexpr int kMaxIcpDevices = 64;
std::atomic<unsigned> g_level_grid_cap[kMaxIcpDevices];

int current_device() {
  int device = 0;
  check(cudaGetDevice(&device), "cudaGetDevice");
  require(device >= 0 && device < kMaxIcpDevices, "ICP: device ordinal out of range");
  return device;
}

}  // namespace

void prepare_icp_kernels() {
  const int device = current_device();
  int per_sm = 0, sms = 0;
  check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, icp_level_kernel<kIcpPixels>, kIcpBlock, 0),
        "icp level kernel occupancy");
  check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
  const long cap = static_cast<long>(per_sm) * sms;
  require(cap >= 1, "ICP: the level kernel cannot be resident on this device");
  g_level_grid_cap[device].store(static_cast<unsigned>(cap < kIcpMaxGrid ? cap : kIcpMaxGrid));
}

void launch_icp_level_begin(IcpState* state, float damping_lambda, cudaStream_t s) {
  icp_level_begin_kernel<<<1, 32, 0, s>>>(state, damping_lambda);
  check(cudaGetLastError(), "icp_level_begin launch");
}

void launch_icp_sweep(const IcpLevelArgs& args, IcpState* state, float* partials, const IcpParams& params,
                      cudaStream_t s) {
  const uint32_t pixels = args.live_width * args.live_height;
  icp_iteration_kernel<false, kIcpPixels><<<icp_grid_for(pixels), kIcpBlock, 0, s>>>(args, state, partials, params, 0);
  check(cudaGetLastError(), "icp_iteration_kernel launch");
}

void launch_icp_level_steps(const IcpLevelArgs& args, IcpState* state, float* partials, const IcpParams& params,
                            uint32_t iterations, int level, cudaStream_t s) {
  icp_level_begin_kernel<<<1, 32, 0, s>>>(state, params.damping_lambda);
  check(cudaGetLastError(), "icp_level_begin launch");
  const uint32_t pixels = args.live_width * args.live_height;
  for (uint32_t i = 0; i < iterations; ++i) {
    icp_iteration_kernel<true, kIcpPixels><<<icp_grid_for(pixels), kIcpBlock, 0, s>>>(args, state, partials, params,
                                                                                       0);
  }
  check(cudaGetLastError(), "icp_iteration_kernel launch");
  icp_level_end_kernel<<<1, 32, 0, s>>>(state, level);
  check(cudaGetLastError(), "icp_level_end launch");
}

void launch_icp_level(const IcpLevelArgs& args, IcpState* state, float* partials, const IcpParams& params,
                      uint32_t iterations, int level, int begin, int want_values, cudaStream_t s) {
  const unsigned cap = g_level_grid_cap[current_device()].load();
  require(cap != 0, "ICP: level kernel not prepared on this device");
  unsigned grid = icp_grid_for(args.live_width * args.live_height);
  if (grid > cap) grid = cap;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kIcpBlock);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  check(cudaLaunchKernelEx(&cfg, icp_level_kernel<kIcpPixels>, args, state, partials, params, iterations, level, begin,
                           want_values),
        "icp_level_kernel launch");
}

void check_icp_barrier(const IcpState& host, IcpState* device, cudaStream_t s) {
  if (host.barrier.broken == 0u) return;
  check(cudaMemsetAsync(reinterpret_cast<char*>(device) + offsetof(IcpState, barrier), 0, sizeof(IcpBarrier), s),
        "ICP barrier reset");
  check(cudaStreamSynchronize(s), "ICP barrier reset");
  throw DeviceTimeout(
      "ICP level kernel: a grid-barrier wait gave up before every CTA arrived; the frame is marked failed");
}

void launch_icp_set_pose(IcpState* state, kf_rigid pose, int reset_frame, cudaStream_t s) {
  icp_set_pose_kernel<<<1, 32, 0, s>>>(state, pose, reset_frame);
  check(cudaGetLastError(), "icp_set_pose launch");
}

}  // namespace kf

// ---------------------------------------------------------------------------
// Allocation-free correspondence sweep.
//
// Some callers of this library cannot allocate device memory: code running
// inside another framework's memory pool or a CUDA-graph-replayed section,
// plug-ins whose host forbids cudaMalloc after start-up, or real-time loops
// that must not hit the allocator.  kf_icp_normal_equations_static serves
// them: the per-CTA partial sums live in a file-scope __device__ array that
// exists on every GPU that loads this library (about 150 KB, held until the
// process exits), so the call needs no tracker object and allocates nothing.
// ---------------------------------------------------------------------------
#include <cstring>
#include <mutex>
#include <string>

namespace kf {
namespace {

constexpr int kStaticBlock = 256;                       // threads per CTA of the static sweep
constexpr int kStaticPixelsPerCta = 4 * kStaticBlock;  // each CTA sweeps 1024 live pixels
constexpr int kStaticSlots = 1200;                  // one partial slot per CTA
constexpr uint64_t kStaticMaxPixels = static_cast<uint64_t>(kStaticSlots) * kStaticPixelsPerCta;  // 1,228,800
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float g_static_partials[kStaticSlots * kIcpSlot];
static __device__ __align__(256) IcpState g_static_state;

// Same association and accumulation as icp_iteration_kernel; the image is cut
// into 1024-pixel tiles, one per CTA, and the last CTA to finish combines the
// partial slots (Kahan-compensated, in slot order) straight from memory.
__global__ void __launch_bounds__(kStaticBlock)
    icp_static_sweep_kernel(IcpLevelArgs a, IcpState* __restrict__ st, float* __restrict__ partials, float max_d,
                            float min_dot) {
  __shared__ int s_last;
  __shared__ float s_warp[kStaticBlock / 32][kIcpSlot];
  __shared__ unsigned s_warp_count[kStaticBlock / 32];
  __shared__ float s_seg_sum[8][kIcpSlot];
  __shared__ float s_seg_comp[8][kIcpSlot];
  const Rigid cam = rigid_load(st->camera);
  const Rigid model = rigid_load(st->model);
  float acc[kIcpSums];
#pragma unroll
  for (int i = 0; i < kIcpSums; ++i) acc[i] = 0.0f;
  unsigned cnt = 0;
  const uint32_t pixels = a.live_width * a.live_height;
  const uint32_t first = blockIdx.x * kStaticPixelsPerCta;
#pragma unroll 1
  for (uint32_t k = 0; k < kStaticPixelsPerCta / kStaticBlock; ++k) {
    const uint32_t pix = first + k * kStaticBlock + threadIdx.x;
    if (pix >= pixels) break;
    float j[6], residual, distance;
    if (!match(a, cam, model, max_d, min_dot, pix % a.live_width, pix / a.live_width, j, residual, distance)) {
      continue;
    }
    int e = 0;
#pragma unroll
    for (int r = 0; r < 6; ++r) {
#pragma unroll
      for (int c = r; c < 6; ++c) {
        acc[e] += j[r] * j[c];
        ++e;
      }
    }
#pragma unroll
    for (int r = 0; r < 6; ++r) acc[21 + r] += j[r] * residual;
    acc[27] += distance;
    acc[28] += residual * residual;
    ++cnt;
  }
#pragma unroll
  for (int i = 0; i < kIcpSums; ++i) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc[i] += __shfl_xor_sync(0xFFFFFFFFu, acc[i], off);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, off);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < kIcpSums; ++i) s_warp[warp][i] = acc[i];
    s_warp_count[warp] = cnt;
  }
  __syncthreads();
  if (threadIdx.x < kIcpSums) {
    float s = 0.0f;
    for (int w = 0; w < kStaticBlock / 32; ++w) s += s_warp[w][threadIdx.x];
    partials[blockIdx.x * kIcpSlot + threadIdx.x] = s;
  } else if (threadIdx.x == kIcpSums) {
    unsigned c = 0;
    for (int w = 0; w < kStaticBlock / 32; ++w) c += s_warp_count[w];
    partials[blockIdx.x * kIcpSlot + kIcpSums] = __uint_as_float(c);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&st->arrived, 1u) == gridDim.x - 1) ? 1 : 0;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  {
    const unsigned i = threadIdx.x % kIcpSlot, g = threadIdx.x / kIcpSlot;
    if (i < kIcpSums) {
      float sum = 0.0f, comp = 0.0f;
      for (unsigned b = g; b < gridDim.x; b += 8) {
        const float y = __ldcg(partials + b * kIcpSlot + i) - comp;
        const float t = sum + y;
        comp = (t - sum) - y;
        sum = t;
      }
      s_seg_sum[g][i] = sum;
      s_seg_comp[g][i] = comp;
    } else if (i == kIcpSums) {
      unsigned c = 0;
      for (unsigned b = g; b < gridDim.x; b += 8) c += __float_as_uint(__ldcg(partials + b * kIcpSlot + kIcpSums));
      s_seg_sum[g][i] = __uint_as_float(c);
    }
  }
  __syncthreads();
  if (threadIdx.x < kIcpSums) {
    float sum = 0.0f, comp = 0.0f;
    for (int g = 0; g < 8; ++g) {
      const float y = (s_seg_sum[g][threadIdx.x] - s_seg_comp[g][threadIdx.x]) - comp;
      const float t = sum + y;
      comp = (t - sum) - y;
      sum = t;
    }
    st->sums[threadIdx.x] = sum;
  } else if (threadIdx.x == kIcpSums) {
    unsigned long long c = 0;
    for (int g = 0; g < 8; ++g) c += __float_as_uint(s_seg_sum[g][kIcpSums]);
    st->count = c;
    st->arrived = 0;
  }
}

// Device addresses of the two scratch symbols, looked up once per device.
struct StaticScratch {
  float* partials;
  IcpState* state;
};

StaticScratch static_scratch_for_current_device() {
  static std::mutex lock;
  static StaticScratch table[kMaxDevices] = {};
  int device = 0;
  check(cudaGetDevice(&device), "cudaGetDevice");
  require(device >= 0 && device < kMaxDevices, "kf_icp_normal_equations_static: device ordinal out of range");
  std::lock_guard<std::mutex> guard(lock);
  StaticScratch& entry = table[device];
  if (entry.partials == nullptr) {
    void* partials = nullptr;
    void* state = nullptr;
    check(cudaGetSymbolAddress(&partials, g_static_partials), "cudaGetSymbolAddress(partials scratch)");
    check(cudaGetSymbolAddress(&state, g_static_state), "cudaGetSymbolAddress(state scratch)");
    entry.partials = static_cast<float*>(partials);
    entry.state = static_cast<IcpState*>(state);
  }
  return entry;
}

}  // namespace
}  // namespace kf

extern "C" kf_status kf_icp_normal_equations_static(const kf_level_view* live, const float* model_points,
                                                    const float* model_normals, uint32_t model_width,
                                                    uint32_t model_height, kf_intrinsics model_intrinsics,
                                                    const kf_rigid* camera, const kf_rigid* model_world_to_camera,
                                                    float max_point_distance, float min_normal_dot, float* sums,
                                                    uint64_t* count) {
  using namespace kf;
  return guarded([&] {
    require(live && model_points && model_normals && camera && model_world_to_camera && sums && count,
            "kf_icp_normal_equations_static: null argument");
    const uint64_t pixels = static_cast<uint64_t>(live->width) * live->height;
    require((live->vertices && live->normals) || pixels == 0,
            "kf_icp_normal_equations_static: null live vertex or normal map");
    if (pixels > kStaticMaxPixels) {
      throw InvalidArgument("kf_icp_normal_equations_static: the live image has " + std::to_string(pixels) +
                            " pixels; the static scratch holds sweeps of at most " +
                            std::to_string(kStaticMaxPixels) + " pixels");
    }
    if (pixels == 0) {
      for (int i = 0; i < kIcpSums; ++i) sums[i] = 0.0f;
      *count = 0;
      return;
    }
    const StaticScratch scratch = static_scratch_for_current_device();
    // Transforms in, arrival ticket cleared: the array keeps the last call's
    // contents otherwise.
    float transforms[24];
    std::memcpy(transforms, camera->r, 9 * sizeof(float));
    std::memcpy(transforms + 9, camera->t, 3 * sizeof(float));
    std::memcpy(transforms + 12, model_world_to_camera->r, 9 * sizeof(float));
    std::memcpy(transforms + 21, model_world_to_camera->t, 3 * sizeof(float));
    static_assert(offsetof(IcpState, model) == offsetof(IcpState, camera) + 12 * sizeof(float),
                  "camera and model transforms are adjacent");
    char* state = reinterpret_cast<char*>(scratch.state);
    const unsigned zero = 0;
    check(cudaMemcpy(state + offsetof(IcpState, camera), transforms, sizeof(transforms), cudaMemcpyHostToDevice),
          "static sweep transforms upload");
    check(cudaMemcpy(state + offsetof(IcpState, arrived), &zero, sizeof(zero), cudaMemcpyHostToDevice),
          "static sweep ticket clear");
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
    const unsigned grid = static_cast<unsigned>((pixels + kStaticPixelsPerCta - 1) / kStaticPixelsPerCta);
    icp_static_sweep_kernel<<<grid, kStaticBlock, 0, 0>>>(a, scratch.state, scratch.partials, max_point_distance,
                                                       min_normal_dot);
    check(cudaGetLastError(), "icp_static_sweep_kernel launch");
    check(cudaMemcpy(sums, state + offsetof(IcpState, sums), kIcpSums * sizeof(float), cudaMemcpyDeviceToHost),
          "static sweep sums download");
    unsigned long long c = 0;
    check(cudaMemcpy(&c, state + offsetof(IcpState, count), sizeof(c), cudaMemcpyDeviceToHost),
          "static sweep count download");
    *count = c;
  });
}
