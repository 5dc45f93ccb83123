"""CPU oracle of the pipeline-set comparator and its CSV rows (test
infrastructure).

A numpy restatement of Comparator::compare (src/kinectfusion/comparison.cpp:
12-81, include/kinectfusion/comparison.hpp:30-90) evaluated the way the
reference's host build evaluates it: every float expression in float32 with
each multiply and add rounded on its own (no contraction), vector helpers in
the order of include/kinectfusion/vector.hpp (dot (x*x' + y*y') + z*z',
cross, norm = sqrt(dot), the host branch of normalized = three divides by
the length), atan2 from the C library (numpy's float32 arctan2), and each
mean a SEQUENTIAL double sum (Deviation::add, comparison.hpp:66-69) divided by
the compared count and cast to float.  It is pinned to the reference's own
known-answer case (test/tests.cpp:837-880) in tests/test_compare_host.py.

Only tests may import this module; the product never does.
"""

from __future__ import annotations

import numpy as np

f32 = np.float32


def _sequential_sum(values: np.ndarray) -> float:
    """Deviation's running double sum, one add at a time in index order."""
    if values.size == 0:
        return 0.0
    return float(np.cumsum(values.astype(np.float64))[-1])


def _max(values: np.ndarray) -> float:
    """std::max(max_, value) from max_ = 0: NaN values are passed over."""
    finite = values[~np.isnan(values)]
    return float(max(f32(0.0), finite.max())) if finite.size else 0.0


def _mean(values: np.ndarray, count: int) -> float:
    return 0.0 if count == 0 else float(f32(_sequential_sum(values) / count))


def _tally(primary_valid: np.ndarray, reference_valid: np.ndarray) -> tuple[np.ndarray, int, int, int]:
    """PairTally::classify (comparison.hpp:43-58) over every element."""
    both = primary_valid & reference_valid
    return (both, int(both.sum()), int((primary_valid & ~reference_valid).sum()),
            int((reference_valid & ~primary_valid).sum()))


def compare_volumes(primary, reference) -> dict:
    """Comparator::compare(ConstHostVolumeView, ConstHostVolumeView)
    (comparison.cpp:12-41) on dense host views: (tsdf, weight) float32
    arrays of the same shape, in the voxel order of the host view."""
    pt, pw = (np.asarray(a, dtype=f32).reshape(-1) for a in primary)
    rt, rw = (np.asarray(a, dtype=f32).reshape(-1) for a in reference)
    if pt.shape != rt.shape:
        raise ValueError("Volume comparison requires matching geometry")
    both, compared, only_p, only_r = _tally(pw > 0, rw > 0)
    distance = np.abs(pt[both] - rt[both])
    weight = np.abs(pw[both] - rw[both])
    return {"compared_voxels": compared, "only_primary": only_p, "only_reference": only_r,
            "max_distance_delta": _max(distance), "mean_distance_delta": _mean(distance, compared),
            "max_weight_delta": _max(weight)}


def _dot(a, b):
    return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def _norm(a):
    return np.sqrt(_dot(a, a))


def _normalized(a):
    """Host branch of normalized (vector.hpp:164-175)."""
    length = _norm(a)
    safe = np.where(length > 0, length, f32(1.0))[..., None]
    return np.where((length > 0)[..., None], a / safe, f32(0.0)).astype(f32)


def angle_between(a, b):
    """angle_between (vector.hpp:177-185)."""
    source, target = _normalized(a), _normalized(b)
    return np.arctan2(_norm(_cross(source, target)), _dot(source, target)).astype(f32)


def compare_surface_maps(p_points, p_normals, r_points, r_normals) -> dict:
    """Comparator::compare(SurfaceMaps, SurfaceMaps) (comparison.cpp:43-81)
    on HxWx3 float32 point and normal maps."""
    pp, pn, rp, rn = (np.asarray(a, dtype=f32).reshape(-1, 3) for a in (p_points, p_normals, r_points, r_normals))
    if pp.shape != rp.shape or pn.shape != pp.shape or rn.shape != rp.shape:
        raise ValueError("Surface map comparison requires matching dimensions")
    pv = np.isfinite(pp).all(-1) & np.isfinite(pn).all(-1)
    rv = np.isfinite(rp).all(-1) & np.isfinite(rn).all(-1)
    both, compared, only_p, only_r = _tally(pv, rv)
    distance = _norm(pp[both] - rp[both]).astype(f32)
    angle = angle_between(pn[both], rn[both])
    return {"compared_pixels": compared, "only_primary": only_p, "only_reference": only_r,
            "max_point_distance": _max(distance), "mean_point_distance": _mean(distance, compared),
            "max_normal_angle": _max(angle), "mean_normal_angle": _mean(angle, compared)}
