"""Fixtures of the reference's unit tests (test/tests.cpp:40-183), shared by
the oracle pins and the GPU parity tests."""

import numpy as np

import kf_oracle as ko
from kinectfusion_b200 import abi

DEPTH_1M = 5000      # tests.cpp:42
DEPTH_1P4M = 7000    # tests.cpp:43
SYNTH_RES = 32       # tests.cpp:46-51
SYNTH_VOXEL = 0.05
SYNTH_ORIGIN = (-0.8, -0.8, 0.2)
SYNTH_TRUNC = 0.05
SYNTH_IMAGE = 16     # tests.cpp:65


def synth_intrinsics():
    return abi.Intrinsics(20.0, 20.0, 7.5, 7.5)  # tests.cpp:80-83


def flat_depth(raw):
    return np.full((SYNTH_IMAGE, SYNTH_IMAGE), raw, dtype=np.uint16)


def synth_volume(**kw):
    return ko.OracleVolume(SYNTH_RES, SYNTH_VOXEL, SYNTH_ORIGIN, SYNTH_TRUNC, **kw)


NORMAL_SEEDS = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0], [1, 0, 1], [0, 1, 1], [1, -1, 0.5],
                         [-1, 0.5, 1], [0.5, 1, -1]], dtype=np.float32)  # tests.cpp:123-132


def _normalized(v):
    v = np.asarray(v, dtype=np.float32)
    length = np.float32(np.sqrt(np.float32(v[0] * v[0] + v[1] * v[1]) + np.float32(v[2] * v[2])))
    return (v / length).astype(np.float32)


def identical_surface(fx=100.0, cx=1.0):
    """3x3 live == model patch with spread normals (tests.cpp:109-146)."""
    verts = np.zeros((3, 3, 3), dtype=np.float32)
    norms = np.zeros((3, 3, 3), dtype=np.float32)
    for y in range(3):
        for x in range(3):
            z = np.float32(1.0) + np.float32(0.05) * np.float32(x + y)
            verts[y, x] = [np.float32((np.float32(x) - np.float32(cx)) * z) / np.float32(fx),
                           np.float32((np.float32(y) - np.float32(cx)) * z) / np.float32(fx), z]
            norms[y, x] = _normalized(NORMAL_SEEDS[y * 3 + x])
    return verts, norms


def planar_surface(fx=100.0, cx=1.0):
    """Fronto-parallel 3x3 plane (tests.cpp:151-178)."""
    verts = np.zeros((3, 3, 3), dtype=np.float32)
    norms = np.zeros((3, 3, 3), dtype=np.float32)
    for y in range(3):
        for x in range(3):
            verts[y, x] = [np.float32(np.float32(x) - np.float32(cx)) / np.float32(fx),
                           np.float32(np.float32(y) - np.float32(cx)) / np.float32(fx), 1.0]
            norms[y, x] = [0.0, 0.0, -1.0]
    return verts, norms


def perturbed_initial(angle=0.01, t=(0.002, -0.001, 0.0015), rotate=True):
    """AngleAxis(0.01, UnitZ) + (2, -1, 1.5) mm (tests.cpp:54-60, 916-921)."""
    m = np.eye(4, dtype=np.float64)
    if rotate:
        c, s = np.cos(angle), np.sin(angle)
        m[:2, :2] = [[c, -s], [s, c]]
    m[:3, 3] = t
    return m.astype(np.float32)


def compare_volumes(primary, reference):
    """Comparator::compare for volumes (comparison.cpp:12-41) on dense
    (tsdf, weight) pairs."""
    pt, pw = primary
    rt, rw = reference
    pv, rv = pw > 0, rw > 0
    both = pv & rv
    dist = np.abs(pt[both] - rt[both])
    wd = np.abs(pw[both] - rw[both])
    return {"compared": int(both.sum()), "only_primary": int((pv & ~rv).sum()),
            "only_reference": int((rv & ~pv).sum()),
            "max_distance_delta": float(dist.max()) if dist.size else 0.0,
            "mean_distance_delta": float(dist.mean()) if dist.size else 0.0,
            "max_weight_delta": float(wd.max()) if wd.size else 0.0}


def compare_maps(p_points, p_normals, r_points, r_normals):
    """Comparator::compare for surface maps (comparison.cpp:43-81)."""
    pv = np.isfinite(p_points).all(-1) & np.isfinite(p_normals).all(-1)
    rv = np.isfinite(r_points).all(-1) & np.isfinite(r_normals).all(-1)
    both = pv & rv
    d = np.linalg.norm((p_points[both] - r_points[both]).astype(np.float64), axis=-1)
    pn = p_normals[both].astype(np.float64)
    rn = r_normals[both].astype(np.float64)
    pn /= np.linalg.norm(pn, axis=-1, keepdims=True)
    rn /= np.linalg.norm(rn, axis=-1, keepdims=True)
    ang = np.arctan2(np.linalg.norm(np.cross(pn, rn), axis=-1), (pn * rn).sum(-1))
    return {"compared": int(both.sum()), "only_primary": int((pv & ~rv).sum()),
            "only_reference": int((rv & ~pv).sum()),
            "max_point_distance": float(d.max()) if d.size else 0.0,
            "max_normal_angle": float(ang.max()) if ang.size else 0.0}


def sphere_volume(vol, radius_fraction=0.3):
    """Writes the clamped signed distance of a sphere at the volume centre into
    a dense float oracle volume, weight 1 (tests.cpp:320-337)."""
    g = vol.geometry
    rx, ry, rz = vol.res
    extent = np.float32(rx) * np.float32(g.voxel_size)
    origin = np.array(g.origin[:], dtype=np.float32)
    center = origin + np.float32(0.5) * extent
    radius = np.float32(radius_fraction) * extent
    z, y, x = np.meshgrid(np.arange(rz), np.arange(ry), np.arange(rx), indexing="ij")
    cells = (np.stack([x, y, z], -1).astype(np.float32) + np.float32(0.5)) * np.float32(g.voxel_size) + origin
    distance = np.linalg.norm(cells - center, axis=-1).astype(np.float32) - radius
    tsdf = np.clip(distance / np.float32(g.truncation_distance), -1.0, 1.0).astype(np.float32)
    vol.voxels[:, 0] = tsdf.reshape(-1)
    vol.voxels[:, 1] = 1.0
    return center, radius


def mesh_edge_uses(triangles):
    """Undirected edge -> number of triangles using it."""
    uses = {}
    for t in np.asarray(triangles, dtype=np.int64):
        for a, b in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0])):
            key = (min(a, b), max(a, b))
            uses[key] = uses.get(key, 0) + 1
    return uses
