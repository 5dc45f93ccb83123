"""Shared loading and comparison helpers of the golden tests
(tests/golden/reference_small.npz, made by tests/golden/make_golden.py from
the reference compiled from its own sources)."""

import hashlib
import pathlib

import numpy as np

from kinectfusion_b200 import abi, synthetic

GOLDEN = pathlib.Path(__file__).with_name("golden") / "reference_small.npz"
SEED, FRAMES = 7, 4
RES, VOXEL, TRUNC = 64, 0.04, 0.12
ORIGIN = (-0.5 * RES * VOXEL, -0.5 * RES * VOXEL, -0.5)
K640 = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)


def load():
    """(fixture arrays, the regenerated input sequence); fails if the seeded
    generator no longer reproduces the frames the fixture was made from."""
    g = np.load(GOLDEN)
    seq = synthetic.make_sequence(seed=SEED, frames=FRAMES)
    for f in range(FRAMES):
        digest = hashlib.sha256(np.ascontiguousarray(seq.depth[f]).tobytes()).hexdigest()
        assert digest == str(g["frame_sha256"][f]), f"synthetic frame {f} differs from the fixture's input"
    return g, seq


def pose_error(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    dt = np.linalg.norm(a[:3, 3] - b[:3, 3])
    r = a[:3, :3].T @ b[:3, :3]
    skew = np.array([r[2, 1] - r[1, 2], r[0, 2] - r[2, 0], r[1, 0] - r[0, 1]]) / 2
    return dt, np.arctan2(np.linalg.norm(skew), (np.trace(r) - 1) / 2)


def check_pyramid(g, level0_depth, level2_vertices, level2_normals):
    """Level-0 filtered depth bit-exact up to a handful of pixels one raw unit
    apart (the reference's bilateral weight is glibc expf, one ulp off the
    correctly rounded exp for ~1e-4 of arguments); level-2 maps bit-exact
    except where such a pixel moved a downsampled depth."""
    d = level0_depth.astype(np.int32) - g["pyramid_l0_depth"].astype(np.int32)
    assert np.abs(d).max() <= 1 and (d != 0).sum() <= 5, (np.abs(d).max(), (d != 0).sum())
    for mine, ref in ((level2_vertices, g["pyramid_l2_vertices"]), (level2_normals, g["pyramid_l2_normals"])):
        same = np.all((mine == ref) | (np.isnan(mine) & np.isnan(ref)), axis=-1)
        assert (~same).sum() <= 10, (~same).sum()


def check_volume(g, raw):
    """Raw voxels bit-exact except the few whose normals came from such a
    pixel (at most 1e-4 of the observed voxels)."""
    ref = g["voxels"]
    diff = np.any(raw.view(np.uint32).reshape(-1, 2) != ref.view(np.uint32), axis=1)
    observed = int((ref[:, 1] > 0).sum())
    assert observed > 20000
    assert diff.sum() <= 1e-4 * observed, (diff.sum(), observed)


def check_maps(g, points, normals):
    same = np.all(((points == g["raycast_points"]) | (np.isnan(points) & np.isnan(g["raycast_points"]))) &
                  ((normals == g["raycast_normals"]) | (np.isnan(normals) & np.isnan(g["raycast_normals"]))),
                  axis=-1)
    assert np.isfinite(g["raycast_points"][..., 0]).sum() > 0.2 * 160 * 120
    assert same.mean() >= 0.999, same.mean()


def check_loop(g, poses, statuses=None):
    """Poses within 1e-4 m / rad; per level the same outcome: a failure code
    equal, a success (converged, or at the iteration cap) a success - which
    of the two can flip where the last update sits at the 1e-5 threshold,
    with the sums' rounding order."""
    for f in range(FRAMES):
        dt, da = pose_error(poses[f], g["loop_poses"][f])
        assert dt < 1e-4 and da < 1e-4, (f, dt, da)
    if statuses is not None:
        success = (abi.KF_ICP_MAX_ITERATIONS, abi.KF_ICP_CONVERGED)
        mine = np.asarray(statuses)[:, :3]
        ref = g["loop_status"][:, :3]
        same = (mine == ref) | (np.isin(mine, success) & np.isin(ref, success))
        assert same.all(), (mine, ref)


SPARSE_RES, SPARSE_VOXEL, SPARSE_TRUNC = 128, 0.02, 0.05
SPARSE_ORIGIN = (-0.5 * SPARSE_RES * SPARSE_VOXEL, -0.5 * SPARSE_RES * SPARSE_VOXEL, -0.5)


def check_mesh(g, positions, triangle_count):
    """The vertex set of the reference's mesh (it depends only on which
    edges cross; the triangle table is this project's own with the same
    triangle count per case), up to the vertices of voxels an expf pixel
    moved."""
    order = np.lexsort(np.asarray(positions).T[::-1])
    mine = np.asarray(positions)[order]
    ref = g["mesh_positions"]
    assert len(ref) > 1000
    assert abs(len(mine) - len(ref)) <= 2 and abs(int(triangle_count) - int(g["mesh_triangles"])) <= 4
    if len(mine) == len(ref):
        assert np.all(mine == ref, axis=1).mean() >= 0.998


def check_sparse(g, grid, block_voxels):
    """The reference's BlockRep<kHost> allocation set, and each allocated
    block's raw voxels (`block_voxels(blocks)` returns them in block order)."""
    blocks = np.nonzero(np.asarray(grid) != 0xFFFFFFFF)[0]
    assert np.array_equal(blocks, g["sparse_blocks"])
    mine = np.asarray(block_voxels(blocks)).view(np.uint32)
    diff = np.any(mine != g["sparse_voxels"].view(np.uint32), axis=1)
    assert diff.sum() <= 2, diff.sum()
