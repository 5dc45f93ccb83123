"""The oracle against golden outputs of the reference itself
(tests/golden/reference_small.npz: the reference's host implementation,
compiled from its own sources, on seeded synthetic frames; see
tests/golden/make_golden.py).  Runs without the reference or its compiled
library: pyramid, 64^3 angle-weighted integration, 160x120 raycast, the
level-2 ICP normal equations (bit-exact: the oracle sums in the reference's
order), the reference's 4-frame loop (poses within 1e-4 m / rad, level
statuses equal), the mesh's vertex set and triangle count, and a sparse
band-integrated store's allocation set and voxels."""

import numpy as np

import golden_common as gc
import kf_oracle as ko
from kinectfusion_b200 import abi


def test_oracle_matches_reference_golden():
    g, seq = gc.load()
    pyr = ko.pyramid(seq.depth[3], gc.K640, ko.depth_options())
    gc.check_pyramid(g, pyr[0]["depth"], pyr[2]["vertices"], pyr[2]["normals"])
    vol = ko.OracleVolume(gc.RES, gc.VOXEL, gc.ORIGIN, gc.TRUNC)
    for f in range(3):
        normals = ko.pyramid(seq.depth[f], gc.K640, ko.depth_options())[0]["normals"]
        w2c = ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[f]))
        ko.integrate(vol, seq.depth[f], gc.K640, w2c, ko.integration_options(), abi.KF_RULE_ANGLE_WEIGHTED,
                     normals_map=normals)
    gc.check_volume(g, vol.voxels)
    k2 = ko.scaled(gc.K640, 2)
    points, normals, _ = ko.raycast(vol, k2, 160, 120, seq.poses[3], ko.raycast_options())
    gc.check_maps(g, points, normals)
    # the normal equations are a function of their inputs: the fixture's own
    camera = abi.rigid_from_matrix(seq.poses[3])
    sums, count = ko.icp_equations(g["pyramid_l2_vertices"], g["pyramid_l2_normals"], g["raycast_points"],
                                   g["raycast_normals"], k2, camera, ko.rigid_inverse(camera))
    assert count == int(g["icp_count"]) > 1000
    assert np.array_equal(np.asarray(sums, np.float32).view(np.uint32), g["icp_sums"].view(np.uint32))
    loop = ko.OracleVolume(gc.RES, gc.VOXEL, gc.ORIGIN, gc.TRUNC)
    pose = np.eye(4, dtype=np.float32)
    poses, statuses = [], []
    for f in range(gc.FRAMES):
        pose, ok, outcomes = ko.track_frame(loop, seq.depth[f], gc.K640, pose, ko.depth_options(),
                                            ko.integration_options(), ko.raycast_options(), ko.icp_options(),
                                            first=(f == 0))
        assert ok
        poses.append(pose)
        statuses.append([outcomes[lv].status if lv in outcomes else abi.KF_ICP_NOT_RUN for lv in range(4)])
    gc.check_loop(g, poses, statuses)
    mesh = ko.marching_cubes(vol, 0.0)
    gc.check_mesh(g, mesh["positions"], len(mesh["triangles"]))
    sparse = ko.OracleVolume(gc.SPARSE_RES, gc.SPARSE_VOXEL, gc.SPARSE_ORIGIN, gc.SPARSE_TRUNC,
                             voxel=abi.KF_VOXEL_BF16, sparse=True)
    io = ko.integration_options(mode=abi.KF_INTEGRATION_BAND)
    for f in range(3):
        normals = ko.pyramid(seq.depth[f], gc.K640, ko.depth_options())[0]["normals"]
        ko.integrate(sparse, seq.depth[f], gc.K640, ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[f])), io,
                     abi.KF_RULE_ANGLE_WEIGHTED, normals_map=normals)
    pool = sparse.voxels.reshape(-1, 512)
    gc.check_sparse(g, sparse.grid, lambda blocks: pool[sparse.grid[blocks]])
