"""The device against golden outputs of the reference itself
(tests/golden/reference_small.npz, made by tests/golden/make_golden.py from
the reference's host implementation compiled from its own sources).  Needs
neither the reference nor its compiled library on the GPU box: pyramid,
64^3 angle-weighted integration, 160x120 raycast, the level-2 ICP normal
equations (count equal, sums within 1e-4 relative: the device reduces in a
fixed tree order, the reference sequentially), the reference's 4-frame loop
(poses within 1e-4 m / rad, level statuses equal), the mesh's vertex set and
triangle count, and a sparse band-integrated store's allocation set and
voxels (the device's voxel-block hash against BlockRep<kHost>)."""

import ctypes as C

import numpy as np
import pytest

import golden_common as gc
import kf_oracle as ko  # the rigid inverse the fixture's integration used (host arithmetic only)
import kinectfusion_b200 as kf
from kinectfusion_b200 import abi

pytestmark = pytest.mark.gpu


def device(a):
    import torch  # device memory plumbing only
    t = torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1)).cuda()
    torch.cuda.synchronize()
    return t


def test_device_matches_reference_golden():
    g, seq = gc.load()
    pyr = kf.PyramidSource()
    pyr.build(seq.depth[3], gc.K640)
    gc.check_pyramid(g, pyr.download_level(0)["depth"], pyr.download_level(2)["vertices"],
                     pyr.download_level(2)["normals"])
    cfg = kf.pipeline_config(gc.RES, gc.VOXEL, gc.ORIGIN, gc.TRUNC, color=abi.KF_COLOR_NONE,
                             rule=abi.KF_RULE_ANGLE_WEIGHTED)
    gpu = kf.Pipeline(cfg)
    for f in range(3):
        pf = kf.PyramidSource()
        pf.build(seq.depth[f], gc.K640)
        w2c = ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[f]))
        gpu.integrate(seq.depth[f], gc.K640, w2c, normals=pf.download_level(0)["normals"])
    gc.check_volume(g, gpu.download_raw())
    k2 = ko.scaled(gc.K640, 2)
    maps = gpu.raycast(k2, 160, 120, seq.poses[3])
    gc.check_maps(g, maps.points, maps.normals)
    # the normal equations over the fixture's own inputs
    lv, ln = device(g["pyramid_l2_vertices"]), device(g["pyramid_l2_normals"])
    mp, mn = device(g["raycast_points"]), device(g["raycast_normals"])
    live = abi.LevelView(None, C.c_void_p(lv.data_ptr()), C.c_void_p(ln.data_ptr()), 160, 120, k2)
    camera = abi.rigid_from_matrix(seq.poses[3])
    model = ko.rigid_inverse(camera)
    sums, count = np.zeros(29, np.float32), C.c_uint64()
    tracker = kf.ProjectiveIcpTracker()
    abi.check(abi.load().kf_icp_normal_equations(tracker.handle, C.byref(live), C.c_void_p(mp.data_ptr()),
                                                 C.c_void_p(mn.data_ptr()), 160, 120, k2,
                                                 C.byref(camera), C.byref(model), sums.ctypes.data_as(C.c_void_p),
                                                 C.byref(count)))
    assert count.value == int(g["icp_count"])
    ref = g["icp_sums"].astype(np.float64)
    assert np.abs(sums.astype(np.float64) - ref).max() <= 1e-4 * np.abs(ref).max()
    loop = kf.Reconstruction(kf.Pipeline(cfg), gc.K640)
    for f in range(gc.FRAMES):
        assert loop.process(seq.depth[f]).tracked
    statuses = [list(r.status) for r in loop.results]
    gc.check_loop(g, loop.trajectory, statuses)
    mesh = gpu.extract_mesh(0.0)
    gc.check_mesh(g, mesh["positions"], len(mesh["triangles"]))
    scfg = kf.pipeline_config(gc.SPARSE_RES, gc.SPARSE_VOXEL, gc.SPARSE_ORIGIN, gc.SPARSE_TRUNC,
                              voxel=abi.KF_VOXEL_BF16, color=abi.KF_COLOR_NONE, rule=abi.KF_RULE_ANGLE_WEIGHTED,
                              storage=abi.KF_STORAGE_SPARSE, integration_mode=abi.KF_INTEGRATION_BAND)
    sparse = kf.Pipeline(scfg)
    for f in range(3):
        pf = kf.PyramidSource()
        pf.build(seq.depth[f], gc.K640)
        sparse.integrate(seq.depth[f], gc.K640, ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[f])),
                         normals=pf.download_level(0)["normals"])
    grid = sparse.block_grid()
    pool = sparse.download_pool().view(np.uint32).reshape(-1, 512)
    gc.check_sparse(g, grid, lambda blocks: pool[grid[blocks]])
