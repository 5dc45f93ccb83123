"""GPU parity: the sm_100a kernels, called through the C ABI, against the CPU
oracle on the same seeded inputs.

Bars (from the reference's parity requirements):
  * pyramid depth, validity masks, vertex and normal maps: bit-exact;
  * TSDF integration on identical inputs: bit-exact raw voxels (float,
    int16, bf16, colour) - the kernels evaluate the host expressions;
  * raycast on identical volumes and cameras: bit-exact maps;
  * ICP normal equations: identical match count, sums within 1e-4 relative
    (FP32 sums in a different order);
  * tracked poses: within 1e-4 m / 1e-4 rad of the oracle's host loop.
"""

import numpy as np
import pytest

import kf_oracle as ko
from fixtures import (DEPTH_1M, DEPTH_1P4M, SYNTH_IMAGE, compare_maps, compare_volumes, flat_depth,
                      synth_intrinsics, synth_volume, SYNTH_ORIGIN, SYNTH_RES, SYNTH_TRUNC, SYNTH_VOXEL)
from kinectfusion_b200 import abi, synthetic
import kinectfusion_b200 as kf

pytestmark = pytest.mark.gpu

K640 = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)


@pytest.fixture(scope="module")
def seq():
    return synthetic.make_sequence(seed=1, frames=5)


def same_float(a, b):
    """Bitwise-equal up to the sign of zero, NaN positions equal."""
    a = np.asarray(a)
    b = np.asarray(b)
    return a.shape == b.shape and np.array_equal(a, b, equal_nan=True)


def cfg1_geometry():
    # 128^3 x 0.02 m, margin 0.5 (app_options.cpp:33-38)
    half = 0.5 * 128 * 0.02
    return 128, 0.02, (-half, -half, -0.5), 0.05


# ---- pyramid ---------------------------------------------------------------------------
def test_pyramid_bit_exact(seq):
    pyr = kf.PyramidSource()
    o = ko.depth_options()
    for frame in range(2):
        raw = seq.depth[frame]
        assert pyr.build(raw, K640) == 3
        ref = ko.pyramid(raw, K640, o)
        for level in range(3):
            got = pyr.download_level(level)
            assert np.array_equal(got["depth"], ref[level]["depth"]), f"depth level {level}"
            assert same_float(got["vertices"], ref[level]["vertices"]), f"vertices level {level}"
            assert same_float(got["normals"], ref[level]["normals"]), f"normals level {level}"


def test_pyramid_edge_sizes():
    # ragged sizes, all-zero and single-pixel inputs
    pyr = kf.PyramidSource()
    o = ko.depth_options()
    rng = np.random.default_rng(7)
    for h, w in ((1, 1), (5, 7), (33, 65)):
        raw = (rng.integers(2000, 20000, size=(h, w)) * (rng.random((h, w)) > 0.1)).astype(np.uint16)
        n = pyr.build(raw, abi.Intrinsics(50.0, 50.0, w / 2, h / 2))
        ref = ko.pyramid(raw, abi.Intrinsics(50.0, 50.0, w / 2, h / 2), o)
        assert n == len(ref)
        for level in range(n):
            got = pyr.download_level(level)
            assert np.array_equal(got["depth"], ref[level]["depth"])
            assert same_float(got["vertices"], ref[level]["vertices"])
            assert same_float(got["normals"], ref[level]["normals"])
    zeros = np.zeros((48, 64), dtype=np.uint16)
    pyr.build(zeros, abi.Intrinsics(50.0, 50.0, 32, 24))
    assert np.isnan(pyr.download_level(0)["vertices"]).all()


# ---- integration -----------------------------------------------------------------------
@pytest.mark.parametrize("voxel", [abi.KF_VOXEL_FLOAT, abi.KF_VOXEL_QUANTIZED, abi.KF_VOXEL_BF16])
@pytest.mark.parametrize("rule", [abi.KF_RULE_CLASSIC, abi.KF_RULE_ANGLE_WEIGHTED])
def test_integration_bit_exact(seq, voxel, rule):
    res, vs, origin, trunc = cfg1_geometry()
    color = voxel == abi.KF_VOXEL_FLOAT
    cfg = kf.pipeline_config(res, vs, origin, trunc, voxel=voxel, rule=rule,
                             color=abi.KF_COLOR_FLOAT if color else abi.KF_COLOR_NONE)
    gpu = kf.Pipeline(cfg)
    ref = ko.OracleVolume(res, vs, origin, trunc, voxel=voxel, color=color)
    o = ko.integration_options()
    for frame in range(3):
        raw = seq.depth[frame]
        normals = ko.pyramid(raw, K640, ko.depth_options())[0]["normals"]
        w2c = ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[frame]))
        col = seq.color[frame] if color else None
        gpu.integrate(raw, K640, w2c, color=col, normals=normals)
        ko.integrate(ref, raw, K640, w2c, o, rule, color=col, normals_map=normals, threads=8)
    got = gpu.download_raw()
    assert np.array_equal(got.view(np.uint32), ref.voxels.view(np.uint32)), "raw voxels differ"
    assert gpu.observed_voxel_count() == ref.observed_voxel_count() > 0
    if color:
        _, _, gcol = gpu.host_view(with_color=True)
        assert same_float(gcol.reshape(-1, 4), ref.colors)


def test_integration_512_frame_bit_exact(seq):
    """One frame into the headline 512^3 float volume (angle-weighted)."""
    half = 0.5 * 512 * 0.01
    origin = (-half, -half, -0.5)
    cfg = kf.pipeline_config(512, 0.01, origin, 0.05, color=abi.KF_COLOR_NONE)
    gpu = kf.Pipeline(cfg)
    ref = ko.OracleVolume(512, 0.01, origin, 0.05)
    raw = seq.depth[1]
    normals = ko.pyramid(raw, K640, ko.depth_options())[0]["normals"]
    w2c = ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[1]))
    gpu.integrate(raw, K640, w2c, normals=normals)
    ko.integrate(ref, raw, K640, w2c, ko.integration_options(), abi.KF_RULE_ANGLE_WEIGHTED, normals_map=normals,
                 threads=8)
    got = gpu.download_raw()
    assert np.array_equal(got.view(np.uint32), ref.voxels.view(np.uint32))


# ---- raycast -----------------------------------------------------------------------------
def _integrated_pair(seq, frames, voxel=abi.KF_VOXEL_FLOAT, color=True, backend=abi.KF_RAYCAST_MARCH, **opts):
    res, vs, origin, trunc = cfg1_geometry()
    cfg = kf.pipeline_config(res, vs, origin, trunc, voxel=voxel, raycast_backend=backend,
                             color=abi.KF_COLOR_FLOAT if color else abi.KF_COLOR_NONE, **opts)
    gpu = kf.Pipeline(cfg)
    ref = ko.OracleVolume(res, vs, origin, trunc, voxel=voxel, color=color)
    for frame in range(frames):
        raw = seq.depth[frame]
        normals = ko.pyramid(raw, K640, ko.depth_options())[0]["normals"]
        w2c = ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[frame]))
        col = seq.color[frame] if color else None
        gpu.integrate(raw, K640, w2c, color=col, normals=normals)
        ko.integrate(ref, raw, K640, w2c, ko.integration_options(), abi.KF_RULE_ANGLE_WEIGHTED, color=col,
                     normals_map=normals, threads=8)
    return gpu, ref


@pytest.mark.parametrize("voxel,color", [(abi.KF_VOXEL_FLOAT, True), (abi.KF_VOXEL_FLOAT, False),
                                         (abi.KF_VOXEL_QUANTIZED, False), (abi.KF_VOXEL_BF16, False)])
def test_raycast_bit_exact(seq, voxel, color):
    gpu, ref = _integrated_pair(seq, 2, voxel=voxel, color=color)
    for level in (0, 2):
        k = ko.scaled(K640, level)
        w, h = 640 >> level, 480 >> level
        maps = gpu.raycast(k, w, h, seq.poses[2])
        p, n, c = ko.raycast(ref, k, w, h, seq.poses[2], ko.raycast_options(), threads=8)
        assert np.isfinite(p).all(-1).sum() > 0.3 * w * h
        assert same_float(maps.points, p) and same_float(maps.normals, n)
        assert np.array_equal(maps.colors, c)


@pytest.mark.parametrize("opt", ["raycast_cell_gradient_normals", "raycast_corner_policy"])
def test_raycast_ablation_knobs_bit_exact(seq, opt):
    gpu, ref = _integrated_pair(seq, 2, **{opt: 1})
    ro = ko.raycast_options(**{opt.split("_", 1)[1]: 1})
    k = ko.scaled(K640, 1)
    maps = gpu.raycast(k, 320, 240, seq.poses[2])
    p, n, c = ko.raycast(ref, k, 320, 240, seq.poses[2], ro, threads=8)
    assert same_float(maps.points, p) and same_float(maps.normals, n) and np.array_equal(maps.colors, c)


def test_bitmap_march_identical_to_march(seq):
    # tests.cpp:772-801: the skip only removes samples that are nullopt
    # (reference) or exactly 1.0 (here), so every byte matches.
    plain, _ = _integrated_pair(seq, 3)
    skip, _ = _integrated_pair(seq, 3, backend=abi.KF_RAYCAST_BITMAP_MARCH)
    a = plain.raycast(K640, 640, 480, seq.poses[3])
    b = skip.raycast(K640, 640, 480, seq.poses[3])
    assert np.isfinite(a.points).all(-1).sum() > 0
    assert a.points.tobytes() == b.points.tobytes()
    assert a.normals.tobytes() == b.normals.tobytes()
    assert a.colors.tobytes() == b.colors.tobytes()


# ---- ICP ---------------------------------------------------------------------------------
def test_icp_normal_equations_match_oracle(seq):
    gpu, ref = _integrated_pair(seq, 2)
    pyr = kf.PyramidSource()
    pyr.build(seq.depth[2], K640)
    tracker = kf.ProjectiveIcpTracker()
    for level in (0, 1, 2):
        live = pyr.download_level(level)
        lv = pyr.level(level)
        k = ko.scaled(K640, level)
        w, h = 640 >> level, 480 >> level
        model_pose = abi.rigid_from_matrix(seq.poses[1])
        mp, mn, _ = ko.raycast(ref, k, w, h, model_pose, ko.raycast_options(), threads=8)
        camera = abi.rigid_from_matrix(seq.poses[1])
        model = ko.rigid_inverse(model_pose)
        s_ref, c_ref = ko.icp_equations(live["vertices"], live["normals"], mp, mn, k, camera, model)
        s64, _ = ko.icp_equations(live["vertices"], live["normals"], mp, mn, k, camera, model, f64=True)
        # device sweep over the same model maps (uploaded by a device raycast of the identical volume)
        maps = gpu.raycast(k, w, h, model_pose)
        assert same_float(maps.points, mp)
        import ctypes as C
        d_points = _to_device(maps.points)
        d_normals = _to_device(maps.normals)
        sums = np.zeros(29, dtype=np.float32)
        count = C.c_uint64()
        abi.check(abi.load().kf_icp_normal_equations(tracker.handle, C.byref(lv), d_points.ptr, d_normals.ptr, w, h,
                                                      k, C.byref(camera), C.byref(model),
                                                      sums.ctypes.data_as(C.c_void_p), C.byref(count)))
        assert count.value == c_ref > 1000
        scale = np.abs(s64).max()
        # deterministic FP32 tree + Kahan combine vs sequential FP32: both near FP64
        assert np.abs(sums - s64).max() <= 1e-4 * scale
        assert np.abs(s_ref - s64).max() <= 1e-3 * scale


class _DeviceBuffer:
    def __init__(self, nbytes):
        import ctypes as C
        import torch  # device memory plumbing only
        self.t = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        self.ptr = C.c_void_p(self.t.data_ptr())


def _to_device(a):
    import torch
    buf = _DeviceBuffer(a.nbytes)
    buf.t.copy_(torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1)))
    torch.cuda.synchronize()
    return buf


def pose_error(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    dt = np.linalg.norm(a[:3, 3] - b[:3, 3])
    r = a[:3, :3].T @ b[:3, :3]
    # atan2 form: arccos of the trace has a sqrt(eps) floor near identity
    skew = np.array([r[2, 1] - r[1, 2], r[0, 2] - r[2, 0], r[1, 0] - r[0, 1]]) / 2
    ang = np.arctan2(np.linalg.norm(skew), (np.trace(r) - 1) / 2)
    return dt, ang


def test_track_level_matches_oracle(seq):
    gpu, ref = _integrated_pair(seq, 2)
    pyr = kf.PyramidSource()
    pyr.build(seq.depth[2], K640)
    tracker = kf.ProjectiveIcpTracker()
    start = seq.poses[1]
    for level, iters in ((2, 4), (1, 5), (0, 10)):
        k = ko.scaled(K640, level)
        w, h = 640 >> level, 480 >> level
        out = gpu.track(tracker, k, w, h, start, pyr.level(level), iters)
        live = pyr.download_level(level)
        mp, mn, _ = ko.raycast(ref, k, w, h, start, ko.raycast_options(), threads=8)
        ro = ko.icp_estimate(live["vertices"], live["normals"], mp, mn, k, start, start, iters, ko.icp_options())
        succeeded = (abi.KF_ICP_MAX_ITERATIONS, abi.KF_ICP_CONVERGED)
        assert out.status in succeeded and ro.status in succeeded
        assert out.correspondences > 0
        dt, da = pose_error(abi.matrix_from_rigid(out.pose), abi.matrix_from_rigid(ro.pose))
        assert dt < 1e-4 and da < 1e-4, (level, dt, da)


# ---- whole frames --------------------------------------------------------------------------
def test_cfg1_sequence_poses_and_volume(seq):
    """Config 1: 5 frames, 128^3 float, classic TSDF, ICP [10, 5, 4]."""
    res, vs, origin, trunc = cfg1_geometry()
    cfg = kf.pipeline_config(res, vs, origin, trunc, rule=abi.KF_RULE_CLASSIC)
    gpu = kf.Pipeline(cfg)
    loop = kf.Reconstruction(gpu, K640)
    ref = ko.OracleVolume(res, vs, origin, trunc, color=True)
    replay = ko.OracleVolume(res, vs, origin, trunc, color=True)
    pose = np.eye(4, dtype=np.float32)
    opts = dict(depth_opts=ko.depth_options(), integ_opts=ko.integration_options(), ray_opts=ko.raycast_options(),
                icp_opts=ko.icp_options(), rule=abi.KF_RULE_CLASSIC, threads=8)
    for frame in range(5):
        result = loop.process(seq.depth[frame], seq.color[frame])
        pose, ok, _ = ko.track_frame(ref, seq.depth[frame], K640, pose, color=seq.color[frame], first=frame == 0,
                                     **opts)
        assert bool(result.tracked) == ok
        dt, da = pose_error(loop.trajectory[-1], pose)
        assert dt < 1e-4 and da < 1e-4, (frame, dt, da)
        # replay the GPU's own pose on the oracle: integration must match bit for bit
        normals = ko.pyramid(seq.depth[frame], K640, ko.depth_options())[0]["normals"]
        if result.tracked:
            ko.integrate(replay, seq.depth[frame], K640, result.world_to_camera, ko.integration_options(),
                         abi.KF_RULE_CLASSIC, color=seq.color[frame], normals_map=normals, threads=8)
    # the raw voxels and colours equal the oracle's replayed at the poses the
    # frame graph integrated at
    assert np.array_equal(gpu.download_raw().view(np.uint32), replay.voxels.view(np.uint32))
    tsdf, weight = gpu.host_view()
    # and against the oracle's independently tracked volume (poses within 1e-4)
    d2 = compare_volumes((tsdf, weight), ref.dense())
    assert d2["compared"] > 0.99 * (weight > 0).sum()


# ---- reference unit tests through the device path -------------------------------------------
def test_factory_rejects_misconfiguration():
    # tests.cpp:560-581, pipeline.cpp:104-147
    with pytest.raises(ValueError):
        kf.Pipeline(kf.pipeline_config(SYNTH_RES, SYNTH_VOXEL, SYNTH_ORIGIN, SYNTH_TRUNC), name="")
    with pytest.raises(ValueError):
        kf.Pipeline(kf.pipeline_config(SYNTH_RES, -1.0, SYNTH_ORIGIN, SYNTH_TRUNC))
    with pytest.raises(ValueError):
        kf.Pipeline(kf.pipeline_config(SYNTH_RES, SYNTH_VOXEL, SYNTH_ORIGIN, SYNTH_TRUNC,
                                       storage=abi.KF_STORAGE_SPARSE))


def test_device_plane_matches_oracle_fixture():
    # tests.cpp:454-474 and 583-610 (factory == direct host integration exactly)
    cfg = kf.pipeline_config(SYNTH_RES, SYNTH_VOXEL, SYNTH_ORIGIN, SYNTH_TRUNC)
    gpu = kf.Pipeline(cfg)
    gpu.integrate(flat_depth(DEPTH_1M), synth_intrinsics(), np.eye(4))
    ref = synth_volume(color=True)
    ko.integrate(ref, flat_depth(DEPTH_1M), synth_intrinsics(), np.eye(4), ko.integration_options())
    assert gpu.observed_voxel_count() == ref.observed_voxel_count() > 0
    d = compare_volumes(gpu.host_view(), ref.dense())
    assert d["max_distance_delta"] == 0.0 and d["max_weight_delta"] == 0.0
    maps = gpu.raycast(synth_intrinsics(), SYNTH_IMAGE, SYNTH_IMAGE, np.eye(4))
    assert compare_maps(maps.points, maps.normals, maps.points, maps.normals)["compared"] > 0


# ---- marching cubes ----------------------------------------------------------------------
def _same_mesh(a, b):
    assert a["positions"].shape == b["positions"].shape and a["triangles"].shape == b["triangles"].shape
    for key in ("positions", "normals", "colors"):
        assert a[key].tobytes() == b[key].tobytes(), key
    assert np.array_equal(a["triangles"], b["triangles"])


@pytest.mark.parametrize("voxel,color,min_weight", [(abi.KF_VOXEL_FLOAT, True, 0.0), (abi.KF_VOXEL_FLOAT, False, 2.0),
                                                    (abi.KF_VOXEL_QUANTIZED, False, 0.0),
                                                    (abi.KF_VOXEL_BF16, True, 1.0)])
def test_mesh_identical_to_oracle(seq, voxel, color, min_weight):
    # MarchingCubes::extract (marching_cubes.cpp:461-485): same cells, welded
    # vertices in first-use order, same positions, normals and colours
    gpu, ref = _integrated_pair(seq, 3, voxel=voxel, color=color)
    got = gpu.extract_mesh(min_weight)
    want = ko.marching_cubes(ref, min_weight)
    assert len(want["triangles"]) > 1000
    _same_mesh(got, want)


def test_mesh_of_unobserved_volume_is_empty():
    # tests.cpp:402-407
    res, vs, origin, trunc = cfg1_geometry()
    gpu = kf.Pipeline(kf.pipeline_config(res, vs, origin, trunc))
    mesh = gpu.extract_mesh()
    assert len(mesh["positions"]) == 0 and len(mesh["triangles"]) == 0


def test_mesh_weight_threshold_and_closed_edges(seq):
    # tests.cpp:439-452 plus the welded-edge property of tests.cpp:368-384:
    # inside the volume every mesh edge has at most two triangles
    from fixtures import mesh_edge_uses
    gpu, _ = _integrated_pair(seq, 1, color=False)
    assert len(gpu.extract_mesh(1e9)["triangles"]) == 0
    mesh = gpu.extract_mesh(0.0)
    assert len(mesh["triangles"]) > 0
    assert max(mesh_edge_uses(mesh["triangles"]).values()) <= 2


# ---- band integration ----------------------------------------------------------------------
@pytest.mark.parametrize("voxel,color", [(abi.KF_VOXEL_FLOAT, True), (abi.KF_VOXEL_BF16, False)])
def test_band_integration_bit_exact(seq, voxel, color):
    # BandIntegrationSweep<kDevice> (tsdf_integration.cu:240-291): the band
    # walk at half-block steps, then the marked blocks fused like the sweep
    res, vs, origin, trunc = cfg1_geometry()
    cfg = kf.pipeline_config(res, vs, origin, trunc, voxel=voxel, integration_mode=abi.KF_INTEGRATION_BAND,
                             color=abi.KF_COLOR_FLOAT if color else abi.KF_COLOR_NONE)
    gpu = kf.Pipeline(cfg)
    ref = ko.OracleVolume(res, vs, origin, trunc, voxel=voxel, color=color)
    full = ko.OracleVolume(res, vs, origin, trunc, voxel=voxel, color=color)
    o = ko.integration_options(mode=abi.KF_INTEGRATION_BAND)
    for frame in range(3):
        raw = seq.depth[frame]
        normals = ko.pyramid(raw, K640, ko.depth_options())[0]["normals"]
        w2c = ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[frame]))
        col = seq.color[frame] if color else None
        gpu.integrate(raw, K640, w2c, color=col, normals=normals)
        ko.integrate(ref, raw, K640, w2c, o, color=col, normals_map=normals, threads=8, band_walk="device")
        ko.integrate(full, raw, K640, w2c, ko.integration_options(), color=col, normals_map=normals, threads=8)
    got = gpu.download_raw()
    assert np.array_equal(got.view(np.uint32), ref.voxels.view(np.uint32)), "raw voxels differ"
    # tests.cpp:698-720: band == full on shared voxels, the full sweep carves more
    d = compare_volumes(gpu.host_view()[:2], full.dense())
    assert d["compared"] > 0 and d["max_distance_delta"] == 0.0 and d["only_primary"] == 0
    assert d["only_reference"] > 0


def test_band_frames_match_oracle(seq):
    # the whole frame loop (kf_frame_process) with band integration
    res, vs, origin, trunc = cfg1_geometry()
    cfg = kf.pipeline_config(res, vs, origin, trunc, integration_mode=abi.KF_INTEGRATION_BAND,
                             rule=abi.KF_RULE_CLASSIC)
    loop = kf.Reconstruction(kf.Pipeline(cfg), K640)
    ref = ko.OracleVolume(res, vs, origin, trunc, color=True)
    pose = np.eye(4, dtype=np.float32)
    opts = dict(depth_opts=ko.depth_options(), integ_opts=ko.integration_options(mode=abi.KF_INTEGRATION_BAND),
                ray_opts=ko.raycast_options(), icp_opts=ko.icp_options(), rule=abi.KF_RULE_CLASSIC, threads=8,
                band_walk="device")
    for frame in range(3):
        result = loop.process(seq.depth[frame], seq.color[frame])
        pose, ok, _ = ko.track_frame(ref, seq.depth[frame], K640, pose, color=seq.color[frame], first=frame == 0,
                                     **opts)
        assert bool(result.tracked) == ok
        dt, da = pose_error(loop.trajectory[-1], pose)
        assert dt < 1e-4 and da < 1e-4, (frame, dt, da)


# ---- sparse storage ------------------------------------------------------------------------
def _sparse_pair(seq, frames, capacity=0, voxel=abi.KF_VOXEL_BF16, color=False):
    res, vs, origin, trunc = cfg1_geometry()
    common = dict(voxel=voxel, integration_mode=abi.KF_INTEGRATION_BAND,
                  color=abi.KF_COLOR_FLOAT if color else abi.KF_COLOR_NONE)
    sparse = kf.Pipeline(kf.pipeline_config(res, vs, origin, trunc, storage=abi.KF_STORAGE_SPARSE,
                                            sparse_block_capacity=capacity, **common))
    dense = kf.Pipeline(kf.pipeline_config(res, vs, origin, trunc, **common))
    ref = ko.OracleVolume(res, vs, origin, trunc, voxel=voxel, color=color, sparse=True, capacity=capacity)
    o = ko.integration_options(mode=abi.KF_INTEGRATION_BAND)
    for frame in range(frames):
        raw = seq.depth[frame]
        normals = ko.pyramid(raw, K640, ko.depth_options())[0]["normals"]
        w2c = ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[frame]))
        col = seq.color[frame] if color else None
        for p in (sparse, dense):
            p.integrate(raw, K640, w2c, color=col, normals=normals)
        ko.integrate(ref, raw, K640, w2c, o, color=col, normals_map=normals, threads=8)
    return sparse, dense, ref


@pytest.mark.parametrize("voxel,color", [(abi.KF_VOXEL_BF16, False), (abi.KF_VOXEL_FLOAT, True)])
def test_sparse_matches_dense_band_and_oracle(seq, voxel, color):
    # BlockRep<kDevice>::integrate (block_rep.cu:100-152) vs the oracle's
    # BlockRep<kHost>: the same blocks allocated, the same voxels (slots differ:
    # the device numbers new blocks in block order, the host first come)
    sparse, dense, ref = _sparse_pair(seq, 3, voxel=voxel, color=color)
    grid = sparse.block_grid()
    assert np.array_equal(grid != 0xFFFFFFFF, ref.grid != 0xFFFFFFFF)
    attempts, capacity = sparse.block_stats()
    assert attempts == ref.struct.allocated == (grid != 0xFFFFFFFF).sum() and attempts <= capacity
    assert np.array_equal(sparse.download_raw().view(np.uint32), dense.download_raw().view(np.uint32))
    st, sw = sparse.host_view()
    rt, rw = ref.dense()
    assert same_float(st, rt) and same_float(sw, rw)
    assert sparse.observed_voxel_count() == dense.observed_voxel_count() == ref.observed_voxel_count() > 0


def test_sparse_overflow_drops_updates_only(seq):
    # tests.cpp:747-770: past the capacity, blocks stay unallocated and their
    # updates are dropped; everything that is stored matches the dense band
    sparse, dense, _ = _sparse_pair(seq, 2, capacity=40)
    attempts, capacity = sparse.block_stats()
    assert capacity == 40 and attempts > capacity
    assert (sparse.block_grid() != 0xFFFFFFFF).sum() == 40
    d = compare_volumes(sparse.host_view()[:2], dense.host_view()[:2])
    assert d["max_distance_delta"] == 0.0 and d["only_primary"] == 0 and d["only_reference"] > 0


def test_sparse_raycast_bit_exact(seq):
    sparse, _, ref = _sparse_pair(seq, 3, voxel=abi.KF_VOXEL_FLOAT, color=True)
    for level in (1, 2):
        k = ko.scaled(K640, level)
        w, h = 640 >> level, 480 >> level
        maps = sparse.raycast(k, w, h, seq.poses[3])
        p, n, c = ko.raycast(ref, k, w, h, seq.poses[3], ko.raycast_options(), threads=8)
        assert np.isfinite(p).all(-1).sum() > 0.3 * w * h
        assert same_float(maps.points, p) and same_float(maps.normals, n) and np.array_equal(maps.colors, c)


def test_sparse_frames_match_oracle(seq):
    res, vs, origin, trunc = cfg1_geometry()
    cfg = kf.pipeline_config(res, vs, origin, trunc, storage=abi.KF_STORAGE_SPARSE, voxel=abi.KF_VOXEL_BF16,
                             integration_mode=abi.KF_INTEGRATION_BAND, color=abi.KF_COLOR_NONE)
    loop = kf.Reconstruction(kf.Pipeline(cfg), K640)
    ref = ko.OracleVolume(res, vs, origin, trunc, voxel=abi.KF_VOXEL_BF16, sparse=True)
    pose = np.eye(4, dtype=np.float32)
    opts = dict(depth_opts=ko.depth_options(), integ_opts=ko.integration_options(mode=abi.KF_INTEGRATION_BAND),
                ray_opts=ko.raycast_options(), icp_opts=ko.icp_options(), threads=8)
    for frame in range(3):
        result = loop.process(seq.depth[frame])
        pose, ok, _ = ko.track_frame(ref, seq.depth[frame], K640, pose, first=frame == 0, **opts)
        assert bool(result.tracked) == ok
        dt, da = pose_error(loop.trajectory[-1], pose)
        assert dt < 1e-4 and da < 1e-4, (frame, dt, da)


def test_reset_clears_skip_structures(seq):
    # kf_pipeline_reset: a reset volume raycasts like a fresh one
    gpu, _ = _integrated_pair(seq, 2)
    gpu.reset()
    fresh, _ = _integrated_pair(seq, 0)
    for p in (gpu, fresh):
        p.integrate(seq.depth[3], K640, ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[3])),
                    color=seq.color[3], normals=ko.pyramid(seq.depth[3], K640, ko.depth_options())[0]["normals"])
    a = gpu.raycast(K640, 640, 480, seq.poses[3])
    b = fresh.raycast(K640, 640, 480, seq.poses[3])
    assert a.points.tobytes() == b.points.tobytes() and a.normals.tobytes() == b.normals.tobytes()


def test_sparse_mesh_identical_to_oracle(seq):
    # MarchingCubes::extract over a sparse view (marching_cubes.cpp:475-485):
    # allocated blocks in order; and tests.cpp:409-437: the sparse mesh has
    # the dense band mesh's vertices
    sparse, dense, ref = _sparse_pair(seq, 3, voxel=abi.KF_VOXEL_FLOAT, color=True)
    got = sparse.extract_mesh()
    want = ko.marching_cubes(ref)
    assert len(want["triangles"]) > 1000
    _same_mesh(got, want)
    band = dense.extract_mesh()
    key = lambda p: p[np.lexsort((p[:, 2], p[:, 1], p[:, 0]))]
    assert len(band["triangles"]) == len(got["triangles"])
    assert np.array_equal(key(band["positions"]), key(got["positions"]))


# ---- band march ----------------------------------------------------------------------------
def _band_pair(seq, frames, res, voxel):
    vs = 5.12 / res
    origin = (-2.56, -2.56, -0.5)
    cfg = kf.pipeline_config(res, vs, origin, 0.05, voxel=voxel, color=abi.KF_COLOR_NONE,
                             raycast_backend=abi.KF_RAYCAST_BAND_MARCH)
    gpu = kf.Pipeline(cfg)
    ref = ko.OracleVolume(res, vs, origin, 0.05, voxel=voxel, color=False)
    for frame in range(frames):
        raw = seq.depth[frame]
        normals = ko.pyramid(raw, K640, ko.depth_options())[0]["normals"]
        w2c = ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[frame]))
        gpu.integrate(raw, K640, w2c, normals=normals)
        ko.integrate(ref, raw, K640, w2c, ko.integration_options(), abi.KF_RULE_ANGLE_WEIGHTED,
                     normals_map=normals, threads=8)
    return gpu, ref


@pytest.mark.parametrize("res,voxel", [(128, abi.KF_VOXEL_FLOAT), (256, abi.KF_VOXEL_FLOAT),
                                       (256, abi.KF_VOXEL_QUANTIZED), (256, abi.KF_VOXEL_BF16)])
def test_band_march_bit_exact(seq, res, voxel):
    # 256^3 has 32 z-blocks: the one-word z scan of BandSkip runs; 128^3 has 16
    gpu, ref = _band_pair(seq, 3, res, voxel)
    _, dilated = ko.band_bitmap(ref)
    assert dilated.any() and np.array_equal(gpu.band_bitmap(), dilated)
    for level in (0, 1):
        k = ko.scaled(K640, level)
        w, h = 640 >> level, 480 >> level
        maps = gpu.raycast(k, w, h, seq.poses[3])
        p, n, c = ko.raycast_band(ref, dilated, k, w, h, seq.poses[3], ko.raycast_options(), threads=8)
        assert np.isfinite(p).all(-1).sum() > 0.3 * w * h
        assert same_float(maps.points, p) and same_float(maps.normals, n)
        assert np.array_equal(maps.colors, c)


def test_band_march_frames_track_like_march(seq):
    # the approximate skip moves interpolation endpoints by sub-voxel amounts
    # (empty_space_skip.hpp:219-222): the tracked poses stay within 1 mm
    def run(backend):
        cfg = kf.pipeline_config(256, 0.02, (-2.56, -2.56, -0.5), 0.05, color=abi.KF_COLOR_NONE,
                                 raycast_backend=backend)
        gpu = kf.Pipeline(cfg)
        loop = kf.Reconstruction(gpu, K640)
        for f in range(5):
            loop.process(seq.depth[f])
            assert loop.results[-1].tracked
        return gpu, np.array(loop.trajectory)
    band, tb = run(abi.KF_RAYCAST_BAND_MARCH)
    _, tm = run(abi.KF_RAYCAST_MARCH)
    assert np.abs(tb[:, :3, 3] - tm[:, :3, 3]).max() < 1e-3
    band.reset()
    assert not band.band_bitmap().any()
