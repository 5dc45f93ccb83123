"""GPU parity of the ablation knobs off the default path: the reference's
--distance-scaled-truncation and --no-projective-tsdf-distance (integration,
full sweep and band), --raycast-seed-previous (raycast) and the
Levenberg-Marquardt damping modes of the tracker, each against the oracle on
the same inputs.  Bars as in test_gpu_parity: raw voxels and maps
bit-exact, tracked poses within 1e-4 m / 1e-4 rad."""

import numpy as np
import pytest

import kf_oracle as ko
import kinectfusion_b200 as kf
from kinectfusion_b200 import abi, synthetic
from test_gpu_parity import K640, _integrated_pair, cfg1_geometry, pose_error, same_float

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def seq():
    return synthetic.make_sequence(seed=3, frames=5)


@pytest.mark.parametrize("mode", [abi.KF_INTEGRATION_FULL, abi.KF_INTEGRATION_BAND])
@pytest.mark.parametrize("knob", [{"distance_scaled_truncation": 1}, {"projective_distance": 0}])
def test_integration_knobs_bit_exact(seq, mode, knob):
    # tsdf_integration.hpp:43-49 (truncation grows with the measured depth),
    # :207-210 (sdf along the optical axis instead of the ray)
    res, vs, origin, trunc = cfg1_geometry()
    cfg = kf.pipeline_config(res, vs, origin, trunc, color=abi.KF_COLOR_NONE, integration_mode=mode,
                             **{"integration_" + k: v for k, v in knob.items()})
    gpu = kf.Pipeline(cfg)
    ref = ko.OracleVolume(res, vs, origin, trunc)
    o = ko.integration_options(mode=mode, **knob)
    for frame in range(3):
        raw = seq.depth[frame]
        normals = ko.pyramid(raw, K640, ko.depth_options())[0]["normals"]
        w2c = ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[frame]))
        gpu.integrate(raw, K640, w2c, normals=normals)
        # the device band walk steps half a block (BandIntegrationSweep<kDevice>)
        ko.integrate(ref, raw, K640, w2c, o, abi.KF_RULE_ANGLE_WEIGHTED, normals_map=normals, threads=8,
                     band_walk="device")
    assert np.array_equal(gpu.download_raw().view(np.uint32), ref.voxels.view(np.uint32))
    assert gpu.observed_voxel_count() == ref.observed_voxel_count() > 0


def test_raycast_seed_previous_bit_exact(seq):
    # raycasting.hpp:121-133: each ray starts at the previous render's point
    # of its pixel (when finite and in range) instead of the near plane
    gpu, ref = _integrated_pair(seq, 3, color=False, raycast_seed_from_previous=1)
    ro = ko.raycast_options(seed_from_previous=1)
    k = ko.scaled(K640, 1)
    first = gpu.raycast(k, 320, 240, seq.poses[2])
    p0, n0, _ = ko.raycast(ref, k, 320, 240, seq.poses[2], ro, threads=8)
    assert same_float(first.points, p0) and same_float(first.normals, n0)
    second = gpu.raycast(k, 320, 240, seq.poses[3], seed_points=first.points)
    p1, n1, c1 = ko.raycast(ref, k, 320, 240, seq.poses[3], ro, threads=8, seed_points=p0)
    assert np.isfinite(p1).all(-1).sum() > 0.3 * 320 * 240
    assert same_float(second.points, p1) and same_float(second.normals, n1)
    assert np.array_equal(second.colors, c1)


@pytest.mark.parametrize("damping", [dict(damping_mode=abi.KF_DAMPING_IDENTITY, damping_lambda=1e-3),
                                     dict(damping_mode=abi.KF_DAMPING_DIAGONAL, damping_lambda=1e-2),
                                     dict(damping_mode=abi.KF_DAMPING_DIAGONAL, damping_lambda=1e-3,
                                          adaptive_damping=1)])
def test_track_damping_modes_match_oracle(seq, damping):
    # icp_correspondence.hpp:56-98: damped normal equations, adaptive lambda
    gpu, ref = _integrated_pair(seq, 2, color=False)
    pyr = kf.PyramidSource()
    pyr.build(seq.depth[2], K640)
    tracker = kf.ProjectiveIcpTracker(kf.default_icp_options(**damping))
    start = seq.poses[1]
    for level, iters in ((2, 4), (1, 5), (0, 10)):
        k = ko.scaled(K640, level)
        w, h = 640 >> level, 480 >> level
        out = gpu.track(tracker, k, w, h, start, pyr.level(level), iters)
        live = pyr.download_level(level)
        mp, mn, _ = ko.raycast(ref, k, w, h, start, ko.raycast_options(), threads=8)
        ro = ko.icp_estimate(live["vertices"], live["normals"], mp, mn, k, start, start, iters,
                             ko.icp_options(**damping))
        succeeded = (abi.KF_ICP_MAX_ITERATIONS, abi.KF_ICP_CONVERGED)
        assert out.status in succeeded and ro.status in succeeded
        assert out.rejected_steps == ro.rejected_steps
        dt, da = pose_error(abi.matrix_from_rigid(out.pose), abi.matrix_from_rigid(ro.pose))
        assert dt < 1e-4 and da < 1e-4, (level, dt, da)
