"""The drop-in: the reference's own host code running on this library.

oracle/_ref/libkf_ref_b200.so is the reference's CPU translation units
(compiled from its sources with KINECTFUSION_HAS_CUDA) with its device seams -
Pipeline::create_device, PyramidSource::create_device, DepthUploader::create
and BasicDeviceCorrespondenceSweep - taken by kinectfusion_b200/glue/
b200_backend.cpp over libkf_b200.so, exactly as a maintainer's build of the
reference with this backend would be.  The frame loop is
Reconstruction::process_frame's (reconstruction.cpp:184-277): the reference's
tracker solves each ICP step on the host (or, with --icp-device-solve, hands
the level to the device loop) from normal equations this library's kernels
reduce.

Checked against the reference's own host pipeline (oracle/_ref/libkf_ref.so)
on the same frames: every level's ICP status, poses within 1e-4 m / 1e-4 rad,
and the TSDF within 1e-5 m; and against this library's native frame graph.
Skipped when the libraries were not built."""

import numpy as np
import pytest

import kf_oracle as ko
import kinectfusion_b200 as kf
from kinectfusion_b200 import abi, synthetic

pytestmark = pytest.mark.gpu

kr = pytest.importorskip("kf_ref")
K640 = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
RES, VOXEL, TRUNC = 128, 0.02, 0.05
ORIGIN = (-0.5 * RES * VOXEL, -0.5 * RES * VOXEL, -0.5)


def pose_error(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    dt = np.linalg.norm(a[:3, 3] - b[:3, 3])
    r = a[:3, :3].T @ b[:3, :3]
    skew = np.array([r[2, 1] - r[1, 2], r[0, 2] - r[2, 0], r[1, 0] - r[0, 1]]) / 2
    return dt, np.arctan2(np.linalg.norm(skew), (np.trace(r) - 1) / 2)


@pytest.fixture(scope="module", autouse=True)
def libraries():
    if not (kr.available() and kr.cuda_available("glue")):
        pytest.skip("oracle/_ref/libkf_ref.so or libkf_ref_b200.so not built")


@pytest.mark.parametrize("device_solve", [False, True])
def test_reference_loop_over_glue_matches_reference_host(device_solve):
    seq = synthetic.make_sequence(seed=31, frames=5)
    cfg = kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_NONE, rule=abi.KF_RULE_ANGLE_WEIGHTED)
    glue = kr.RefDevicePipeline(cfg, ko.depth_options(), ko.icp_options(), device_solve=device_solve,
                                backend="glue")
    host = kr.RefPipeline(cfg)
    native = kf.Reconstruction(kf.Pipeline(cfg), K640)
    pose = np.eye(4, dtype=np.float32)
    for f in range(5):
        ok, status = glue.process(seq.depth[f], K640)
        pose, ok_host, status_host = host.track_frame(seq.depth[f], K640, pose, ko.depth_options(), ko.icp_options(),
                                                      first=(f == 0))
        native.process(seq.depth[f])
        assert ok and ok_host
        if not device_solve:  # the device loop vetoes instability itself, the host check follows it
            assert np.array_equal(status, status_host)
        dt, da = pose_error(glue.trajectory[-1], pose)
        assert dt < 1e-4 and da < 1e-4, (f, dt, da)
        dt, da = pose_error(glue.trajectory[-1], native.trajectory[-1])
        assert dt < 1e-4 and da < 1e-4, (f, dt, da)
    # the volumes: this library's integration at the reference loop's poses
    # against the reference's host integration at its own
    v_glue = glue.host_view()
    v_host = host.voxels()
    both = (v_glue[:, 1] > 0) & (v_host[:, 1] > 0)
    assert both.sum() > 50000
    delta_m = np.abs(v_glue[both, 0] - v_host[both, 0]) * TRUNC
    assert np.percentile(delta_m, 99.9) < 1e-5
    assert (delta_m > 1e-5).sum() <= 1e-3 * both.sum()
    assert glue.observed_voxel_count() == int((v_glue[:, 1] > 0).sum())


def test_glue_integrate_and_raycast_match_reference_host():
    """Pipeline::integrate and Pipeline::raycast through the glue on a volume
    both integrate from the same pose."""
    seq = synthetic.make_sequence(seed=32, frames=3)
    cfg = kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_NONE, rule=abi.KF_RULE_CLASSIC)
    glue = kr.RefDevicePipeline(cfg, ko.depth_options(), ko.icp_options(), backend="glue")
    host = kr.RefPipeline(cfg)
    glue.process(seq.depth[0], K640)  # first frame: fused at identity, no tracking
    host.track_frame(seq.depth[0], K640, np.eye(4, dtype=np.float32), ko.depth_options(), ko.icp_options(),
                     first=True)
    v_glue, v_host = glue.host_view(), host.voxels()
    # first frame at the same (identity) pose: bit-exact up to the bilateral's
    # rare exp rounding, which moves a normal only where a depth moved
    assert (v_glue.view(np.uint32) != v_host.view(np.uint32)).any(axis=1).sum() <= 1e-5 * len(v_glue)
    gp, gn, _ = glue.raycast(K640, 640, 480, seq.poses[1])
    hp, hn, _ = host.raycast(K640, 640, 480, seq.poses[1])
    same = np.all((gp == hp) | (np.isnan(gp) & np.isnan(hp)), axis=-1)
    assert np.isfinite(gp[..., 0]).sum() > 0.3 * 640 * 480
    assert same.mean() > 0.9999
