"""A frame whose tracking fails, through the whole-frame graph, against the
oracle (Reconstruction::process_frame, reconstruction.cpp:184-277): an
all-zero depth frame in the middle of a sequence has too few
correspondences at the coarsest level, the later levels do not run, the
frame is not fused and the pose stays; the next frame tracks from that pose.
Each frame is compared with the oracle tracking the same frame against the
same state (its volume replayed at the device's poses, from the device's
previous pose): flags and level outcomes equal, poses within 1e-4 m / rad,
and the replayed volume equal to the device's bit for bit.  Frames in
flight and a batch member (per-step ICP launches) reproduce the synchronous
run bit for bit."""

import numpy as np
import pytest

import kf_oracle as ko
import kinectfusion_b200 as kf
from kinectfusion_b200 import abi, synthetic

pytestmark = pytest.mark.gpu

K640 = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
RES, VOXEL, TRUNC = 128, 0.02, 0.05
ORIGIN = (-0.5 * RES * VOXEL, -0.5 * RES * VOXEL, -0.5)


def frames():
    seq = synthetic.make_sequence(seed=51, frames=5)
    depth = seq.depth.copy()
    depth[2] = 0  # no valid pixel
    return depth


def pose_error(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    dt = np.linalg.norm(a[:3, 3] - b[:3, 3])
    r = a[:3, :3].T @ b[:3, :3]
    skew = np.array([r[2, 1] - r[1, 2], r[0, 2] - r[2, 0], r[1, 0] - r[0, 1]]) / 2
    return dt, np.arctan2(np.linalg.norm(skew), (np.trace(r) - 1) / 2)


@pytest.fixture(scope="module")
def synchronous():
    depth = frames()
    gpu = kf.Pipeline(kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_NONE))
    loop = kf.Reconstruction(gpu, K640)
    observed = []
    for f in range(len(depth)):
        loop.process(depth[f])
        observed.append(gpu.observed_voxel_count())
    return depth, loop, observed, gpu.download_raw()


def test_failed_frame_against_the_oracle(synchronous):
    depth, loop, observed, raw = synchronous
    replay = ko.OracleVolume(RES, VOXEL, ORIGIN, TRUNC)
    for f in range(len(depth)):
        r = loop.results[f]
        levels = ko.pyramid(depth[f], K640, ko.depth_options())
        if f > 0:
            tracked, ok, outcomes = ko.track(replay, levels, depth[f].shape, loop.trajectory[f - 1],
                                             ko.raycast_options(), ko.icp_options())
            assert bool(r.tracked) == ok, f
            success = (abi.KF_ICP_MAX_ITERATIONS, abi.KF_ICP_CONVERGED)
            for lv, o in outcomes.items():
                # a failure code equal; converged or at the cap can flip
                # where the last update sits at the threshold
                assert r.status[lv] == o.status or (r.status[lv] in success and o.status in success), \
                    (f, lv, r.status[lv], o.status)
            dt, da = pose_error(loop.trajectory[f], tracked if ok else loop.trajectory[f - 1])
            assert dt < 1e-4 and da < 1e-4, (f, dt, da)
        if r.tracked:
            ko.integrate(replay, depth[f], K640, r.world_to_camera, ko.integration_options(),
                         abi.KF_RULE_ANGLE_WEIGHTED, normals_map=levels[0]["normals"])
    assert np.array_equal(raw.view(np.uint32), replay.voxels.view(np.uint32))
    failed = loop.results[2]
    assert not failed.tracked and failed.status[2] == abi.KF_ICP_TOO_FEW_CORRESPONDENCES
    assert failed.status[1] == abi.KF_ICP_NOT_RUN and failed.status[0] == abi.KF_ICP_NOT_RUN
    assert np.array_equal(loop.trajectory[2], loop.trajectory[1]) and observed[2] == observed[1]
    assert loop.results[3].tracked and loop.results[4].tracked


def test_failed_frame_in_flight_and_in_a_batch(synchronous):
    depth, loop, observed, raw = synchronous
    gpu = kf.Pipeline(kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_NONE))
    pipelined = kf.PipelinedReconstruction(gpu, K640)
    for f in range(len(depth)):
        pipelined.submit(depth[f])
    results = [pipelined.next_result() for _ in range(len(depth))]
    for f in range(len(depth)):
        assert results[f].tracked == loop.results[f].tracked, f
        assert np.array_equal(abi.matrix_from_rigid(results[f].camera_to_world), loop.trajectory[f]), f
    assert np.array_equal(gpu.download_raw().view(np.uint32), raw.view(np.uint32))
    import torch  # device memory plumbing only
    member = kf.Pipeline(kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_NONE))
    batch = kf.Batch([member], K640)
    dev = torch.from_numpy(np.ascontiguousarray(depth).view(np.int16)).cuda()
    torch.cuda.synchronize()
    for f in range(len(depth)):
        batch.step([dev.data_ptr() + f * 640 * 480 * 2])
        r = batch.result(0)
        assert r.tracked == loop.results[f].tracked, f
        assert np.array_equal(abi.matrix_from_rigid(r.camera_to_world), loop.trajectory[f]), f
    assert np.array_equal(member.download_raw().view(np.uint32), raw.view(np.uint32))
