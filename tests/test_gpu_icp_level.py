"""The whole-level ICP kernel: one cooperative launch per pyramid level runs
the level's Gauss-Newton steps with a grid barrier between each sweep and
its FP64 step (BasicDeviceCorrespondenceSweep::run_loop,
icp_correspondence.cu:397-439, over the sweep of :216-343).

* Its sweep and combine are the one-sweep kernel's: one step of
  kf_icp_level returns the same 29 sums and count, bit for bit, as
  kf_icp_normal_equations at the same camera and model, at every level.
* A level of N steps follows the oracle's ProjectiveIcpTracker loop
  (icp_optimizer.cpp:208-302): same status, poses within 1e-4 m / 1e-4 rad.
* A pipeline declared concurrent runs the same levels as per-step launches
  with bit-identical poses and voxels.
* The barrier's waits are bounded: with the barrier stalled
  (kf_tracker_stall_next_level) the level's waits give up after their time
  limit, the call returns KF_ERR_DEVICE_TIMEOUT, the frame is not fused, and
  the tracker runs normally afterwards.  Nothing faults or hangs.
"""

import ctypes as C

import numpy as np
import pytest

import kf_oracle as ko
import kinectfusion_b200 as kf
from kinectfusion_b200 import abi, synthetic

pytestmark = pytest.mark.gpu

K640 = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
RES, VOXEL, TRUNC = 128, 0.02, 0.05
ORIGIN = (-0.5 * RES * VOXEL, -0.5 * RES * VOXEL, -0.5)


@pytest.fixture(scope="module")
def seq():
    return synthetic.make_sequence(seed=41, frames=4)


def fused(seq, frames):
    gpu = kf.Pipeline(kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_NONE))
    for f in range(frames):
        normals = ko.pyramid(seq.depth[f], K640, ko.depth_options())[0]["normals"]
        gpu.integrate(seq.depth[f], K640, ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[f])), normals=normals)
    return gpu


def device(a):
    import torch  # device memory plumbing only
    t = torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1)).cuda()
    torch.cuda.synchronize()
    return t


def pose_error(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    dt = np.linalg.norm(a[:3, 3] - b[:3, 3])
    r = a[:3, :3].T @ b[:3, :3]
    skew = np.array([r[2, 1] - r[1, 2], r[0, 2] - r[2, 0], r[1, 0] - r[0, 1]]) / 2
    return dt, np.arctan2(np.linalg.norm(skew), (np.trace(r) - 1) / 2)


def test_level_step_equals_single_sweep(seq):
    gpu = fused(seq, 3)
    pyr = kf.PyramidSource()
    pyr.build(seq.depth[3], K640)
    tracker = kf.ProjectiveIcpTracker()
    lib = abi.load()
    model_pose = abi.rigid_from_matrix(seq.poses[2])
    model = ko.rigid_inverse(model_pose)
    for level in (0, 1, 2):
        lv = pyr.level(level)
        w, h = 640 >> level, 480 >> level
        maps = gpu.raycast(lv.intrinsics, w, h, seq.poses[2])
        d_points, d_normals = device(maps.points), device(maps.normals)
        sweep = np.zeros(29, dtype=np.float32)
        count = C.c_uint64()
        abi.check(lib.kf_icp_normal_equations(tracker.handle, C.byref(lv), C.c_void_p(d_points.data_ptr()),
                                              C.c_void_p(d_normals.data_ptr()), w, h, lv.intrinsics,
                                              C.byref(model_pose), C.byref(model), sweep.ctypes.data_as(C.c_void_p),
                                              C.byref(count)))
        step = np.zeros(29, dtype=np.float32)
        out = abi.IcpOutcome()
        abi.check(lib.kf_icp_level(tracker.handle, C.byref(lv), C.c_void_p(d_points.data_ptr()),
                                   C.c_void_p(d_normals.data_ptr()), w, h, lv.intrinsics, C.byref(model),
                                   C.byref(model_pose), 1, C.byref(out), step.ctypes.data_as(C.c_void_p)))
        assert count.value > 1000
        assert out.correspondences == count.value
        assert np.array_equal(step.view(np.uint32), sweep.view(np.uint32)), level


def test_level_loop_matches_oracle(seq):
    gpu = fused(seq, 3)
    pyr = kf.PyramidSource()
    pyr.build(seq.depth[3], K640)
    tracker = kf.ProjectiveIcpTracker()
    lib = abi.load()
    start = abi.rigid_from_matrix(seq.poses[2])
    model = ko.rigid_inverse(start)
    for level, iters in ((2, 4), (1, 5), (0, 10)):
        lv = pyr.level(level)
        w, h = 640 >> level, 480 >> level
        maps = gpu.raycast(lv.intrinsics, w, h, seq.poses[2])
        d_points, d_normals = device(maps.points), device(maps.normals)
        out = abi.IcpOutcome()
        abi.check(lib.kf_icp_level(tracker.handle, C.byref(lv), C.c_void_p(d_points.data_ptr()),
                                   C.c_void_p(d_normals.data_ptr()), w, h, lv.intrinsics, C.byref(model),
                                   C.byref(start), iters, C.byref(out), None))
        live = pyr.download_level(level)
        ro = ko.icp_estimate(live["vertices"], live["normals"], maps.points, maps.normals, lv.intrinsics, start, start,
                             iters, ko.icp_options())
        assert out.status == ro.status, (level, out.status, ro.status)
        assert out.status in (abi.KF_ICP_MAX_ITERATIONS, abi.KF_ICP_CONVERGED)
        dt, da = pose_error(abi.matrix_from_rigid(out.pose), abi.matrix_from_rigid(ro.pose))
        assert dt < 1e-4 and da < 1e-4, (level, dt, da)


def test_stalled_barrier_times_out_and_recovers(seq):
    lib = abi.load()
    gpu = kf.Pipeline(kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_NONE))
    loop = kf.Reconstruction(gpu, K640)
    loop.process(seq.depth[0])
    assert loop.process(seq.depth[1]).tracked
    observed = gpu.observed_voxel_count()
    # the frame path: the first level's waits run out, the frame fails
    abi.check(lib.kf_tracker_stall_next_level(loop.tracker.handle))
    pose = abi.rigid_from_matrix(loop.trajectory[-1])
    result = abi.FrameResult()
    depth = np.ascontiguousarray(seq.depth[2])
    status = lib.kf_frame_process(gpu.handle, loop.pyramid.handle, loop.tracker.handle,
                                  depth.ctypes.data_as(C.c_void_p), None, 640, 480, K640, abi.KF_MEMORY_HOST,
                                  loop.iterations, 0, C.byref(pose), C.byref(result))
    assert status == abi.KF_ERR_DEVICE_TIMEOUT
    assert b"grid-barrier" in lib.kf_last_error()
    assert gpu.observed_voxel_count() == observed  # not fused
    # the barrier was cleared: the same frame tracks from the last good pose
    pose = abi.rigid_from_matrix(loop.trajectory[-1])
    abi.check(lib.kf_frame_process(gpu.handle, loop.pyramid.handle, loop.tracker.handle,
                                   depth.ctypes.data_as(C.c_void_p), None, 640, 480, K640, abi.KF_MEMORY_HOST,
                                   loop.iterations, 0, C.byref(pose), C.byref(result)))
    assert result.tracked
    dt, _ = pose_error(abi.matrix_from_rigid(pose), seq.poses[2])
    assert dt < 5e-3
    # the single-level path reports the same way
    pyr = kf.PyramidSource()
    pyr.build(seq.depth[3], K640)
    tracker = kf.ProjectiveIcpTracker()
    abi.check(lib.kf_tracker_stall_next_level(tracker.handle))
    cam = abi.RaycastCamera(pyr.level(2).intrinsics, 160, 120, abi.rigid_from_matrix(seq.poses[2]))
    out = abi.IcpOutcome()
    status = lib.kf_pipeline_track(gpu.handle, tracker.handle, C.byref(cam), C.byref(pyr.level(2)), 4, C.byref(out))
    assert status == abi.KF_ERR_DEVICE_TIMEOUT
    abi.check(lib.kf_pipeline_track(gpu.handle, tracker.handle, C.byref(cam), C.byref(pyr.level(2)), 4, C.byref(out)))
    assert out.status in (abi.KF_ICP_MAX_ITERATIONS, abi.KF_ICP_CONVERGED)


def test_concurrent_pipeline_is_bit_identical(seq):
    """A pipeline declared concurrent (kf_pipeline_set_concurrent) records the
    ICP levels as per-step launches; the frames give the same poses and
    voxels as the cooperative level kernel."""
    runs = []
    for concurrent in (False, True):
        gpu = kf.Pipeline(kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_NONE))
        gpu.set_concurrent(concurrent)
        loop = kf.Reconstruction(gpu, K640)
        for f in range(4):
            loop.process(seq.depth[f])
        assert all(r.tracked for r in loop.results)
        runs.append((np.array(loop.trajectory), gpu.download_raw().view(np.uint32),
                     [list(r.iterations) for r in loop.results]))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])
    assert runs[0][2] == runs[1][2]
