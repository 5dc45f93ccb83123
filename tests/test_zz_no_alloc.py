"""The allocation-free ICP sweep, kf_icp_normal_equations_static.

Callers that cannot allocate device memory (plug-ins whose host owns the
GPU's memory through its own pool, hosts that forbid cudaMalloc after
start-up, real-time loops kept off the allocator because it can stall the
device) use this entry point: its scratch is a fixed device array instead of
a tracker's buffers.  It must
give the same normal equations as the allocating entry point,
kf_icp_normal_equations, call after call.  This file sorts last so that a run
stopping at the first failure has already run every other test.
"""

import ctypes as C

import numpy as np
import pytest

import kinectfusion_b200 as kf
from kinectfusion_b200 import abi, synthetic

pytestmark = pytest.mark.gpu

K640 = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)


def _device_copy(a):
    import torch  # device memory plumbing only
    t = torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1)).cuda()
    torch.cuda.synchronize()
    return t


@pytest.fixture(scope="module")
def scene():
    seq = synthetic.make_sequence(seed=11, frames=3)
    half = 0.5 * 128 * 0.02
    pipe = kf.Pipeline(kf.pipeline_config(128, 0.02, (-half, -half, -0.5), 0.05, color=abi.KF_COLOR_NONE))
    for f in range(2):
        pipe.integrate(seq.depth[f], K640, np.linalg.inv(seq.poses[f]))
    pyr = kf.PyramidSource()
    pyr.build(seq.depth[2], K640)
    return seq, pipe, pyr


def _sweeps(scene, level):
    seq, pipe, pyr = scene
    lib = abi.load()
    k = abi.Intrinsics(K640.fx / 2 ** level, K640.fy / 2 ** level, K640.cx / 2 ** level, K640.cy / 2 ** level)
    w, h = 640 >> level, 480 >> level
    maps = pipe.raycast(k, w, h, seq.poses[1])
    points, normals = _device_copy(maps.points), _device_copy(maps.normals)
    live = pyr.level(level)
    camera = abi.rigid_from_matrix(seq.poses[1])
    model = abi.rigid_from_matrix(np.linalg.inv(seq.poses[1]))
    tracker = kf.ProjectiveIcpTracker()
    opts = tracker.options
    ref_sums = np.zeros(29, dtype=np.float32)
    ref_count = C.c_uint64()
    abi.check(lib.kf_icp_normal_equations(tracker.handle, C.byref(live), C.c_void_p(points.data_ptr()),
                                          C.c_void_p(normals.data_ptr()), w, h, k, C.byref(camera),
                                          C.byref(model), ref_sums.ctypes.data_as(C.c_void_p), C.byref(ref_count)))
    results = []
    for _ in range(2):  # two calls in a row share the static scratch
        sums = np.zeros(29, dtype=np.float32)
        count = C.c_uint64()
        abi.check(lib.kf_icp_normal_equations_static(C.byref(live), C.c_void_p(points.data_ptr()),
                                                     C.c_void_p(normals.data_ptr()), w, h, k, C.byref(camera),
                                                     C.byref(model), opts.max_point_distance, opts.min_normal_dot,
                                                     sums.ctypes.data_as(C.c_void_p), C.byref(count)))
        results.append((sums, count.value))
    return ref_sums, ref_count.value, results


@pytest.mark.parametrize("level", [0, 1, 2])
def test_static_sweep_matches_allocating_sweep(scene, level):
    ref_sums, ref_count, results = _sweeps(scene, level)
    assert ref_count > 100
    scale = np.abs(ref_sums).max()
    for sums, count in results:
        assert count == ref_count
        # both are FP32 sums in different orders; the tests' relative bound
        assert np.abs(sums - ref_sums).max() <= 1e-4 * scale
    # the shared scratch keeps no state between calls: identical inputs, identical sums
    assert np.array_equal(results[0][0], results[1][0])


def test_static_sweep_rejects_oversized_images():
    import torch  # device memory plumbing only
    lib = abi.load()
    # One pixel past the limit, with real device maps of that size (zeros: no
    # pixel would match), so the call stays in bounds even if it launched.
    w, h = 1228801, 1
    maps = [torch.zeros(w * h * 3, dtype=torch.float32, device="cuda") for _ in range(4)]
    torch.cuda.synchronize()
    big = abi.LevelView(None, C.c_void_p(maps[0].data_ptr()), C.c_void_p(maps[1].data_ptr()), w, h, K640)
    sums = np.zeros(29, dtype=np.float32)
    count = C.c_uint64()
    rigid = abi.rigid_from_matrix(np.eye(4))
    status = lib.kf_icp_normal_equations_static(C.byref(big), C.c_void_p(maps[2].data_ptr()),
                                                C.c_void_p(maps[3].data_ptr()), w, h, K640,
                                                C.byref(rigid), C.byref(rigid), 0.05, 0.9,
                                                sums.ctypes.data_as(C.c_void_p), C.byref(count))
    assert status == abi.KF_ERR_INVALID_ARGUMENT
    assert b"1228800" in lib.kf_last_error()
