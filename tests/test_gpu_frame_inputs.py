"""Host inputs of kf_frame_process: page-locked buffers are copied to the
device straight from the caller's memory, pageable ones through the
pipeline's pinned staging; both give bit-identical frames."""

import numpy as np
import pytest

import kinectfusion_b200 as kf
from kinectfusion_b200 import abi, synthetic

pytestmark = pytest.mark.gpu

K640 = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)


def test_page_locked_and_pageable_inputs_match():
    import torch  # pinned host memory
    seq = synthetic.make_sequence(seed=7, frames=4)
    depth_pinned = torch.from_numpy(seq.depth.view(np.int16)).pin_memory().numpy().view(np.uint16)
    color_pinned = torch.from_numpy(seq.color.view(np.int32)).pin_memory().numpy().view(np.uint32)
    half = 0.5 * 128 * 0.02
    cfg = kf.pipeline_config(128, 0.02, (-half, -half, -0.5), 0.05)
    pageable = kf.Reconstruction(kf.Pipeline(cfg), K640)
    pinned = kf.Reconstruction(kf.Pipeline(cfg), K640)
    mixed = kf.Reconstruction(kf.Pipeline(cfg), K640)
    for f in range(4):
        pageable.process(seq.depth[f].copy(), seq.color[f].copy())
        pinned.process(depth_pinned[f], color_pinned[f])
        mixed.process(depth_pinned[f], seq.color[f].copy())
    for other in (pinned, mixed):
        assert all(np.array_equal(a, b) for a, b in zip(pageable.trajectory, other.trajectory))
        assert np.array_equal(pageable.pipeline.download_raw(), other.pipeline.download_raw())
        _, _, ca = pageable.pipeline.host_view(with_color=True)
        _, _, cb = other.pipeline.host_view(with_color=True)
        assert np.array_equal(ca, cb)
    assert all(r.tracked for r in pinned.results)


def _cfg1(**kw):
    half = 0.5 * 128 * 0.02
    return kf.pipeline_config(128, 0.02, (-half, -half, -0.5), 0.05, color=abi.KF_COLOR_NONE, **kw)


def test_frames_in_flight_match_one_at_a_time():
    import ctypes as C
    from kinectfusion_b200.pipeline import _check, _ptr, lib
    seq = synthetic.make_sequence(seed=8, frames=8)
    piped = kf.PipelinedReconstruction(kf.Pipeline(_cfg1()), K640)
    for f in range(8):
        piped.submit(seq.depth[f])  # up to three frames ahead of the results read
        if f >= 2:
            piped.next_result()
    while len(piped.results) < 8:
        piped.next_result()
    # the same frames through kf_frame_enqueue, each result read before the next
    pipe, pyr, tracker = kf.Pipeline(_cfg1()), kf.PyramidSource(), kf.ProjectiveIcpTracker()
    iters = (C.c_uint32 * 4)(*kf.ICP_ITERATIONS)
    one_at_a_time = []
    for f in range(8):
        d = np.ascontiguousarray(seq.depth[f])
        _check(lib().kf_frame_enqueue(pipe.handle, pyr.handle, tracker.handle, _ptr(d), None, 640, 480, K640,
                                      abi.KF_MEMORY_HOST, iters, 1 if f == 0 else 0))
        r = abi.FrameResult()
        _check(lib().kf_frame_result_fetch(pipe.handle, C.byref(r)))
        one_at_a_time.append(abi.matrix_from_rigid(r.camera_to_world))
    assert all(np.array_equal(a, b) for a, b in zip(piped.trajectory, one_at_a_time))
    assert np.array_equal(piped.pipeline.download_raw(), pipe.download_raw())
    assert piped.results[0].status[0] == abi.KF_ICP_NOT_RUN and all(r.tracked for r in piped.results)
    # the host-synchronous loop rounds the pose to float between frames
    sync = kf.Reconstruction(kf.Pipeline(_cfg1()), K640)
    for f in range(8):
        sync.process(seq.depth[f])
    assert max(np.abs(a - b).max() for a, b in zip(sync.trajectory, piped.trajectory)) < 1e-4


def test_frames_in_flight_queue_limits():
    seq = synthetic.make_sequence(seed=9, frames=2)
    piped = kf.PipelinedReconstruction(kf.Pipeline(_cfg1()), K640)
    with pytest.raises(ValueError, match="no submitted frame"):
        piped.next_result()
    for f in range(piped.RESULTS_IN_FLIGHT):
        piped.submit(seq.depth[f % 2])
    with pytest.raises(ValueError, match="eight results"):
        piped.submit(seq.depth[0])
    for _ in range(piped.RESULTS_IN_FLIGHT):
        piped.next_result()
    piped.submit(seq.depth[1])
    assert piped.next_result() is not None and len(piped.results) == piped.RESULTS_IN_FLIGHT + 1
