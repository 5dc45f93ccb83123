"""Batches of independent sequences (kf_batch_*): one graph launch per step
runs every member's frame; the results are those of the members run alone."""

import ctypes as C

import numpy as np
import pytest

import kinectfusion_b200 as kf
from kinectfusion_b200 import abi, synthetic

pytestmark = pytest.mark.gpu

K640 = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
MEMBERS = [(64, 0.04, abi.KF_VOXEL_QUANTIZED), (96, 0.03, abi.KF_VOXEL_BF16), (128, 0.02, abi.KF_VOXEL_QUANTIZED)]


def _config(res, vs, voxel):
    half = 0.5 * res * vs
    return kf.pipeline_config(res, vs, (-half, -half, -0.5), 0.05, voxel=voxel, color=abi.KF_COLOR_NONE)


def test_batch_matches_members_run_alone():
    import torch  # device memory plumbing only
    seqs = [synthetic.make_sequence(seed=40 + i, frames=4) for i in range(len(MEMBERS))]
    frames = [torch.from_numpy(s.depth.view(np.int16)).cuda() for s in seqs]
    torch.cuda.synchronize()
    batch = kf.Batch([kf.Pipeline(_config(*m)) for m in MEMBERS], K640)
    poses = [[] for _ in MEMBERS]
    for f in range(4):
        # member 1 sits out step 2 and catches up at the end
        ptrs = [frames[i][f].data_ptr() if not (i == 1 and f == 2) else None for i in range(len(MEMBERS))]
        batch.step(ptrs)
        for i, p in enumerate(ptrs):
            if p is not None:
                poses[i].append(abi.matrix_from_rigid(batch.result(i).camera_to_world))
    batch.step([None, frames[1][2].data_ptr(), None])
    poses[1].insert(2, abi.matrix_from_rigid(batch.result(1).camera_to_world))
    assert batch.kernel_count() > 0
    for i, m in enumerate(MEMBERS):
        alone = kf.Reconstruction(kf.Pipeline(_config(*m)), K640)
        order = [0, 1, 2, 3] if i != 1 else [0, 1, 3, 2]
        got = {}
        for f in order:
            alone.process(seqs[i].depth[f])
            got[f] = alone.trajectory[-1]
        for f in range(4):
            assert np.array_equal(np.asarray(got[f], dtype=np.float32), np.asarray(poses[i][f], dtype=np.float32)), (i, f)
        assert np.array_equal(alone.pipeline.download_raw(), batch.pipelines[i].download_raw()), i


def test_autotuned_shapes_change_no_bit():
    # kf_pipeline_autotune: the tuned launch shapes give the same poses and
    # volume as the defaults
    import torch
    seq = synthetic.make_sequence(seed=50, frames=5)
    frames = torch.from_numpy(seq.depth.view(np.int16)).cuda()
    torch.cuda.synchronize()
    tuned = kf.Pipeline(_config(128, 0.02, abi.KF_VOXEL_BF16))
    shapes, ms = tuned.autotune(frames.data_ptr(), 4, K640)
    assert shapes.raycast_block_x * shapes.raycast_block_y <= 64 and shapes.integrate_ctas > 0 and ms > 0
    odd = kf.Pipeline(_config(128, 0.02, abi.KF_VOXEL_BF16))
    odd.set_launch_shapes((32, 2), 148 * 4, raycast_lanes=(4, 2, 1))
    odd2 = kf.Pipeline(_config(128, 0.02, abi.KF_VOXEL_BF16))
    odd2.set_launch_shapes((8, 8), 148 * 12, raycast_lanes=(2, 4, 4))
    plain = kf.Pipeline(_config(128, 0.02, abi.KF_VOXEL_BF16))
    plain.set_launch_shapes((8, 8), 148 * 12, raycast_lanes=(1, 1, 1))
    loops = [kf.Reconstruction(p, K640) for p in (tuned, odd, odd2, plain)]
    for f in range(5):
        for loop in loops:
            loop.process(seq.depth[f])
    # the renders themselves, at every size class
    for size in ((160, 120), (320, 240), (640, 480)):
        k = abi.Intrinsics(K640.fx * size[0] / 640, K640.fy * size[0] / 640,
                           (K640.cx + 0.5) * size[0] / 640 - 0.5, (K640.cy + 0.5) * size[0] / 640 - 0.5)
        ref = plain.raycast(k, size[0], size[1], seq.poses[4])
        for p in (odd, odd2):
            got = p.raycast(k, size[0], size[1], seq.poses[4])
            assert got.points.tobytes() == ref.points.tobytes() and got.normals.tobytes() == ref.normals.tobytes()
    for loop in loops[:3]:
        assert all(np.array_equal(a, b) for a, b in zip(loop.trajectory, loops[3].trajectory))
        assert np.array_equal(loop.pipeline.download_raw(), plain.download_raw())
