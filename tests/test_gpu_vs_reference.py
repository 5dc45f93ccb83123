"""The device pipeline against the reference ITSELF, on the GPU box.

oracle/_ref/libkf_ref.so is the reference's host implementation and
oracle/_ref/libkf_ref_cuda.so the same with its CUDA path, both compiled from
the reference's sources by oracle/ref_build.sh (prebuilt files on the box;
nothing reads the reference's sources at run time).  These tests skip when
the libraries were not built.

* Stage by stage against the reference's host code (cfg1 geometry, identical
  inputs): raw voxels of every storage and the raycast maps are bit-exact.
* The whole cfg2 loop (512^3, 10 frames) against the reference's own CUDA
  pipeline (--space cuda, default switches) on the same GPU: both track every
  frame; the reference's device ICP sums in FP32 with atomicAdd, in an order
  that changes from run to run, and its kernels contract multiply-adds, so
  the poses are compared at a tolerance, against the spread between two runs
  of the reference itself and against ground truth.
"""

import numpy as np
import pytest

import kf_oracle as ko
import kinectfusion_b200 as kf
from kinectfusion_b200 import abi, synthetic

pytestmark = pytest.mark.gpu

kr = pytest.importorskip("kf_ref")
K640 = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)


def pose_error(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    dt = np.linalg.norm(a[:3, 3] - b[:3, 3])
    r = a[:3, :3].T @ b[:3, :3]
    skew = np.array([r[2, 1] - r[1, 2], r[0, 2] - r[2, 0], r[1, 0] - r[0, 1]]) / 2
    return dt, np.arctan2(np.linalg.norm(skew), (np.trace(r) - 1) / 2)


@pytest.fixture(scope="module")
def seq():
    return synthetic.make_sequence(seed=5, frames=4)


@pytest.mark.parametrize("voxel,color", [(abi.KF_VOXEL_FLOAT, True), (abi.KF_VOXEL_QUANTIZED, False),
                                         (abi.KF_VOXEL_BF16, False)])
def test_device_stages_bit_exact_vs_reference_host(seq, voxel, color):
    if not kr.available():
        pytest.skip("oracle/_ref/libkf_ref.so not built")
    res, vs, trunc = 128, 0.02, 0.05
    origin = (-0.5 * res * vs, -0.5 * res * vs, -0.5)
    cfg = kf.pipeline_config(res, vs, origin, trunc, voxel=voxel,
                             color=abi.KF_COLOR_FLOAT if color else abi.KF_COLOR_NONE)
    gpu, ref = kf.Pipeline(cfg), kr.RefPipeline(cfg)
    for f in range(3):
        normals = ko.pyramid(seq.depth[f], K640, ko.depth_options())[0]["normals"]
        w2c = ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[f]))
        col = seq.color[f] if color else None
        gpu.integrate(seq.depth[f], K640, w2c, color=col, normals=normals)
        ref.integrate(seq.depth[f], K640, w2c, color=col, normals=normals)
    assert np.array_equal(gpu.download_raw().view(np.uint32).reshape(-1), ref.voxels().view(np.uint32).reshape(-1))
    assert gpu.observed_voxel_count() == ref.observed_voxel_count()
    for level in (0, 2):
        k = ko.scaled(K640, level)
        w, h = 640 >> level, 480 >> level
        maps = gpu.raycast(k, w, h, seq.poses[3])
        p, n, c = ref.raycast(k, w, h, seq.poses[3])
        assert np.isfinite(p[..., 0]).sum() > 0.2 * w * h
        assert np.array_equal(maps.points, p, equal_nan=True) and np.array_equal(maps.normals, n, equal_nan=True)
        if color:
            assert np.array_equal(maps.colors, c)


def test_cfg2_loop_vs_reference_cuda():
    if not kr.cuda_available():
        pytest.skip("oracle/_ref/libkf_ref_cuda.so not built")
    res, vs, trunc = 512, 0.01, 0.05
    origin = (-0.5 * res * vs, -0.5 * res * vs, -0.5)
    frames = 10
    seq = synthetic.make_sequence(seed=1000, frames=frames)
    cfg = kf.pipeline_config(res, vs, origin, trunc, color=abi.KF_COLOR_NONE, rule=abi.KF_RULE_ANGLE_WEIGHTED)
    ours = kf.Reconstruction(kf.Pipeline(cfg), K640)
    for f in range(frames):
        assert ours.process(seq.depth[f]).tracked or f == 0
    runs = []
    for _ in range(2):
        ref = kr.RefDevicePipeline(cfg, ko.depth_options(), ko.icp_options())
        for f in range(frames):
            ok, _ = ref.process(seq.depth[f], K640)
            assert ok
        runs.append(ref.trajectory)
        del ref
    worst = [0.0, 0.0]
    spread = [0.0, 0.0]
    for f in range(frames):
        dt, da = pose_error(ours.trajectory[f], runs[0][f])
        worst = [max(worst[0], dt), max(worst[1], da)]
        st, sa = pose_error(runs[1][f], runs[0][f])
        spread = [max(spread[0], st), max(spread[1], sa)]
    print(f"ours vs reference CUDA: {worst[0]:.2e} m, {worst[1]:.2e} rad; reference run to run: "
          f"{spread[0]:.2e} m, {spread[1]:.2e} rad")
    assert worst[0] < 5e-4 and worst[1] < 5e-4
    gt = [seq.poses[f] for f in range(frames)]
    err_ours = max(pose_error(ours.trajectory[f], gt[f])[0] for f in range(frames))
    err_ref = max(pose_error(runs[0][f], gt[f])[0] for f in range(frames))
    assert err_ours <= err_ref + 1e-4, (err_ours, err_ref)
