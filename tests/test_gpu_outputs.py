"""Outputs written from device data (FrameOutput, src/app/frame_output.cpp:100-213):
the per-frame raycast PNG and point-cloud PLY of a pipeline set written by
SetReconstruction(frame_output=...) from device maps, and mesh.ply from the
device mesher, read back and compared byte for byte with the host writers
fed with the same data computed independently (a fresh render of the final
volume; the CPU oracle's mesh of the same volume)."""

import numpy as np
import pytest

import kf_oracle as ko
import kinectfusion_b200 as kf
from kinectfusion_b200 import abi, synthetic, tum
from kinectfusion_b200.pipeline_set import PipelineSet, SetReconstruction

pytestmark = pytest.mark.gpu

K640 = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
RES, VOXEL, TRUNC = 128, 0.02, 0.05
ORIGIN = (-0.5 * RES * VOXEL, -0.5 * RES * VOXEL, -0.5)


def test_set_reconstruction_writes_device_maps(tmp_path):
    seq = synthetic.make_sequence(seed=21, frames=3)
    members = [kf.Pipeline(kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC), "baseline"),
               kf.Pipeline(kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, voxel=abi.KF_VOXEL_BF16,
                                              color=abi.KF_COLOR_NONE), "bf16")]
    out = tum.FrameOutput(tmp_path / "out", write_raycast_images=True, write_point_clouds=True)
    loop = SetReconstruction(PipelineSet(members, reference="baseline"), K640, frame_output=out)
    for f in range(3):
        results = loop.process(seq.depth[f], seq.color[f])
        assert all(r.tracked for r in results) or f == 0
    out.close()
    root = tmp_path / "out"
    assert sorted(p.name for p in root.glob("frame_*_raycast.png")) == [f"frame_{f:06d}_raycast.png"
                                                                       for f in range(3)]
    assert len(list((root / "bf16").glob("frame_*_raycast_point_cloud.ply"))) == 3
    # the last frame's files against the host writers fed with a fresh render
    # of each member's final volume from the reference's final pose
    pose = abi.matrix_from_rigid(loop.results[0][-1].camera_to_world)
    for member, directory in ((members[0], root), (members[1], root / "bf16")):
        maps = member.raycast(K640, 640, 480, pose)
        assert np.isfinite(maps.points).all(-1).sum() > 0.3 * 640 * 480
        tum.write_color_png(tmp_path / "png.png", maps.colors)
        tum.write_point_cloud_ply(tmp_path / "cloud.ply", maps.points, maps.normals, maps.colors)
        assert (directory / "frame_000002_raycast.png").read_bytes() == (tmp_path / "png.png").read_bytes()
        assert ((directory / "frame_000002_raycast_point_cloud.ply").read_bytes() ==
                (tmp_path / "cloud.ply").read_bytes())
        np.testing.assert_array_equal(tum.read_color_png(directory / "frame_000002_raycast.png"), maps.colors)


def test_mesh_ply_from_device_mesher(tmp_path):
    seq = synthetic.make_sequence(seed=22, frames=3)
    gpu = kf.Pipeline(kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC))
    ref = ko.OracleVolume(RES, VOXEL, ORIGIN, TRUNC, color=True)
    for f in range(3):
        normals = ko.pyramid(seq.depth[f], K640, ko.depth_options())[0]["normals"]
        w2c = ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[f]))
        gpu.integrate(seq.depth[f], K640, w2c, color=seq.color[f], normals=normals)
        ko.integrate(ref, seq.depth[f], K640, w2c, ko.integration_options(), color=seq.color[f],
                     normals_map=normals, threads=8)
    out = tum.FrameOutput(tmp_path / "out")
    out.write_mesh(gpu.extract_mesh(2.0))  # the app's mesh min weight (app_options.hpp:28)
    out.close()
    tum.write_mesh_ply(tmp_path / "oracle.ply", ko.marching_cubes(ref, 2.0))
    written = (tmp_path / "out" / "mesh.ply").read_bytes()
    assert len(written) > 10000
    assert written == (tmp_path / "oracle.ply").read_bytes()
