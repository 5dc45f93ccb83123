"""Frames replayed from a TUM RGB-D directory track exactly like the same
frames in memory, and the outputs of the run write out (GPU)."""

import numpy as np
import pytest

import kinectfusion_b200 as kf
from kinectfusion_b200 import abi, synthetic, tum

pytestmark = pytest.mark.gpu

K640 = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)


def test_tum_directory_replay_matches_memory(tmp_path):
    seq = synthetic.make_sequence(seed=12, frames=5)
    root = tmp_path / "rgbd_dataset_synthetic"
    tum.write_sequence(root, seq.depth, seq.color)
    half = 0.5 * 128 * 0.02
    cfg = kf.pipeline_config(128, 0.02, (-half, -half, -0.5), 0.05)
    runs = []
    for source in ("memory", "files"):
        loop = kf.Reconstruction(kf.Pipeline(cfg), K640)
        frames = (zip(seq.depth, seq.color) if source == "memory"
                  else ((f.depth, f.color) for f in tum.TumSequence(root, prefetch=2)))
        for depth, color in frames:
            loop.process(depth, color)
        runs.append(loop)
    assert all(np.array_equal(a, b) for a, b in zip(runs[0].trajectory, runs[1].trajectory))
    assert np.array_equal(runs[0].pipeline.download_raw(), runs[1].pipeline.download_raw())
    # the run's outputs
    loop = runs[1]
    mesh = loop.pipeline.extract_mesh(2.0)
    tum.write_mesh_ply(tmp_path / "mesh.ply", mesh)
    maps = loop.pipeline.raycast(K640, 640, 480, loop.trajectory[-1])
    tum.write_point_cloud_ply(tmp_path / "cloud.ply", maps.points, maps.normals, maps.colors)
    tum.write_color_png(tmp_path / "raycast.png", maps.colors)
    tum.write_trajectory(tmp_path / "trajectory.txt", loop.trajectory, [i / 30 for i in range(5)])
    data = (tmp_path / "mesh.ply").read_bytes()
    head = data[:data.index(b"end_header")].decode()
    assert f"element vertex {len(mesh['positions'])}" in head
    assert f"element face {len(mesh['triangles'])}" in head
    hits = int(np.isfinite(maps.points).all(-1).sum())
    cloud = (tmp_path / "cloud.ply").read_bytes()
    assert f"element vertex {hits}" in cloud[:cloud.index(b"end_header")].decode()
    np.testing.assert_array_equal(tum.read_color_png(tmp_path / "raycast.png"), maps.colors)
    assert len((tmp_path / "trajectory.txt").read_text().splitlines()) == 5
