"""Generates tests/golden/reference_small.npz: outputs of the reference's OWN
host implementation (oracle/_ref/libkf_ref.so, compiled from the reference's
sources by oracle/ref_build.sh) on seeded synthetic inputs, so that the
golden tests can check the oracle and the device against the reference on a
machine where that library was not built.

Run from the repository root where the reference's sources are available:

    python tests/golden/make_golden.py

Inputs: synthetic.make_sequence(seed=7, frames=4) (the fixture stores each
frame's SHA-256; the tests regenerate the frames and check it).  Outputs:

* the depth pyramid of frame 3 (DepthProcessor<kHost>::build_surface_pyramid,
  depth_processing.cpp:139-162): level-0 filtered depth, level-2 vertex and
  normal maps;
* a 64^3 float volume at 4 cm (angle-weighted, colour off) after frames 0-2
  fused at their ground-truth poses with the reference's own level-0
  normals (BasicHostPipeline::integrate, pipeline.cpp:23-103): raw voxels;
* the 160x120 raycast of that volume at frame 3's pose (Raycaster): points
  and normals;
* the level-2 ICP normal equations of frame 3 against that render
  (IcpNormalEquations over CorrespondenceSearch, icp_correspondence.hpp):
  the 29 sums and the count;
* the reference's frame loop (Reconstruction::process_frame,
  reconstruction.cpp:184-277) over frames 0-3 on a fresh 64^3 volume: the
  poses and level statuses;
* the marching-cubes mesh of the 64^3 volume at min weight 0
  (MarchingCubes::extract, marching_cubes.cpp:367-507): the vertex positions
  in lexicographic order and the triangle count;
* a sparse bf16 store over a 128^3 domain at 2 cm (BlockRep<kHost>,
  block_rep.hpp:193-329) after frames 0-2 with band integration: the blocks
  it allocated and each allocated block's voxels, in block order.
"""

import hashlib
import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "oracle")]

import kf_oracle as ko  # noqa: E402  (option structs and small helpers)
import kf_ref as kr  # noqa: E402
import kinectfusion_b200 as kf  # noqa: E402
from kinectfusion_b200 import abi, synthetic  # noqa: E402

SEED, FRAMES = 7, 4
RES, VOXEL, TRUNC = 64, 0.04, 0.12
ORIGIN = (-0.5 * RES * VOXEL, -0.5 * RES * VOXEL, -0.5)
SPARSE_RES, SPARSE_VOXEL, SPARSE_TRUNC = 128, 0.02, 0.05
SPARSE_ORIGIN = (-0.5 * SPARSE_RES * SPARSE_VOXEL, -0.5 * SPARSE_RES * SPARSE_VOXEL, -0.5)


def frame_hashes(seq) -> np.ndarray:
    return np.array([hashlib.sha256(np.ascontiguousarray(seq.depth[f]).tobytes()).hexdigest()
                     for f in range(FRAMES)])


def main() -> None:
    if not kr.available():
        raise SystemExit("oracle/_ref/libkf_ref.so is not built (python oracle/ref_build.sh needs the reference)")
    seq = synthetic.make_sequence(seed=SEED, frames=FRAMES)
    k = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
    pyr3 = kr.pyramid(seq.depth[3], k, ko.depth_options())
    cfg = kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_NONE, rule=abi.KF_RULE_ANGLE_WEIGHTED)
    ref = kr.RefPipeline(cfg)
    for f in range(3):
        normals = kr.pyramid(seq.depth[f], k, ko.depth_options())[0]["normals"]
        ref.integrate(seq.depth[f], k, ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[f])), normals=normals)
    k2 = ko.scaled(k, 2)
    map_points, map_normals, _ = ref.raycast(k2, 160, 120, seq.poses[3])
    camera = abi.rigid_from_matrix(seq.poses[3])
    sums, count = kr.icp_equations(pyr3[2]["vertices"], pyr3[2]["normals"], map_points, map_normals, k2, camera,
                                   ko.rigid_inverse(camera))
    loop = kr.RefPipeline(cfg)
    pose = np.eye(4, dtype=np.float32)
    poses, statuses = [], []
    for f in range(FRAMES):
        pose, tracked, status = loop.track_frame(seq.depth[f], k, pose, ko.depth_options(), ko.icp_options(),
                                                 first=(f == 0))
        assert tracked
        poses.append(pose)
        statuses.append(status)
    mesh = ref.mesh(0.0)
    order = np.lexsort(mesh["positions"].T[::-1])
    scfg = kf.pipeline_config(SPARSE_RES, SPARSE_VOXEL, SPARSE_ORIGIN, SPARSE_TRUNC, voxel=abi.KF_VOXEL_BF16,
                              color=abi.KF_COLOR_NONE, rule=abi.KF_RULE_ANGLE_WEIGHTED,
                              storage=abi.KF_STORAGE_SPARSE, integration_mode=abi.KF_INTEGRATION_BAND)
    sparse = kr.RefPipeline(scfg)
    for f in range(3):
        normals = kr.pyramid(seq.depth[f], k, ko.depth_options())[0]["normals"]
        sparse.integrate(seq.depth[f], k, ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[f])), normals=normals)
    assert not sparse.overflowed()
    grid = sparse.grid()
    blocks = np.nonzero(grid != 0xFFFFFFFF)[0].astype(np.uint32)
    pool = sparse.voxels().reshape(-1, 512)
    out = pathlib.Path(__file__).with_name("reference_small.npz")
    np.savez_compressed(out, frame_sha256=frame_hashes(seq),
                        pyramid_l0_depth=pyr3[0]["depth"], pyramid_l2_vertices=pyr3[2]["vertices"],
                        pyramid_l2_normals=pyr3[2]["normals"],
                        voxels=ref.voxels(), raycast_points=map_points, raycast_normals=map_normals,
                        icp_sums=np.asarray(sums, np.float32), icp_count=np.uint64(count),
                        loop_poses=np.array(poses, np.float32), loop_status=np.array(statuses, np.int32),
                        mesh_positions=mesh["positions"][order], mesh_triangles=np.uint64(len(mesh["triangles"])),
                        sparse_blocks=blocks, sparse_voxels=pool[grid[blocks]])
    print(out, out.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
