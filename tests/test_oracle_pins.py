"""Pins the CPU oracle to the reference's own known-answer tests.

Each test re-expresses one TEST_CASE of test/tests.cpp (cited by line) against
oracle/libkf_oracle.so.  These run on the CPU; they prove the restatement
behaves like the reference before it is trusted as the GPU checker.
"""

import numpy as np
import pytest

import kf_oracle as ko
from fixtures import (DEPTH_1M, DEPTH_1P4M, SYNTH_IMAGE, SYNTH_VOXEL, compare_maps, compare_volumes, flat_depth,
                      identical_surface, perturbed_initial, planar_surface, synth_intrinsics, synth_volume)
from kinectfusion_b200 import abi


def test_flat_depth_back_projection_and_normal():
    # tests.cpp:187-210
    depth = np.full((3, 3), DEPTH_1M, dtype=np.uint16)
    k = abi.Intrinsics(1.0, 1.0, 1.0, 1.0)
    o = ko.depth_options()
    v = ko.vertices(depth, k, o)
    assert np.allclose(v[1, 1], [0.0, 0.0, 1.0])
    assert np.allclose(v[1, 2], [1.0, 0.0, 1.0])
    n = ko.normals(v, o)
    assert np.allclose(n[1, 1], [0.0, 0.0, -1.0])
    # border normals are invalid (depth_processing.hpp:255-258)
    assert np.isnan(n[0]).all() and np.isnan(n[:, 0]).all()


def test_downsample_rejects_mixed_depth():
    # tests.cpp:212-225
    depth = np.array([[DEPTH_1M, DEPTH_1P4M], [DEPTH_1M, DEPTH_1M]], dtype=np.uint16)
    out = ko.downsample(depth, ko.depth_options())
    assert out.shape == (1, 1) and out[0, 0] == 0


def test_downsample_rounded_average():
    # BlockDownsample averages valid samples with (sum + count/2) / count
    depth = np.array([[5000, 5001], [0, 5002]], dtype=np.uint16)
    assert ko.downsample(depth, ko.depth_options())[0, 0] == (15003 + 1) // 3


def test_bilateral_flat_and_invalid():
    o = ko.depth_options()
    flat = np.full((9, 9), DEPTH_1M, dtype=np.uint16)
    assert (ko.bilateral(flat, o) == DEPTH_1M).all()
    hole = flat.copy()
    hole[4, 4] = 0
    out = ko.bilateral(hole, o)
    assert out[4, 4] == 0 and out[4, 5] == DEPTH_1M


def _plane_volume(rule=abi.KF_RULE_ANGLE_WEIGHTED, **kw):
    vol = synth_volume(**kw)
    ko.integrate(vol, flat_depth(DEPTH_1M), synth_intrinsics(), np.eye(4), ko.integration_options(), rule)
    return vol


def test_plane_integrates_and_raycasts():
    # tests.cpp:454-474
    vol = _plane_volume()
    assert vol.observed_voxel_count() > 0
    pts, nrm, _ = ko.raycast(vol, synth_intrinsics(), SYNTH_IMAGE, SYNTH_IMAGE, np.eye(4), ko.raycast_options())
    assert compare_maps(pts, nrm, pts, nrm)["compared"] > 0
    valid = np.isfinite(pts).all(-1)
    # the plane lies at z = 1 m
    assert np.abs(pts[valid][:, 2] - 1.0).max() < 0.05


def test_rules_differ_and_repeat_exactly():
    # tests.cpp:505-558
    k = synth_intrinsics()
    normals = np.zeros((SYNTH_IMAGE, SYNTH_IMAGE, 3), dtype=np.float32)
    normals[..., 2] = -1.0

    def two_planes(rule):
        vol = synth_volume()
        for raw in (DEPTH_1M, DEPTH_1P4M):
            ko.integrate(vol, flat_depth(raw), k, np.eye(4), ko.integration_options(), rule, normals_map=normals)
        return vol.dense()

    classic = two_planes(abi.KF_RULE_CLASSIC)
    angle = two_planes(abi.KF_RULE_ANGLE_WEIGHTED)
    d = compare_volumes(classic, angle)
    assert d["compared"] > 0 and d["only_primary"] == 0 and d["only_reference"] == 0
    assert d["max_weight_delta"] > 0 and d["max_distance_delta"] > 0
    again = two_planes(abi.KF_RULE_ANGLE_WEIGHTED)
    same = compare_volumes(angle, again)
    assert same["max_distance_delta"] == 0.0 and same["max_weight_delta"] == 0.0


def test_voxel_storages_agree_within_quantum():
    # tests.cpp:667-696
    ref = _plane_volume(rule=abi.KF_RULE_ANGLE_WEIGHTED).dense()
    for kind, bound in ((abi.KF_VOXEL_QUANTIZED, 1e-4), (abi.KF_VOXEL_BF16, 5e-3)):
        got = _plane_volume(voxel=kind).dense()
        d = compare_volumes(got, ref)
        assert d["compared"] > 0 and d["only_primary"] == 0 and d["only_reference"] == 0
        assert 0.0 < d["max_distance_delta"] < bound


def test_band_matches_full_near_surface():
    # tests.cpp:698-720
    full = _plane_volume().dense()
    vol = synth_volume()
    ko.integrate(vol, flat_depth(DEPTH_1M), synth_intrinsics(), np.eye(4),
                 ko.integration_options(mode=abi.KF_INTEGRATION_BAND))
    d = compare_volumes(vol.dense(), full)
    assert d["compared"] > 0 and d["max_distance_delta"] == 0.0
    assert d["only_reference"] > 0 and d["only_primary"] == 0


def test_sparse_matches_dense_band_and_overflow_drops():
    # tests.cpp:722-770
    o = ko.integration_options(mode=abi.KF_INTEGRATION_BAND)
    dense = synth_volume()
    ko.integrate(dense, flat_depth(DEPTH_1M), synth_intrinsics(), np.eye(4), o)
    sparse = synth_volume(sparse=True)
    ko.integrate(sparse, flat_depth(DEPTH_1M), synth_intrinsics(), np.eye(4), o)
    d = compare_volumes(sparse.dense(), dense.dense())
    assert d["compared"] > 0 and d["max_distance_delta"] == 0.0
    assert d["only_primary"] == 0 and d["only_reference"] == 0
    tiny = synth_volume(sparse=True, capacity=1)
    ko.integrate(tiny, flat_depth(DEPTH_1M), synth_intrinsics(), np.eye(4), o)
    d = compare_volumes(tiny.dense(), dense.dense())
    assert d["max_distance_delta"] == 0.0 and d["only_primary"] == 0 and d["only_reference"] > 0
    assert tiny.struct.allocated > tiny.capacity  # the overflow is recorded


def _icp(surface, initial, iterations, **opts):
    v, n = surface
    k = abi.Intrinsics(100.0, 100.0, 1.0, 1.0)
    return ko.icp_estimate(v, n, v, n, k, np.eye(4, dtype=np.float32), initial, iterations, ko.icp_options(**opts))


STRICT = dict(min_correspondences=6, max_point_distance=0.1, min_system_eigenvalue=1e-12, max_condition_number=1e12)


def test_icp_identity_converges():
    # tests.cpp:880-904
    out = _icp(identical_surface(), np.eye(4, dtype=np.float32), 3, min_normal_dot=0.99, **STRICT)
    assert out.status == abi.KF_ICP_CONVERGED
    assert out.correspondences == 9
    assert abs(out.update_translation) < 1e-5 and abs(out.update_rotation) < 1e-5


def test_icp_recovers_perturbation():
    # tests.cpp:906-942
    out = _icp(identical_surface(), perturbed_initial(), 15, min_normal_dot=0.9, **STRICT)
    assert out.status == abi.KF_ICP_CONVERGED
    assert out.correspondences == 9
    assert np.linalg.norm(abi.matrix_from_rigid(out.pose) - np.eye(4)) < 1e-3
    assert abs(out.mean_point_distance) < 1e-4


@pytest.mark.parametrize("mode", [abi.KF_DAMPING_IDENTITY, abi.KF_DAMPING_DIAGONAL])
@pytest.mark.parametrize("adaptive", [0, 1])
def test_damped_icp_recovers_perturbation(mode, adaptive):
    # tests.cpp:944-981
    out = _icp(identical_surface(), perturbed_initial(), 25, min_normal_dot=0.9, damping_mode=mode,
               damping_lambda=1e-4, adaptive_damping=adaptive, **STRICT)
    assert out.status in (abi.KF_ICP_CONVERGED, abi.KF_ICP_MAX_ITERATIONS)
    assert out.correspondences == 9 and out.damping_lambda > 0
    assert np.linalg.norm(abi.matrix_from_rigid(out.pose) - np.eye(4)) < 1e-3


def test_planar_system_vetoed_then_damped():
    # tests.cpp:983-1009
    opts = dict(min_correspondences=6, max_point_distance=0.1, min_normal_dot=0.9)
    out = _icp(planar_surface(), np.eye(4, dtype=np.float32), 3, **opts)
    assert out.status == abi.KF_ICP_UNCONSTRAINED_SYSTEM
    out = _icp(planar_surface(), np.eye(4, dtype=np.float32), 3, damping_mode=abi.KF_DAMPING_DIAGONAL,
               damping_lambda=1e-3, **opts)
    assert out.status in (abi.KF_ICP_CONVERGED, abi.KF_ICP_MAX_ITERATIONS) and out.correspondences == 9


def test_adaptive_damping_shrinks_lambda():
    # tests.cpp:1011-1045
    out = _icp(identical_surface(), perturbed_initial(rotate=False), 25, min_normal_dot=0.9,
               damping_mode=abi.KF_DAMPING_IDENTITY, damping_lambda=1e-2, adaptive_damping=1, **STRICT)
    assert out.status in (abi.KF_ICP_CONVERGED, abi.KF_ICP_MAX_ITERATIONS)
    assert out.rejected_steps == 0 and out.damping_lambda < 1e-2
    assert np.linalg.norm(abi.matrix_from_rigid(out.pose) - np.eye(4)) < 1e-3


def test_icp_rejects_empty_correspondences():
    # tests.cpp:1047-1074
    nan = np.full((2, 2, 3), np.nan, dtype=np.float32)
    out = ko.icp_estimate(nan, nan, nan, nan, abi.Intrinsics(0, 0, 0, 0), np.eye(4, dtype=np.float32),
                          np.eye(4, dtype=np.float32), 10, ko.icp_options(min_correspondences=1))
    assert out.status == abi.KF_ICP_TOO_FEW_CORRESPONDENCES and out.correspondences == 0


def test_icp_f64_sums_agree_with_f32():
    v, n = identical_surface()
    k = abi.Intrinsics(100.0, 100.0, 1.0, 1.0)
    s32, c32 = ko.icp_equations(v, n, v, n, k, np.eye(4), np.eye(4), 0.1, 0.9)
    s64, c64 = ko.icp_equations(v, n, v, n, k, np.eye(4), np.eye(4), 0.1, 0.9, f64=True)
    assert c32 == c64 == 9
    assert np.allclose(s32, s64, rtol=1e-5, atol=1e-7)


# ---- marching cubes (tests.cpp:320-452) -------------------------------------------------
def test_marching_cubes_sphere_is_closed_and_outward():
    # tests.cpp:320-385
    from fixtures import mesh_edge_uses, sphere_volume
    vol = synth_volume()
    center, radius = sphere_volume(vol)
    mesh = ko.marching_cubes(vol)
    p, n, t = mesh["positions"], mesh["normals"], mesh["triangles"].astype(np.int64)
    assert len(p) > 0 and len(t) > 0 and len(n) == len(p) == len(mesh["colors"])
    radial = p - center
    assert (np.abs(np.linalg.norm(radial, axis=1) - radius) < vol.geometry.voxel_size).all()
    assert ((n * radial).sum(1) > 0).all()
    face = np.cross(p[t[:, 1]] - p[t[:, 0]], p[t[:, 2]] - p[t[:, 0]])
    centroid = (p[t[:, 0]] + p[t[:, 1]] + p[t[:, 2]]) / 3
    assert ((face * (centroid - center)).sum(1) > 0).all()
    uses = mesh_edge_uses(t)
    assert set(uses.values()) == {2}
    assert len(p) - len(uses) + len(t) == 2  # Euler characteristic of a sphere
    assert (mesh["colors"] == 255.0).all()   # no colour facet: white


def test_marching_cubes_plane_at_one_metre():
    # tests.cpp:387-400
    mesh = ko.marching_cubes(_plane_volume(rule=abi.KF_RULE_CLASSIC))
    assert len(mesh["triangles"]) > 0
    assert (np.abs(mesh["positions"][:, 2] - 1.0) < SYNTH_VOXEL).all()


def test_marching_cubes_unobserved_is_empty():
    # tests.cpp:402-407
    mesh = ko.marching_cubes(synth_volume())
    assert len(mesh["positions"]) == 0 and len(mesh["triangles"]) == 0


def test_sparse_marching_cubes_matches_dense_band_mesh():
    # tests.cpp:409-437
    o = ko.integration_options(mode=abi.KF_INTEGRATION_BAND)
    dense = synth_volume()
    ko.integrate(dense, flat_depth(DEPTH_1M), synth_intrinsics(), np.eye(4), o)
    sparse = synth_volume(sparse=True)
    ko.integrate(sparse, flat_depth(DEPTH_1M), synth_intrinsics(), np.eye(4), o)
    a, b = ko.marching_cubes(sparse), ko.marching_cubes(dense)
    assert len(a["triangles"]) > 0
    assert len(a["triangles"]) == len(b["triangles"]) and len(a["positions"]) == len(b["positions"])
    key = lambda p: p[np.lexsort((p[:, 2], p[:, 1], p[:, 0]))]
    assert np.array_equal(key(a["positions"]), key(b["positions"]))


def test_marching_cubes_weight_threshold():
    # tests.cpp:439-452: one classic frame leaves every weight at 1
    vol = _plane_volume(rule=abi.KF_RULE_CLASSIC)
    assert len(ko.marching_cubes(vol, 2.0)["triangles"]) == 0
    assert len(ko.marching_cubes(vol, 1.0)["triangles"]) > 0


def test_marching_cubes_table_is_the_generated_one():
    # the committed header is what the generator writes
    import importlib.util
    import pathlib
    here = pathlib.Path(__file__).resolve().parent.parent / "kinectfusion_b200" / "csrc"
    spec = importlib.util.spec_from_file_location("mc_tables", here / "mc_tables.py")
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    masks, table = gen.build()
    counts = ko.mc_case_triangle_counts()
    assert counts[0] == 0 and counts[255] == 0
    assert [sum(1 for v in row if v >= 0) // 3 for row in table] == counts.tolist()
    assert all(bin(m).count("1") >= 3 for m in masks[1:255])
