"""Pins the CPU oracle to the reference ITSELF.

oracle/_ref/libkf_ref.so is the reference's own host implementation
(src/kinectfusion/*.cpp and include/kinectfusion/*.hpp) compiled from its
sources by oracle/ref_build.sh against this project's Eigen stand-in; the
oracle (oracle/kf_oracle.c) is the C restatement the sm_100a kernels are
checked against bit for bit.  Here both run on the same seeded cfg1 inputs
(640x480 synthetic frames, 128^3 volume at 2 cm, 5 cm truncation):

* integration (float / int16 / bf16 voxels, classic and angle-weighted,
  full and band sweeps, colour), raycasts (plain, bitmap and band march, both
  corner policies, cell normals, the integration knobs), sparse allocation
  (grid slots, pool, overflow) and the ICP normal-equation sums are
  BIT-EXACT: the restatement evaluates the reference's float expressions in
  the reference's order; so is the depth pyramid, except about one pixel in
  a million where glibc's expf (the reference's bilateral weight) is one ulp
  off the correctly rounded exp the oracle and the device use;
* where the reference's arithmetic runs through Eigen (the 6x6 eigenvalue
  veto, the LDLT solve, AngleAxis, the 4x4 inverse of a pose) the stand-in's
  arithmetic replaces Eigen's and the oracle uses its own (FP64 Jacobi, its
  LDL^T, rigid inverse): ICP poses agree within 1e-6 m / rad per level, the
  5-frame loop within 1e-4 m / rad, and the loop's TSDF within 1e-5 m on all
  but a handful of voxels whose projection lands on another pixel;
* marching cubes on identical volumes gives the same vertex set (positions,
  colours, gradient normals) and the same triangle count; the triangle table
  is this project's own (kinectfusion_b200/csrc/mc_tables.py), so triangles
  and first-use vertex numbering differ, and so do the face-average normals
  of vertices without a gradient (the reference averages over its own
  triangles) - counted, bounded and exact at the configs' min weight 2.

CPU only.  Skipped when the reference library cannot be built (no sources).
"""

import numpy as np
import pytest

import kf_oracle as ko
import kinectfusion_b200 as kf
from fixtures import identical_surface, perturbed_initial, planar_surface
from kinectfusion_b200 import abi, synthetic

kr = pytest.importorskip("kf_ref")

K640 = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
RES, VOXEL, TRUNC = 128, 0.02, 0.05
ORIGIN = (-0.5 * RES * VOXEL, -0.5 * RES * VOXEL, -0.5)


@pytest.fixture(scope="module", autouse=True)
def reference_library():
    if not kr.available():
        try:
            kr.build()
        except Exception as exc:  # pragma: no cover - depends on the sources being present
            pytest.skip(f"reference library not built: {exc}")
    if not kr.available():
        pytest.skip("reference sources absent: oracle/_ref/libkf_ref.so not built")
    kr.load()


@pytest.fixture(scope="module")
def seq():
    return synthetic.make_sequence(seed=7, frames=5)


def nan_equal(a, b):
    return np.array_equal(a, b, equal_nan=True)


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32).reshape(-1)


def _integrate_both(seq, frames, voxel=abi.KF_VOXEL_FLOAT, color=False, rule=abi.KF_RULE_ANGLE_WEIGHTED,
                    storage=abi.KF_STORAGE_DENSE, capacity=0, **kw):
    integ = {key.split("_", 1)[1]: v for key, v in kw.items() if key.startswith("integration_")}
    cfg = kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, voxel=voxel,
                             color=abi.KF_COLOR_FLOAT if color else abi.KF_COLOR_NONE, rule=rule, storage=storage,
                             sparse_block_capacity=capacity, **kw)
    ref = kr.RefPipeline(cfg)
    ora = ko.OracleVolume(RES, VOXEL, ORIGIN, TRUNC, voxel=voxel, color=color,
                          sparse=storage == abi.KF_STORAGE_SPARSE, capacity=capacity)
    io = ko.integration_options(**integ)
    for f in frames:
        normals = ko.pyramid(seq.depth[f], K640, ko.depth_options())[0]["normals"]
        w2c = ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[f]))
        col = seq.color[f] if color else None
        ref.integrate(seq.depth[f], K640, w2c, color=col, normals=normals)
        ko.integrate(ora, seq.depth[f], K640, w2c, io, rule, color=col, normals_map=normals, threads=8)
    return ref, ora


# ---- depth processing -----------------------------------------------------------------
def _near(mask: np.ndarray, radius: int) -> np.ndarray:
    """Pixels within `radius` (Chebyshev) of a set pixel."""
    out = mask.copy()
    h, w = mask.shape
    for dy in range(-radius, radius + 1):
        for dx in range(-radius, radius + 1):
            shifted = np.zeros_like(mask)
            shifted[max(dy, 0):h + min(dy, 0), max(dx, 0):w + min(dx, 0)] = \
                mask[max(-dy, 0):h + min(-dy, 0), max(-dx, 0):w + min(-dx, 0)]
            out |= shifted
    return out


@pytest.mark.parametrize("seed,frame", [(7, 0), (7, 2), (7, 3), (11, 1)])
def test_pyramid_matches_reference(seed, frame):
    """DepthProcessor<kHost>::build_surface_pyramid (depth_processing.cpp:139-162).

    The oracle (and the device) weigh the bilateral samples with exp in double
    rounded once; the reference calls glibc's expf, which is one ulp off the
    correctly rounded value for a small share of arguments.  On about one
    pixel in a million that moves the rounded filtered depth by one raw unit.
    Everything else is bit-exact, and the maps differ only where their
    stencils read such a pixel."""
    depth = synthetic.make_sequence(seed=seed, frames=frame + 1).depth[frame]
    ref = kr.pyramid(depth, K640, ko.depth_options())
    ora = ko.pyramid(depth, K640, ko.depth_options())
    assert len(ref) == len(ora) == 3
    d0 = ref[0]["depth"].astype(np.int32) - ora[0]["depth"].astype(np.int32)
    moved = d0 != 0
    assert moved.sum() <= 5 and np.abs(d0).max() <= 1
    for level, (r, o) in enumerate(zip(ref, ora)):
        h, w = r["depth"].shape
        # pixels of this level whose source block holds a moved level-0 pixel
        src = moved[:h << level, :w << level].reshape(h, 1 << level, w, 1 << level).any(axis=(1, 3))
        assert not (r["depth"] != o["depth"])[~src].any()
        vert_bad = ~np.all((r["vertices"] == o["vertices"]) | (np.isnan(r["vertices"]) & np.isnan(o["vertices"])), -1)
        norm_bad = ~np.all((r["normals"] == o["normals"]) | (np.isnan(r["normals"]) & np.isnan(o["normals"])), -1)
        assert not vert_bad[~src].any()
        assert not norm_bad[~_near(src, 1)].any()


# ---- integration ----------------------------------------------------------------------
@pytest.mark.parametrize("voxel", [abi.KF_VOXEL_FLOAT, abi.KF_VOXEL_QUANTIZED, abi.KF_VOXEL_BF16])
@pytest.mark.parametrize("rule", [abi.KF_RULE_CLASSIC, abi.KF_RULE_ANGLE_WEIGHTED])
@pytest.mark.parametrize("mode", [abi.KF_INTEGRATION_FULL, abi.KF_INTEGRATION_BAND])
def test_integration_raw_voxels_bit_exact(seq, voxel, rule, mode):
    """IntegrationSweep / BandIntegrationSweep<kHost> over BasicVolume
    (tsdf_integration.hpp:127-342, 378-497): raw storage codes equal."""
    color = voxel == abi.KF_VOXEL_FLOAT
    ref, ora = _integrate_both(seq, range(3), voxel=voxel, color=color, rule=rule, integration_mode=mode)
    assert np.array_equal(bits(ref.voxels()), bits(ora.voxels))
    if color:
        assert np.array_equal(bits(ref.colors()), bits(ora.colors))
    assert ref.observed_voxel_count() == ora.observed_voxel_count() > 10000


@pytest.mark.parametrize("knob", ["distance_scaled_truncation", "no_projective_distance"])
def test_integration_knobs_bit_exact(seq, knob):
    kw = ({"integration_distance_scaled_truncation": 1} if knob == "distance_scaled_truncation"
          else {"integration_projective_distance": 0})
    ref, ora = _integrate_both(seq, range(3), **kw)
    assert np.array_equal(bits(ref.voxels()), bits(ora.voxels))


# ---- raycast --------------------------------------------------------------------------
@pytest.mark.parametrize("case", ["march", "bitmap_march", "band_march", "require_all_corners", "cell_normals",
                                  "int16", "bf16_colour"])
def test_raycast_maps_bit_exact(seq, case):
    """SurfaceRaycast::render_pixel through EmptySpaceIndex (raycasting.hpp:94-252,
    empty_space_skip.hpp:20-287): points, normals and colours equal."""
    kw, ro, voxel, color = {}, {}, abi.KF_VOXEL_FLOAT, False
    if case == "bitmap_march":
        kw["raycast_backend"] = abi.KF_RAYCAST_BITMAP_MARCH
    elif case == "band_march":
        kw["raycast_backend"] = abi.KF_RAYCAST_BAND_MARCH
    elif case == "require_all_corners":
        kw["raycast_corner_policy"] = ro["corner_policy"] = abi.KF_CORNERS_REQUIRE_ALL
    elif case == "cell_normals":
        kw["raycast_cell_gradient_normals"] = ro["cell_gradient_normals"] = 1
    elif case == "int16":
        voxel = abi.KF_VOXEL_QUANTIZED
    elif case == "bf16_colour":
        voxel, color = abi.KF_VOXEL_FLOAT, True
    ref, ora = _integrate_both(seq, range(3), voxel=voxel, color=color, **kw)
    for level, pose in ((0, seq.poses[3]), (2, seq.poses[2])):
        k = ko.scaled(K640, level)
        w, h = 640 >> level, 480 >> level
        rp, rn, rc = ref.raycast(k, w, h, pose)
        if case == "band_march":
            raw, dilated = ko.band_bitmap(ora)
            op, on, oc = ko.raycast_band(ora, dilated, k, w, h, pose, ko.raycast_options(**ro), threads=8)
        else:
            op, on, oc = ko.raycast(ora, k, w, h, pose, ko.raycast_options(**ro), threads=8)
        assert np.isfinite(rp[..., 0]).sum() > 0.2 * w * h
        assert nan_equal(rp, op) and nan_equal(rn, on)
        if color:
            assert np.array_equal(rc, oc)


# ---- sparse storage -------------------------------------------------------------------
@pytest.mark.parametrize("capacity", [0, 120])
def test_sparse_allocation_and_pool_bit_exact(seq, capacity):
    """BlockRep<kHost> (block_rep.hpp:193-329): the block grid (slot per block,
    in the reference's allocation order), the pool and the overflow flag;
    capacity 120 overflows on the second frame."""
    ref, ora = _integrate_both(seq, range(3), voxel=abi.KF_VOXEL_BF16, storage=abi.KF_STORAGE_SPARSE,
                               capacity=capacity, integration_mode=abi.KF_INTEGRATION_BAND)
    assert np.array_equal(ref.grid(), ora.grid)
    assert np.array_equal(bits(ref.voxels()), bits(ora.voxels))
    assert ref.overflowed() == (ora.struct.allocated > ora.capacity)
    assert ref.overflowed() == (capacity != 0)
    rp, rn, _ = ref.raycast(K640, 640, 480, seq.poses[2])
    op, on, _ = ko.raycast(ora, K640, 640, 480, seq.poses[2], ko.raycast_options(), threads=8)
    assert nan_equal(rp, op) and nan_equal(rn, on)


# ---- ICP ------------------------------------------------------------------------------
@pytest.fixture(scope="module")
def tracking_case(seq):
    ora = ko.OracleVolume(RES, VOXEL, ORIGIN, TRUNC)
    for f in range(2):
        normals = ko.pyramid(seq.depth[f], K640, ko.depth_options())[0]["normals"]
        ko.integrate(ora, seq.depth[f], K640, ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[f])),
                     ko.integration_options(), abi.KF_RULE_CLASSIC, normals_map=normals, threads=8)
    live = ko.pyramid(seq.depth[2], K640, ko.depth_options())
    models = []
    for level in range(3):
        k = ko.scaled(K640, level)
        p, n, _ = ko.raycast(ora, k, 640 >> level, 480 >> level, seq.poses[1], ko.raycast_options(), threads=8)
        models.append((k, p, n))
    return live, models


@pytest.mark.parametrize("level", [0, 1, 2])
def test_icp_normal_equations_bit_exact(seq, tracking_case, level):
    """CorrespondenceSearch::match + IcpNormalEquations::accumulate in pixel
    order (icp_correspondence.hpp:104-176, 244-294)."""
    live, models = tracking_case
    k, p, n = models[level]
    camera = abi.rigid_from_matrix(seq.poses[1])
    model = ko.rigid_inverse(camera)
    s_ref, c_ref = kr.icp_equations(live[level]["vertices"], live[level]["normals"], p, n, k, camera, model)
    s_ora, c_ora = ko.icp_equations(live[level]["vertices"], live[level]["normals"], p, n, k, camera, model)
    assert c_ref == c_ora > 1000
    assert np.array_equal(s_ref, s_ora)


@pytest.mark.parametrize("level", [0, 1, 2])
@pytest.mark.parametrize("damping", ["none", "diagonal", "identity_adaptive"])
def test_icp_estimate_matches_reference(seq, tracking_case, level, damping):
    """ProjectiveIcpTracker::estimate_with (icp_optimizer.cpp:208-302): the
    reference's Eigen steps run on the stand-in, the oracle's on its own
    FP64 / LDL^T restatement; statuses equal, poses within 1e-6."""
    live, models = tracking_case
    k, p, n = models[level]
    opts = {"none": {}, "diagonal": {"damping_mode": abi.KF_DAMPING_DIAGONAL},
            "identity_adaptive": {"damping_mode": abi.KF_DAMPING_IDENTITY, "adaptive_damping": 1}}[damping]
    o_ref = kr.icp_estimate(live[level]["vertices"], live[level]["normals"], p, n, k, seq.poses[1], seq.poses[1], 10,
                            ko.icp_options(**opts))
    o_ora = ko.icp_estimate(live[level]["vertices"], live[level]["normals"], p, n, k, seq.poses[1], seq.poses[1], 10,
                            ko.icp_options(**opts))
    assert o_ref.status == o_ora.status
    assert o_ref.status in (abi.KF_ICP_CONVERGED, abi.KF_ICP_MAX_ITERATIONS)
    assert o_ref.correspondences == o_ora.correspondences
    assert np.abs(abi.matrix_from_rigid(o_ref.pose) - abi.matrix_from_rigid(o_ora.pose)).max() < 1e-6
    assert abs(o_ref.min_system_eigenvalue - o_ora.min_system_eigenvalue) <= 1e-4 * o_ora.min_system_eigenvalue
    assert abs(o_ref.condition_number - o_ora.condition_number) <= 1e-4 * o_ora.condition_number


def _icp_known(impl, surface, initial, iterations, **opts):
    v, n = surface
    k = abi.Intrinsics(100.0, 100.0, 1.0, 1.0)
    return impl.icp_estimate(v, n, v, n, k, np.eye(4, dtype=np.float32), initial, iterations, ko.icp_options(**opts))


STRICT = dict(min_correspondences=6, max_point_distance=0.1, min_system_eigenvalue=1e-12, max_condition_number=1e12)


def test_icp_known_answers_agree():
    """The reference's ICP unit cases (test/tests.cpp:880-1074) on both: the
    Eigen stand-in keeps the reference's own expected outcomes."""
    for impl in (kr, ko):
        out = _icp_known(impl, identical_surface(), np.eye(4, dtype=np.float32), 3, min_normal_dot=0.99, **STRICT)
        assert out.status == abi.KF_ICP_CONVERGED and out.correspondences == 9
        out = _icp_known(impl, identical_surface(), perturbed_initial(), 15, min_normal_dot=0.9, **STRICT)
        assert out.status == abi.KF_ICP_CONVERGED
        assert np.linalg.norm(abi.matrix_from_rigid(out.pose) - np.eye(4)) < 1e-3
        opts = dict(min_correspondences=6, max_point_distance=0.1, min_normal_dot=0.9)
        assert _icp_known(impl, planar_surface(), np.eye(4, dtype=np.float32), 3,
                          **opts).status == abi.KF_ICP_UNCONSTRAINED_SYSTEM
        out = _icp_known(impl, planar_surface(), np.eye(4, dtype=np.float32), 3, damping_mode=abi.KF_DAMPING_DIAGONAL,
                         damping_lambda=1e-3, **opts)
        assert out.status in (abi.KF_ICP_CONVERGED, abi.KF_ICP_MAX_ITERATIONS) and out.correspondences == 9
        out = _icp_known(impl, identical_surface(), perturbed_initial(rotate=False), 25, min_normal_dot=0.9,
                         damping_mode=abi.KF_DAMPING_IDENTITY, damping_lambda=1e-2, adaptive_damping=1, **STRICT)
        assert out.rejected_steps == 0 and out.damping_lambda < 1e-2
        nan = np.full((2, 2, 3), np.nan, dtype=np.float32)
        out = impl.icp_estimate(nan, nan, nan, nan, abi.Intrinsics(0, 0, 0, 0), np.eye(4, dtype=np.float32),
                                np.eye(4, dtype=np.float32), 10, ko.icp_options(min_correspondences=1))
        assert out.status == abi.KF_ICP_TOO_FEW_CORRESPONDENCES


# ---- the frame loop -------------------------------------------------------------------
def test_frame_loop_matches_reference(seq):
    """cfg1: 5 frames of Reconstruction::process_frame (reconstruction.cpp:184-277),
    classic TSDF, ICP [10, 5, 4]."""
    cfg = kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_NONE, rule=abi.KF_RULE_CLASSIC)
    ref = kr.RefPipeline(cfg)
    ora = ko.OracleVolume(RES, VOXEL, ORIGIN, TRUNC)
    p_ref = p_ora = np.eye(4, dtype=np.float32)
    for f in range(5):
        p_ref, ok_ref, status = ref.track_frame(seq.depth[f], K640, p_ref, ko.depth_options(), ko.icp_options(),
                                                first=(f == 0))
        p_ora, ok_ora, outcomes = ko.track_frame(ora, seq.depth[f], K640, p_ora, ko.depth_options(),
                                                 ko.integration_options(), ko.raycast_options(), ko.icp_options(),
                                                 rule=abi.KF_RULE_CLASSIC, threads=8, first=(f == 0))
        assert ok_ref and ok_ora
        for level, out in outcomes.items():
            assert status[level] == out.status
        p_ref, p_ora = np.asarray(p_ref), np.asarray(p_ora)
        assert np.abs(p_ref[:3, 3] - p_ora[:3, 3]).max() < 1e-4
        assert np.abs(p_ref[:3, :3] - p_ora[:3, :3]).max() < 1e-4
    # TSDF after the loop: equal to 1e-5 m except where a pose ulp moves a
    # voxel's projection onto another pixel
    r, o = ref.voxels(), ora.voxels
    both = (r[:, 1] > 0) & (o[:, 1] > 0)
    delta_m = np.abs(r[both, 0] - o[both, 0]) * TRUNC
    assert both.sum() > 100000
    assert (delta_m > 1e-5).sum() <= 1e-4 * both.sum()
    assert np.percentile(delta_m, 99.9) < 1e-5
    assert ((r[:, 1] > 0) != (o[:, 1] > 0)).sum() <= 1e-4 * both.sum()


# ---- marching cubes -------------------------------------------------------------------
@pytest.mark.parametrize("min_weight", [0.0, 2.0])
def test_mesh_vertex_set_matches_reference(seq, min_weight):
    """MarchingCubes::extract (marching_cubes.cpp:367-507) on identical volumes."""
    ref, ora = _integrate_both(seq, range(3), color=True)
    m_ref, m_ora = ref.mesh(min_weight), ko.marching_cubes(ora, min_weight)
    assert len(m_ref["positions"]) == len(m_ora["positions"]) > 100
    assert len(m_ref["triangles"]) == len(m_ora["triangles"])
    a = np.lexsort(m_ref["positions"].T[::-1])
    b = np.lexsort(m_ora["positions"].T[::-1])
    assert np.array_equal(m_ref["positions"][a], m_ora["positions"][b])
    assert np.array_equal(m_ref["colors"][a], m_ora["colors"][b])
    nr, no = m_ref["normals"][a], m_ora["normals"][b]
    differ = np.any(nr != no, axis=1)
    if min_weight >= 2.0:
        assert not differ.any()
    else:
        # face-average normals of vertices without a gradient normal follow
        # each table's triangles
        assert differ.sum() <= 0.05 * len(nr)
        cos = (nr[differ] * no[differ]).sum(1) / np.linalg.norm(nr[differ], axis=1) / np.linalg.norm(no[differ], axis=1)
        assert cos.min() > 0.9
