"""The march's skip structures against their definitions, recomputed on the
host from the fused voxels (kf_pipeline_download_skip_structures).

* Per voxel: observed (weight > 0) and exactly 1.0.
* Per stencil (the eight corners (x..x+1, y..y+1, z..z+1); corners past the
  volume are unobserved), packed per brick layer: decided nullopt, decided
  1.0, undecided with every observed corner exactly 1.0 (the corner weights
  decide), undecided with another observed value (only the gather decides).
  With REQUIRE_ALL a missing corner decides nullopt.
* Per brick: class 1 when every stencil based in it is decided nullopt, 2
  when every one is exactly 1.0, else 0; and the largest radius r <= 7 such
  that every brick within Chebyshev distance r lies in the brick grid and has
  the brick's class (0 for class 0).

The raycast's bit-exact maps rest on these: a radius or a decided stencil
that is wrong in the permissive direction would let the march skip a sample
it must take, one wrong in the other direction only costs time.  Both
directions are pinned here, after every one of several frames and after a
reset.
"""

import itertools

import numpy as np
import pytest
from scipy import ndimage

import kf_oracle as ko
import kinectfusion_b200 as kf
from kinectfusion_b200 import abi, synthetic

pytestmark = pytest.mark.gpu

K640 = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
RES, VOXEL, TRUNC = 128, 0.02, 0.05
ORIGIN = (-0.5 * RES * VOXEL, -0.5 * RES * VOXEL, -0.5)


@pytest.fixture(scope="module")
def seq():
    return synthetic.make_sequence(seed=43, frames=4)


def _pack(bits: np.ndarray, bricks: tuple[int, int, int]) -> tuple[np.ndarray, np.ndarray]:
    """(z, y, x) bits -> per (brick z, y, x, layer) the two 32-bit words of bit y*8+x."""
    bz, by, bx = bricks
    b = bits.reshape(bz, 8, by, 8, bx, 8).transpose(0, 2, 4, 1, 3, 5).reshape(bz, by, bx, 8, 64)
    weights = np.uint64(1) << np.arange(32, dtype=np.uint64)
    lo = (b[..., :32].astype(np.uint64) * weights).sum(-1).astype(np.uint32)
    hi = (b[..., 32:].astype(np.uint64) * weights).sum(-1).astype(np.uint32)
    return lo, hi


def expected_structures(tsdf: np.ndarray, weight: np.ndarray, require_all: bool):
    rz, ry, rx = tsdf.shape
    bricks = (rz // 8, ry // 8, rx // 8)
    observed = np.zeros((rz + 1, ry + 1, rx + 1), dtype=bool)
    one = np.zeros_like(observed)
    observed[:rz, :ry, :rx] = weight > 0.0
    one[:rz, :ry, :rx] = (weight > 0.0) & (tsdf == np.float32(1.0))
    any_obs = np.zeros((rz, ry, rx), dtype=bool)
    all_obs = np.ones_like(any_obs)
    no_bad = np.ones_like(any_obs)
    for dz, dy, dx in itertools.product((0, 1), repeat=3):
        o = observed[dz:dz + rz, dy:dy + ry, dx:dx + rx]
        n = one[dz:dz + rz, dy:dy + ry, dx:dx + rx]
        any_obs |= o
        all_obs &= o
        no_bad &= n | ~o
    exactly_one = all_obs & no_bad
    decided = (~all_obs | no_bad) if require_all else (~any_obs | exactly_one)
    undecided = ~decided
    weigh = undecided & no_bad
    ulo, uhi = _pack(undecided, bricks)
    olo, ohi = _pack(exactly_one | weigh, bricks)
    records = np.stack([ulo, uhi, olo, ohi], axis=-1)

    def per_brick(bits):
        bz, by, bx = bricks
        return bits.reshape(bz, 8, by, 8, bx, 8).all(axis=(1, 3, 5))

    cls = np.where(per_brick(~undecided & ~exactly_one), 1, np.where(per_brick(exactly_one), 2, 0)).astype(np.uint8)
    radius = np.zeros_like(cls)
    alive = cls > 0
    for k in range(1, 8):
        # out-of-grid bricks count as different (255 above, 0 below any class)
        hi = ndimage.maximum_filter(cls, size=2 * k + 1, mode="constant", cval=255)
        lo = ndimage.minimum_filter(cls, size=2 * k + 1, mode="constant", cval=0)
        alive &= (hi == cls) & (lo == cls)
        radius[alive] = k
    return records, cls, radius


def check(gpu: kf.Pipeline, require_all: bool):
    tsdf, weight = gpu.host_view()
    records, cls, radius = expected_structures(tsdf, weight, require_all)
    got_cls, got_radius, got_records = gpu.skip_structures()
    assert np.array_equal(got_records, records), np.argwhere(got_records != records)[:5]
    assert np.array_equal(got_cls, cls)
    assert np.array_equal(got_radius, radius), np.argwhere(got_radius != radius)[:5]
    return cls, radius


@pytest.mark.parametrize("policy", [abi.KF_CORNERS_SKIP_MISSING, abi.KF_CORNERS_REQUIRE_ALL])
def test_skip_structures_match_definitions(seq, policy):
    gpu = kf.Pipeline(kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_NONE,
                                         raycast_corner_policy=policy))
    require_all = policy == abi.KF_CORNERS_REQUIRE_ALL
    for f in range(4):
        normals = ko.pyramid(seq.depth[f], K640, ko.depth_options())[0]["normals"]
        gpu.integrate(seq.depth[f], K640, ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[f])), normals=normals)
        cls, radius = check(gpu, require_all)
    # the fixture exercises every case: all three classes, several radii,
    # and both kinds of undecided stencil
    assert set(np.unique(cls)) == {0, 1, 2}
    assert radius.max() >= 3 and len(np.unique(radius[cls > 0])) >= 3
    _, _, records = gpu.skip_structures()
    undecided = (records[..., 0] != 0) | (records[..., 1] != 0)
    weighing = (records[..., 0] & records[..., 2]) | (records[..., 1] & records[..., 3])
    gathering = (records[..., 0] & ~records[..., 2]) | (records[..., 1] & ~records[..., 3])
    assert undecided.any() and (gathering != 0).any()
    if not require_all:
        assert (weighing != 0).any()
    # a reset volume: everything decided nullopt, every brick class 1
    gpu.reset()
    got_cls, _, got_records = gpu.skip_structures()
    assert (got_records == 0).all() and (got_cls == 1).all()


def test_sparse_pipeline_has_no_skip_structures():
    gpu = kf.Pipeline(kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_NONE,
                                         storage=abi.KF_STORAGE_SPARSE, integration_mode=abi.KF_INTEGRATION_BAND,
                                         sparse_block_capacity=4096))
    with pytest.raises(ValueError):  # KF_ERR_INVALID_ARGUMENT
        gpu.skip_structures()
