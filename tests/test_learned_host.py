"""Host-side logic of the learned warm start (CPU only): the twist
convention shared with the device, the constant-velocity prediction, the
mirroring used in training, the parameter layout, and the CLI seed ranges."""

import ctypes as C

import numpy as np
import pytest

import kf_learn_oracle as lo
from kinectfusion_b200 import abi, learned


def _pose(rng, rot=0.3, trans=1.0):
    m = np.eye(4)
    m[:3, :3] = learned.so3_exp(rng.normal(size=3) * rot)
    m[:3, 3] = rng.normal(size=3) * trans
    return m


def test_twist_round_trip_and_convention():
    rng = np.random.default_rng(0)
    for _ in range(20):
        p = _pose(rng)
        tw = rng.normal(size=6) * 0.05
        q = learned.apply_twist(p, tw)
        np.testing.assert_allclose(learned.twist_between(p, q), tw, atol=1e-12)
        # translation is added in the pose's frame, rotation right-multiplied
        np.testing.assert_allclose(q[:3, 3], p[:3, 3] + p[:3, :3] @ tw[:3], atol=1e-12)
        np.testing.assert_allclose(q[:3, :3], p[:3, :3] @ learned.so3_exp(tw[3:]), atol=1e-12)
    assert learned.TWIST_SCALE == 50.0


def test_so3_log_small_and_large_angles():
    for w in ([1e-10, 0, 0], [0.1, -0.2, 0.3], [0, 0, 3.0]):
        w = np.array(w)
        np.testing.assert_allclose(learned.so3_log(learned.so3_exp(w)), w, atol=1e-9)


def test_constant_velocity_repeats_the_last_motion():
    rng = np.random.default_rng(1)
    a = _pose(rng)
    tw = rng.normal(size=6) * 0.02
    b = learned.apply_twist(a, tw)
    c = learned.constant_velocity([a, b])
    # the relative motion b^-1 c equals a^-1 b
    np.testing.assert_allclose(np.linalg.inv(b) @ c, np.linalg.inv(a) @ b, atol=1e-12)
    np.testing.assert_array_equal(learned.constant_velocity([a]), a)


@pytest.mark.parametrize("dim", [1, 2])
def test_mirror_signs_follow_the_camera_reflection(dim):
    # mirroring the image along `dim` (2: x, 1: y) reflects the camera axis;
    # the relative twist of reflected poses equals the signed twist
    rng = np.random.default_rng(dim)
    axis = 0 if dim == 2 else 1
    s = np.eye(4)
    s[axis, axis] = -1
    for _ in range(10):
        a = _pose(rng)
        tw = rng.normal(size=6) * 0.02
        b = learned.apply_twist(a, tw)
        got = learned.twist_between(s @ a @ s, s @ b @ s)
        np.testing.assert_allclose(got, tw * np.array(learned._FLIP_SIGNS[dim]), atol=1e-12)


def test_parameter_layout_matches_the_oracle_and_the_shipped_file():
    lay, total = lo.layout()
    params = np.load(learned.PARAMS)
    assert params.dtype == np.float32 and params.size == total
    for w, rows, cols, b in lay:
        assert w % 8 == 0 and b % 8 == 0
    # conv1's padded columns stay zero after training
    w, rows, cols, _ = lay[0]
    assert not params[w:w + rows * cols].reshape(rows, cols)[:, 18:].any()
    assert np.isfinite(params).all()


def test_seed_ranges():
    assert learned._seed_range("3-6") == [3, 4, 5, 6]
    assert learned._seed_range("7") == [7]


def test_warm_start_result_layout():
    # kf_warm_start_result: two kf_rigid, six floats, four floats, one int
    assert C.sizeof(abi.WarmStartResult) == 2 * 48 + 6 * 4 + 4 * 4 + 4
