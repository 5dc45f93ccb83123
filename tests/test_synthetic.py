"""The seeded synthetic frame source (CPU)."""

import numpy as np

from kinectfusion_b200 import synthetic


def test_sequence_is_deterministic_and_in_range():
    a = synthetic.make_sequence(seed=5, frames=3)
    b = synthetic.make_sequence(seed=5, frames=3)
    assert np.array_equal(a.depth, b.depth) and np.array_equal(a.color, b.color)
    assert a.depth.shape == (3, 480, 640) and a.depth.dtype == np.uint16
    valid = a.depth[a.depth > 0] / synthetic.DEPTH_SCALE
    assert valid.min() >= 0.4 and valid.max() <= 4.0
    drop = (a.depth == 0).mean()
    assert 0.02 <= drop < 0.2
    assert (a.color >> 24 == 255).all()


def test_trajectory_step_bounds():
    seq = synthetic.make_sequence(seed=9, frames=12, max_step_m=0.02, max_step_deg=1.0)
    assert np.allclose(seq.poses[0], np.eye(4))
    for k in range(1, 12):
        rel = np.linalg.inv(seq.poses[k - 1]) @ seq.poses[k]
        step_t = np.linalg.norm(seq.poses[k][:3, 3] - seq.poses[k - 1][:3, 3])
        ang = np.degrees(np.arccos(np.clip((np.trace(rel[:3, :3]) - 1) / 2, -1, 1)))
        assert step_t <= 0.02 + 1e-9 and ang <= 1.0 + 1e-6


def test_ate_of_identical_trajectories_is_zero():
    seq = synthetic.make_sequence(seed=2, frames=4)
    stats = synthetic.ate_rmse(seq.poses, seq.poses)
    assert stats["rmse"] < 1e-12 and stats["pairs"] == 4
