"""The learned warm start on the device: the CNN's forward pass and
gradients against the CPU oracle (which emulates the device's bf16 rounding),
training, the net input against host arithmetic, and the proposal's fallback
rule."""

import numpy as np
import pytest

import kf_learn_oracle as lo
import kinectfusion_b200 as kf
from kinectfusion_b200 import abi, learned, synthetic

pytestmark = pytest.mark.gpu


def _inputs(batch, seed):
    import torch
    rng = np.random.default_rng(seed)
    x = (rng.normal(size=(batch, 60, 80, 2)) * 0.5).astype(np.float32)
    x[:, :5] = 0.0  # a band of invalid (zero) pixels
    xb = lo.bf16(x)
    return torch.from_numpy(xb).to(torch.bfloat16).cuda(), xb


@pytest.mark.parametrize("batch", [8, 24])
def test_forward_matches_oracle(batch):
    net = learned.Learner(32, seed=1)
    params = lo.init_params(3)
    net.set_params(params)
    x, xh = _inputs(batch, batch)
    out = net.forward(x).cpu().numpy()
    ref, _ = lo.forward(params, xh, emulate=True)
    # fp32 accumulation order and the bf16 roundings it can flip between layers
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-2 * np.abs(ref).max())
    assert np.array_equal(net.params(), params)


def test_gradients_match_oracle():
    import torch
    net = learned.Learner(16, seed=2)
    params = lo.init_params(4)
    net.set_params(params)
    x, xh = _inputs(16, 7)
    rng = np.random.default_rng(9)
    t = rng.normal(size=(16, 6)).astype(np.float32)
    g, loss = net.gradients(x, torch.from_numpy(t).cuda())
    ref_loss, ref_g = lo.loss_and_gradients(params, xh, t, emulate=True)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss
    lay, _ = lo.layout()
    for i, (w, rows, cols, b) in enumerate(lay):
        gw, rw = g[w:w + rows * cols], ref_g[w:w + rows * cols]
        assert np.linalg.norm(gw - rw) <= 3e-2 * np.linalg.norm(rw), f"layer {i} weights"
        gb, rb = g[b:b + rows], ref_g[b:b + rows]
        assert np.linalg.norm(gb - rb) <= 3e-2 * np.linalg.norm(rb) + 1e-7, f"layer {i} bias"
    cos = g @ ref_g / (np.linalg.norm(g) * np.linalg.norm(ref_g))
    assert cos > 0.999
    # conv1's padded columns get no gradient
    w, rows, cols, _ = lay[0]
    assert not g[w:w + rows * cols].reshape(rows, cols)[:, 18:].any()


def test_training_fits_a_fixed_batch():
    import torch
    net = learned.Learner(64, seed=3)
    x, _ = _inputs(64, 11)
    t = torch.from_numpy(np.random.default_rng(12).normal(size=(64, 6)).astype(np.float32) * 0.5).cuda()
    loss = torch.zeros(400, device="cuda")
    for s in range(400):
        net.train_step(x, t, 1e-3, loss[s])
    torch.cuda.synchronize()
    assert not net.timed_out()
    curve = loss.cpu().numpy()
    assert curve[-10:].mean() < 0.1 * curve[:10].mean()
    p = net.params()
    lay, _ = lo.layout()
    w, rows, cols, _ = lay[0]
    assert not p[w:w + rows * cols].reshape(rows, cols)[:, 18:].any()


def test_rejects_bad_batches():
    net = learned.Learner(16, seed=0)
    x, _ = _inputs(24, 0)
    with pytest.raises(ValueError):
        net.forward(x[:12])
    with pytest.raises(ValueError):
        net.forward(x)  # beyond the capacity
    with pytest.raises(ValueError):
        learned.Learner(12)


def _fused_pipeline(frames=3):
    seq = synthetic.make_sequence(21, frames)
    k = learned.intrinsics640()
    gpu = kf.Pipeline(learned.volume_config(256, 0.02))
    loop = kf.Reconstruction(gpu, k)
    for f in range(frames):
        loop.process(seq.depth[f])
    return seq, gpu, loop, k


def test_net_input_matches_host_arithmetic():
    import torch
    seq, gpu, loop, k = _fused_pipeline()
    pose = np.asarray(loop.trajectory[-1], dtype=np.float64)
    depth = seq.depth[-1]
    out = torch.zeros(9600, dtype=torch.bfloat16, device="cuda")
    learned.WarmStart().input(gpu, depth, k, pose, out)
    torch.cuda.synchronize()
    got = out.float().cpu().numpy().reshape(60, 80, 2)
    # current depth: 8x8 block means of the valid depths
    d = depth.astype(np.float32).reshape(60, 8, 80, 8) / np.float32(synthetic.DEPTH_SCALE)
    n = (depth.reshape(60, 8, 80, 8) != 0).sum(axis=(1, 3))
    cur = np.where(n > 0, d.sum(axis=(1, 3)) / np.maximum(n, 1), 0).astype(np.float32)
    # predicted depth: the model rendered at the pose with 1/8 intrinsics
    kn = abi.Intrinsics(k.fx / 8, k.fy / 8, (k.cx + 0.5) / 8 - 0.5, (k.cy + 0.5) / 8 - 0.5)
    maps = gpu.raycast(kn, 80, 60, abi.matrix_from_rigid(abi.rigid_from_matrix(pose)))
    pts = maps.points.reshape(60, 80, 3).astype(np.float64)
    r = abi.matrix_from_rigid(abi.rigid_from_matrix(pose)).astype(np.float64)
    z = ((pts - r[:3, 3]) @ r[:3, :3])[..., 2]
    z = np.where(np.isfinite(z) & (z > 0), z, 0.0)
    mean = z[z > 0].mean()
    c0 = np.where(cur > 0, cur - mean, 0.0)
    c1 = np.where((cur > 0) & (z > 0), np.clip((cur - z) * 10.0, -1, 1), 0.0)
    # one bf16 step of the value's magnitude (and float32 summation order)
    assert np.abs(got[..., 0] - c0).max() <= 2 ** -7 * max(1.0, np.abs(c0).max())
    assert np.abs(got[..., 1] - c1).max() <= 2 ** -7 + 1e-4
    assert (got[..., 0] != 0).sum() > 0.8 * 4800 and (got[..., 1] != 0).sum() > 0.5 * 4800


def test_proposal_fallback_rule():
    seq, gpu, loop, k = _fused_pipeline()
    net = learned.Learner(8, seed=5)
    warm = learned.WarmStart()
    pred = learned.constant_velocity(loop.trajectory)
    res = warm.propose(net, gpu, seq.depth[-1], k, pred)
    assert res.matches_predicted > 1000
    chosen = abi.matrix_from_rigid(res.start)
    if res.used_proposal:
        assert res.cost_proposal <= res.cost_predicted
        assert np.array_equal(chosen, abi.matrix_from_rigid(res.proposal))
    else:
        assert res.cost_proposal > res.cost_predicted
        assert np.array_equal(chosen, abi.matrix_from_rigid(abi.rigid_from_matrix(pred)))
    # the proposal is pred * exp(twist)
    want = learned.apply_twist(pred, np.array(res.twist, dtype=np.float64))
    np.testing.assert_allclose(abi.matrix_from_rigid(res.proposal), want, atol=1e-5)
    # a far-off net output loses to the constant-velocity start
    p = net.params()
    lay, _ = lo.layout()
    _, _, _, b = lay[5]
    p[b:b + 3] = 0.2 * abi.WARM_START_TWIST_SCALE  # +20 cm on every axis
    net.set_params(p)
    res = warm.propose(net, gpu, seq.depth[-1], k, pred)
    assert res.used_proposal == 0 and res.cost_proposal > res.cost_predicted


def test_trained_net_gains_over_constant_velocity():
    """The shipped network (trained on seeds 0-399 by `python -m
    kinectfusion_b200.learned train`) on held-out seeds at 512^3: from the
    plain loop's own state, its starts (proposal or fallback) lie closer to
    the pose plain ICP reaches than the constant-velocity prediction, and a
    short learned loop tracks like the plain loop (within 1 mm RMS)."""
    net = learned.Learner(8)
    net.load(learned.PARAMS)
    one = learned.one_step_errors(net, [5000, 5002], 20)
    assert one["frames"] >= 30
    assert one["median_start_error_learned_m"] < 0.8 * one["median_start_error_velocity_m"]
    assert one["start_error_learned_m"] < one["start_error_velocity_m"]
    assert one["proposal_used"] > 0.5
    report = learned.evaluate(net, [5002], 12)
    m = report["mean"]
    assert m["learned_vs_plain_rms_m"] < 1e-3
    assert abs(m["ate_learned_m"] - m["ate_velocity_m"]) < 1e-3


def test_asynchronous_learned_loop_matches_the_synchronous_one():
    """kf_warm_start_enqueue keeps the prediction, the net and the fallback
    test on the device; the loop it drives tracks like the host-driven
    loop (WarmStartedReconstruction) and makes the same choices."""
    net = learned.Learner(8)
    net.load(learned.PARAMS)
    frames = 12
    seq = synthetic.make_sequence_device(5002, frames, 0.05, 3.0)
    k = learned.intrinsics640()
    gpu = kf.Pipeline(learned.volume_config(512, 0.01))
    sync = learned.WarmStartedReconstruction(gpu, k, start="learned", learner=net)
    for f in range(frames):
        sync.process(seq.depth[f])
    sync_traj = np.array(sync.trajectory, dtype=np.float64)
    sync_used = [p.used_proposal for p in sync.proposals[2:]]
    gpu.reset()
    loop = learned.AsyncLearnedLoop(gpu, k, net)
    traj, used = [], []
    for f in range(frames):
        loop.enqueue(seq.depth[f])
        r = loop.result()
        traj.append(abi.matrix_from_rigid(r.camera_to_world))
        if f >= 2:
            used.append(loop.proposal().used_proposal)
    traj = np.array(traj, dtype=np.float64)
    assert np.abs(traj[:, :3, 3] - sync_traj[:, :3, 3]).max() < 1e-3
    assert sum(a == b for a, b in zip(used, sync_used)) >= 0.8 * len(used)
    assert sum(used) > 0
