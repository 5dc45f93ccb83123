"""The learned warm-start network's CPU oracle against torch autograd (float64).

The network is new (the reference has none), so its oracle is pinned by an
independent implementation: torch's conv2d / linear autograd on the same
parameters, which fixes the layout conventions and the backward pass.
"""

import numpy as np
import pytest
import torch

import kf_learn_oracle as lo


def _torch_loss(params, x, target):
    lay, _ = lo.layout()
    p = torch.tensor(params, dtype=torch.float64, requires_grad=True)
    h = torch.tensor(x, dtype=torch.float64).permute(0, 3, 1, 2)  # NCHW
    for i, conv in enumerate(lo.CONV):
        w, rows, cols, b = lay[i]
        cin, cout, k = conv[0], conv[1], conv[6]
        weight = p[w:w + rows * cols].view(rows, cols)[:, :k].reshape(cout, cin, 3, 3)
        h = torch.relu(torch.nn.functional.conv2d(h, weight, p[b:b + rows], stride=2, padding=1))
    h = h.permute(0, 2, 3, 1).reshape(x.shape[0], -1)  # (y, x, c) flattening
    w, rows, cols, b = lay[4]
    h = torch.relu(h @ p[w:w + rows * cols].view(rows, cols).T + p[b:b + rows])
    w, rows, cols, b = lay[5]
    out = h @ p[w:w + rows * cols].view(rows, cols).T + p[b:b + rows]
    loss = ((out - torch.tensor(target, dtype=torch.float64)) ** 2).sum() / x.shape[0]
    loss.backward()
    return float(loss), p.grad.numpy(), out.detach().numpy()


@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_matches_torch_autograd(seed):
    rng = np.random.default_rng(seed)
    params = lo.init_params(seed).astype(np.float64)
    x = rng.normal(size=(3, 60, 80, 2)) * 0.5
    target = rng.normal(size=(3, 6))
    loss_t, grad_t, out_t = _torch_loss(params, x, target)
    out_o, _ = lo.forward(params, x, emulate=False)
    loss_o, grad_o = lo.loss_and_gradients(params, x, target, emulate=False)
    np.testing.assert_allclose(out_o, out_t, rtol=1e-10, atol=1e-12)
    assert abs(loss_o - loss_t) <= 1e-10 * max(1.0, loss_t)
    np.testing.assert_allclose(grad_o, grad_t, rtol=1e-8, atol=1e-12)
    # conv1's padded columns carry no gradient
    lay, _ = lo.layout()
    w, rows, cols, _ = lay[0]
    assert not grad_o[w:w + rows * cols].reshape(rows, cols)[:, 18:].any()


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-3], dtype=np.float32)
    r = lo.bf16(v)
    # ties to even: 1 + 2^-8 -> 1, 1 + 3 * 2^-8 -> 1 + 2^-6
    np.testing.assert_array_equal(r[:3], np.array([1.0, 1.0, 1.0 + 2 ** -6], dtype=np.float32))
    assert r[3] == -2.5
    assert (r.view(np.uint32) & 0xFFFF == 0).all()
    np.testing.assert_array_equal(lo.bf16(np.array([3.0e-3], np.float32)),
                                  torch.tensor([3.0e-3]).to(torch.bfloat16).float().numpy())


def test_emulated_gradients_close_to_exact():
    """bf16 rounding (plus the ReLU gates it flips) moves the gradient by about
    ten percent in the first layers and keeps its direction."""
    rng = np.random.default_rng(5)
    params = lo.init_params(5)
    x = (rng.normal(size=(8, 60, 80, 2)) * 0.5).astype(np.float32)
    target = rng.normal(size=(8, 6)).astype(np.float32)
    _, g_exact = lo.loss_and_gradients(params.astype(np.float64), x.astype(np.float64), target, emulate=False)
    _, g_emul = lo.loss_and_gradients(params, x, target, emulate=True)
    rel = np.linalg.norm(g_emul - g_exact) / np.linalg.norm(g_exact)
    cos = g_emul @ g_exact / (np.linalg.norm(g_emul) * np.linalg.norm(g_exact))
    assert rel < 0.2 and cos > 0.98
