"""CPU oracle of the learned ICP warm-start network (test infrastructure).

The network has no counterpart in the reference (it is the one part of the
pipeline the reference lacks), so this file is its specification: a numpy
restatement of the forward and backward passes that libkf_b200.so runs on the
tensor cores (kf_learner_* in include/kf_b200.h).  With `emulate=True` it
rounds where the device rounds to bf16 - inputs, weights, the activations
passed between layers and the gradients fed to the weight and input GEMMs -
and accumulates each product in float64; with `emulate=False` everything is
float64, which the tests compare with torch autograd to pin the layout (NHWC
activations, weights [out][c*9 + ky*3 + kx], conv1 padded to 24 columns,
(y, x, c) flattening before the first dense layer).

Only tests may import this module; the product never does.
"""

from __future__ import annotations

import numpy as np

# (cin, cout, hin, win, hout, wout, k, kpad) of each 3x3 stride-2 pad-1 convolution
CONV = [(2, 32, 60, 80, 30, 40, 18, 24), (32, 32, 30, 40, 15, 20, 288, 288),
        (32, 64, 15, 20, 8, 10, 288, 288), (64, 64, 8, 10, 4, 5, 576, 576)]
FLAT, HIDDEN, OUT = 1280, 256, 6


def layout():
    """[(weight offset, rows, cols, bias offset)] per layer, and the total."""
    out, off = [], 0
    for i in range(6):
        rows = CONV[i][1] if i < 4 else (HIDDEN if i == 4 else OUT)
        cols = CONV[i][7] if i < 4 else (FLAT if i == 4 else HIDDEN)
        w = off
        off += rows * cols
        b = off
        off += (rows + 7) // 8 * 8
        out.append((w, rows, cols, b))
    return out, off


def bf16(x):
    """float32 values rounded to bf16 (nearest, ties to even), kept as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(params):
    lay, _ = layout()
    ws, bs = [], []
    for w, rows, cols, b in lay:
        ws.append(params[w:w + rows * cols].reshape(rows, cols))
        bs.append(params[b:b + rows])
    return ws, bs


def im2col(x, conv):
    """x [B, H, W, C] -> [B*hout*wout, kpad]: column c*9 + ky*3 + kx, zero
    outside the image and past k."""
    cin, cout, hin, win, hout, wout, k, kpad = conv
    bsz = x.shape[0]
    pad = np.zeros((bsz, hin + 2, win + 2, cin), dtype=x.dtype)
    pad[:, 1:-1, 1:-1, :] = x
    col = np.zeros((bsz, hout, wout, kpad), dtype=x.dtype)
    for c in range(cin):
        for ky in range(3):
            for kx in range(3):
                col[..., c * 9 + ky * 3 + kx] = pad[:, ky:ky + 2 * hout:2, kx:kx + 2 * wout:2, c]
    return col.reshape(bsz * hout * wout, kpad)


def col2im(dcol, conv, bsz):
    cin, cout, hin, win, hout, wout, k, kpad = conv
    d = dcol.reshape(bsz, hout, wout, kpad)
    pad = np.zeros((bsz, hin + 2, win + 2, cin), dtype=dcol.dtype)
    for c in range(cin):
        for ky in range(3):
            for kx in range(3):
                pad[:, ky:ky + 2 * hout:2, kx:kx + 2 * wout:2, c] += d[..., c * 9 + ky * 3 + kx]
    return pad[:, 1:-1, 1:-1, :]


def _ops(emulate):
    if emulate:
        return bf16, np.float32
    return (lambda a: a), np.float64


def forward(params, x, emulate=True):
    """x [B, 60, 80, 2] -> (out [B, 6], cache)."""
    r, dt = _ops(emulate)
    ws, bs = unpack(np.asarray(params, dtype=dt))
    bsz = x.shape[0]
    h = r(np.asarray(x, dtype=dt))
    cache = {"cols": [], "acts": []}
    for i, conv in enumerate(CONV):
        col = im2col(h, conv)
        z = (col.astype(np.float64) @ r(ws[i]).astype(np.float64).T + bs[i]).astype(dt)
        a = np.maximum(z, 0)
        cache["cols"].append(col)
        cache["acts"].append(a)
        h = r(a).reshape(bsz, conv[4], conv[5], conv[1])
    x4 = h.reshape(bsz, FLAT)
    z4 = (x4.astype(np.float64) @ r(ws[4]).astype(np.float64).T + bs[4]).astype(dt)
    a4 = np.maximum(z4, 0)
    x5 = r(a4)
    out = (x5.astype(np.float64) @ r(ws[5]).astype(np.float64).T + bs[5]).astype(dt)
    cache.update(x4=x4, a4=a4, x5=x5, out=out)
    return out, cache


def loss_and_gradients(params, x, target, emulate=True):
    """The batch mean of the squared twist error and its gradient (flat, in
    the parameter layout)."""
    r, dt = _ops(emulate)
    params = np.asarray(params, dtype=dt)
    ws, _ = unpack(params)
    out, c = forward(params, x, emulate)
    bsz = x.shape[0]
    e = out - np.asarray(target, dtype=dt)
    loss = float((e.astype(np.float64) ** 2).sum() / bsz)
    lay, total = layout()
    g = np.zeros(total, dtype=np.float64)

    def put(i, dw, db):
        w, rows, cols, b = lay[i]
        g[w:w + rows * cols] = dw.reshape(-1)
        g[b:b + rows] = db

    def f64(a):
        return a.astype(np.float64)

    dout = (2.0 * e / bsz).astype(dt)
    put(5, f64(r(dout)).T @ f64(c["x5"]), f64(dout).sum(0))
    dx5 = (f64(r(dout)) @ f64(r(ws[5]))).astype(dt)
    dz4 = np.where(c["a4"] > 0, dx5, 0).astype(dt)
    put(4, f64(r(dz4)).T @ f64(c["x4"]), f64(dz4).sum(0))
    d = (f64(r(dz4)) @ f64(r(ws[4]))).astype(dt).reshape(-1, CONV[3][1])
    for i in range(3, -1, -1):
        dz = np.where(c["acts"][i] > 0, d, 0).astype(dt)
        put(i, f64(r(dz)).T @ f64(c["cols"][i]), f64(dz).sum(0))
        if i == 0:
            break
        dcol = (f64(r(dz)) @ f64(r(ws[i]))).astype(dt)
        d = col2im(dcol, CONV[i], bsz).astype(dt).reshape(-1, CONV[i][0])
    return loss, g


def init_params(seed=0):
    """A random parameter vector in the device layout (zero padded columns)."""
    rng = np.random.default_rng(seed)
    lay, total = layout()
    p = np.zeros(total, dtype=np.float32)
    for i, (w, rows, cols, b) in enumerate(lay):
        fan = CONV[i][6] if i < 4 else cols
        m = rng.uniform(-1, 1, size=(rows, cols)) * np.sqrt(6.0 / fan)
        if i < 4:
            m[:, CONV[i][6]:] = 0
        p[w:w + rows * cols] = m.reshape(-1)
        p[b:b + rows] = rng.uniform(-0.1, 0.1, size=rows)
    return p
