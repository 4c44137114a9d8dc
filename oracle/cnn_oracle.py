"""FP64 restatement of the morphology surrogate's forward and backward passes.

TEST INFRASTRUCTURE ONLY: the checker for the BF16 tensor-core kernels of
langmuir_b200/csrc/lgm_cnn.cu.  Only tests/ and bench.py import it.

The network has no counterpart in the reference (its screening step is the
descriptor regression of LangmuirPython/ga2d/ga.py:83-141), so this oracle is
pinned by central finite differences of its own FP64 gradient
(tests/test_surrogate.py) rather than by reference vectors.

Layouts follow include/langmuir_b200_cnn.h: images NHWC, conv weights
[cout][(ky*3 + kx)*cin + c].  ``bf16=True`` rounds to bfloat16 (nearest, ties
to even) exactly where the kernels store BF16 -- weights, activations after
ReLU, pooled maps, the global pool, the hidden layer and every gradient
between layers -- so that the remaining difference is FP32 accumulation
order; ``bf16=False`` is the exact FP64 network on the given weights.
"""
from __future__ import annotations

import numpy as np

CH, HIDDEN, OUTPUTS = 32, 64, 2


def round_bf16(a):
    """Round to bfloat16 (via FP32, nearest-even), returned as float64."""
    f = np.asarray(a, np.float64).astype(np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (u.astype(np.uint32)).view(np.float32).astype(np.float64)


def im2col(x):
    """x [B,H,W,C] -> [B,H,W,9*C] with column (ky*3 + kx)*C + c, zero padding 1."""
    B, H, W, C = x.shape
    xp = np.zeros((B, H + 2, W + 2, C), x.dtype)
    xp[:, 1:-1, 1:-1] = x
    cols = [xp[:, ky:ky + H, kx:kx + W, :] for ky in range(3) for kx in range(3)]
    return np.concatenate(cols, axis=-1)


def conv3x3(x, w, b=None):
    """Pre-activation of a 3x3 'same' convolution, FP64."""
    out = im2col(x) @ np.asarray(w, np.float64).T
    return out if b is None else out + b


def avgpool2(a):
    B, H, W, C = a.shape
    return a.reshape(B, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4))


def upsample2(d):
    return np.repeat(np.repeat(d, 2, axis=1), 2, axis=2)


def conv_wgrad(x, dA):
    """dW[o][k] = sum_p dA[p][o] im2col(x)[p][k], db[o] = sum_p dA[p][o]."""
    cols = im2col(x).reshape(-1, 9 * x.shape[-1])
    d = dA.reshape(-1, dA.shape[-1])
    return d.T @ cols, d.sum(0)


def conv_dgrad(dA, w, cin):
    """Input gradient of conv3x3 (correlation): full transpose conv."""
    B, H, W, _ = dA.shape
    w = np.asarray(w, np.float64).reshape(-1, 3, 3, cin)  # [o][ky][kx][c]
    dxp = np.zeros((B, H + 2, W + 2, cin))
    for ky in range(3):
        for kx in range(3):
            dxp[:, ky:ky + H, kx:kx + W, :] += dA @ w[:, ky, kx, :]
    return dxp[:, 1:-1, 1:-1, :]


def forward(phases, params, bf16=True):
    """phases uint8 [B,H,W]; params FP32/FP64 arrays in the order
    c1w,c1b,c2w,c2b,c3w,c3b,c4w,c4b,f1w,f1b,f2w,f2b.  Returns y [B,2] and the
    cache for ``backward``."""
    r = round_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
    c1w, c1b, c2w, c2b, c3w, c3b, c4w, c4b, f1w, f1b, f2w, f2b = [np.asarray(p, np.float64)
                                                                   for p in params]
    x = (2.0 * np.asarray(phases, np.float64) - 1.0)[..., None]
    ws = [r(c1w), r(c2w), r(c3w), r(c4w)]
    bs = [c1b, c2b, c3b, c4b]
    cache = {"x": x, "ws": ws}
    h = x
    for i in range(3):
        pre = conv3x3(h, ws[i], bs[i])
        relu = np.maximum(pre, 0.0)
        cache[f"a{i + 1}"] = r(relu)
        h = r(avgpool2(relu))
        cache[f"p{i + 1}"] = h
    pre4 = conv3x3(h, ws[3], bs[3])
    a4 = r(np.maximum(pre4, 0.0))
    cache["a4"] = a4
    g = a4.mean(axis=(1, 2))
    g16 = r(g)
    f1w_, f2w_ = r(f1w), r(f2w)
    h32 = np.maximum(g16 @ f1w_.T + f1b, 0.0)
    h16 = r(h32)
    y = h16 @ f2w_.T + f2b
    cache.update(g16=g16, h32=h32, h16=h16, f1w=f1w_, f2w=f2w_)
    return y, cache


def backward(dy, cache, bf16=True):
    """Gradients in parameter order (conv weights [CH, 9*cin])."""
    r = round_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
    dy16 = r(dy)
    h16, h32, g16 = cache["h16"], cache["h32"], cache["g16"]
    df2w = dy16.T @ h16
    df2b = dy16.sum(0)
    dh16 = r((dy16 @ cache["f2w"]) * (h32 > 0))
    df1w = dh16.T @ g16
    df1b = dh16.sum(0)
    dg = dh16 @ cache["f1w"]
    a4 = cache["a4"]
    HW = a4.shape[1] * a4.shape[2]
    dA = r((a4 > 0) * (dg / HW)[:, None, None, :])
    grads = {}
    ins = [cache["x"], cache["p1"], cache["p2"], cache["p3"]]
    for i in (3, 2, 1, 0):
        dw, db = conv_wgrad(ins[i], dA)
        grads[i] = (dw, db)
        if i == 0:
            break
        dp = r(conv_dgrad(dA, cache["ws"][i], CH))
        act = cache[f"a{i}"]
        dA = r((act > 0) * 0.25 * upsample2(dp))
    return (grads[0][0], grads[0][1], grads[1][0], grads[1][1], grads[2][0], grads[2][1],
            grads[3][0], grads[3][1], df1w, df1b, df2w, df2b)


def init_params(seed):
    """He-normal weights, small random biases (FP64), for tests."""
    rng = np.random.default_rng(seed)
    shapes = [(CH, 9), (CH,), (CH, 9 * CH), (CH,), (CH, 9 * CH), (CH,), (CH, 9 * CH), (CH,),
              (HIDDEN, CH), (HIDDEN,), (OUTPUTS, HIDDEN), (OUTPUTS,)]
    out = []
    for s in shapes:
        if len(s) == 1:
            out.append(0.05 * rng.standard_normal(s))
        else:
            out.append(rng.standard_normal(s) * np.sqrt(2.0 / s[1]))
    return out
