"""CPU (numpy, FP64) restatement of the learned RFI flagger: feature
extraction, label construction from the plain flagger's masks, the 4-layer
3x3 conv net forward/backward, BCE-with-logits and Adam.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA training and inference
kernels (gradient checks, feature/label parity).  It has no counterpart in
the reference, which flags only with the statistics of src/gpu_flagger.cu;
the label rule below restates how that flagger's masks are applied
(flag :459-474 replaces whole (beam, channel) columns, flagts :479-494
replaces (beam, time) rows inside the guard band).

Layouts (NHWC): features [B][H=T/tds][W=C][8]; weights [Cout][3][3][Cin].
"""
from __future__ import annotations

import numpy as np

LAYERS = [(8, 32), (32, 64), (64, 64), (64, 1)]
TBIN = 128


def n_params() -> int:
    return sum(co * 9 * ci + co for ci, co in LAYERS)


def init_params(seed: int):
    """He-normal weights, zero biases from numpy's generator (tests copy
    these into the library with dsax_lf_set_params)."""
    rng = np.random.default_rng(seed)
    ps = []
    for ci, co in LAYERS:
        w = rng.standard_normal((co, 3, 3, ci)) * np.sqrt(2.0 / (9 * ci))
        ps.append((w, np.zeros(co)))
    return ps


def _slog(v):
    return np.sign(v) * np.log1p(np.abs(v))


def features(x: np.ndarray, tds: int = 32) -> np.ndarray:
    """x [B][T][C] -> [B][T/tds][C][8], slog(v) = sign(v) log(1 + |v|) of
    z-scores against the beam mean mu and standard deviation sigma:
    f0 pixel mean (x sqrt(tds)), f1 pixel max, f2 row channel-mean
    (x sqrt(tds C)), f3 column mean (x sqrt(T)), f4 max over the pixel's
    samples of the channel-mean series (x sqrt(C)), f5 column max,
    f6 (column variance / sigma^2 - 1) x sqrt(T/2), f7 column peak-to-peak
    of TBIN-sample means / sigma x sqrt(TBIN)."""
    B, T, C = x.shape
    H = T // tds
    xd = x[:, :H * tds].astype(np.float64)
    mu = x.reshape(B, -1).astype(np.float64).mean(axis=1)
    sd = x.reshape(B, -1).astype(np.float64).std(axis=1)
    blk = xd.reshape(B, H, tds, C)
    pm = blk.mean(axis=2)
    px = blk.max(axis=2)
    rm = pm.mean(axis=2)                          # [B][H]
    tsmax = blk.mean(axis=3).max(axis=2)          # [B][H]
    cm = x.astype(np.float64).mean(axis=1)        # [B][C]
    cmax = x.max(axis=1).astype(np.float64)
    cvar = x.astype(np.float64).var(axis=1)
    pb = max(TBIN // tds, 1)
    nb = H // pb
    if nb > 0:
        bm = pm[:, :nb * pb].reshape(B, nb, pb, C).mean(axis=2)
        cpp = bm.max(axis=1) - bm.min(axis=1)
    else:
        cpp = np.zeros((B, C))
    m = mu[:, None, None]
    s = sd[:, None, None]
    ones_c = np.ones((1, 1, C))
    ones_h = np.ones((1, H, 1))
    f = np.empty((B, H, C, 8))
    f[..., 0] = _slog((pm - m) / s * np.sqrt(tds))
    f[..., 1] = _slog((px - m) / s)
    f[..., 2] = _slog(((rm - mu[:, None]) / sd[:, None] * np.sqrt(tds * C))[:, :, None] * ones_c)
    f[..., 3] = _slog(((cm - mu[:, None]) / sd[:, None] * np.sqrt(T))[:, None, :] * ones_h)
    f[..., 4] = _slog(((tsmax - mu[:, None]) / sd[:, None] * np.sqrt(C))[:, :, None] * ones_c)
    f[..., 5] = _slog(((cmax - mu[:, None]) / sd[:, None])[:, None, :] * ones_h)
    f[..., 6] = _slog(((cvar / (sd[:, None] ** 2) - 1.0) * np.sqrt(0.5 * T))[:, None, :] * ones_h)
    f[..., 7] = _slog((cpp / sd[:, None] * np.sqrt(max(TBIN, tds)))[:, None, :] * ones_h)
    return f


def labels(chanmask, tsmask, tds: int, guard: int) -> np.ndarray:
    """Pixel mask the plain flagger applies, on the downsampled grid:
    L[b][h][c] = chanmask[b][c] or (any tsmask in the h-th tds samples and
    guard <= c < C - guard)."""
    B, C = chanmask.shape
    T = tsmask.shape[1]
    H = T // tds
    ts = tsmask[:, :H * tds].reshape(B, H, tds).any(axis=2)
    inside = np.zeros(C, bool)
    inside[guard:C - guard] = True
    return (chanmask[:, None, :].astype(bool) | (ts[:, :, None] & inside[None, None, :]))


def conv3x3(x, w, b):
    """x [B][H][W][Ci], w [Co][3][3][Ci] -> [B][H][W][Co] (zero padding)."""
    B, H, W, Ci = x.shape
    xp = np.zeros((B, H + 2, W + 2, Ci))
    xp[:, 1:-1, 1:-1] = x
    out = np.zeros((B, H, W, w.shape[0])) + b
    for ky in range(3):
        for kx in range(3):
            out += np.einsum("bhwc,oc->bhwo", xp[:, ky:ky + H, kx:kx + W], w[:, ky, kx])
    return out


def conv3x3_backward(x, w, dout):
    """Returns (dx, dw, db) of conv3x3."""
    B, H, W, Ci = x.shape
    xp = np.zeros((B, H + 2, W + 2, Ci))
    xp[:, 1:-1, 1:-1] = x
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    for ky in range(3):
        for kx in range(3):
            dw[:, ky, kx] = np.einsum("bhwo,bhwc->oc", dout, xp[:, ky:ky + H, kx:kx + W])
            dxp[:, ky:ky + H, kx:kx + W] += np.einsum("bhwo,oc->bhwc", dout, w[:, ky, kx])
    return dxp[:, 1:-1, 1:-1], dw, dout.sum(axis=(0, 1, 2))


def forward(params, f):
    acts = [f]
    h = f
    for li, (w, b) in enumerate(params):
        z = conv3x3(h, w, b)
        h = np.maximum(z, 0.0) if li < len(params) - 1 else z
        acts.append(h)
    return acts  # acts[-1] = logits [B][H][W][1]


def bce_loss_grad(logits, y, valid, pos_weight: float):
    """Weighted BCE-with-logits over valid pixels (mean), and d/dlogits."""
    z = logits[..., 0]
    yv = y.astype(np.float64)
    wgt = np.where(yv > 0, pos_weight, 1.0) * valid
    n = valid.sum()
    sp = np.maximum(z, 0) + np.log1p(np.exp(-np.abs(z)))   # softplus(z)
    loss = (wgt * (sp - yv * z)).sum() / n
    sig = 1.0 / (1.0 + np.exp(-z))
    g = wgt * (sig - yv) / n
    return loss, g[..., None]


def backward(params, acts, dlogits):
    grads = [None] * len(params)
    d = dlogits
    for li in range(len(params) - 1, -1, -1):
        w, _ = params[li]
        dx, dw, db = conv3x3_backward(acts[li], w, d)
        grads[li] = (dw, db)
        if li > 0:
            d = dx * (acts[li] > 0)
    return grads


def adam_step(p, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v


def prf1(pred, truth):
    pred = pred.astype(bool)
    truth = truth.astype(bool)
    tp = int((pred & truth).sum())
    fp = int((pred & ~truth).sum())
    fn = int((~pred & truth).sum())
    p = tp / (tp + fp) if tp + fp else 1.0
    r = tp / (tp + fn) if tp + fn else 1.0
    f1 = 2 * p * r / (p + r) if p + r else 0.0
    return p, r, f1
