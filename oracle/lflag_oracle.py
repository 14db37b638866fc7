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
The features restate lf_stat_features_kernel: the plain flagger's own test
statistics (scaled so that its rule fires at 1) and the downsampled
spectrogram, from one statistics pass.
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


def _lower_median(v):
    """sorted(v)[(n+1)/2 - 1] (src/gpu_flagger.cu medval :534-560)."""
    s = np.sort(np.asarray(v, np.float32), kind="stable")
    return s[(len(s) + 1) // 2 - 1]


def _ratio(num, den):
    """num / den in float32, +-1e6 (0 for num == 0) where den == 0."""
    num = np.float32(num)
    if den > 0:
        return np.float32(num / np.float32(den))
    return np.float32(1e6) * np.float32(np.sign(num))


def flag_stats(x, tbin):
    """Per-(beam, chan) mean, variance, max and peak-to-peak of tbin-sample
    bin means, and the per-(beam, t) channel mean (src/gpu_flagger.cu
    calc_spectrum :175-223, calc_varspec :229-278, calc_maxspec :283-319,
    calc_ppspec :324-376, make_ts :414-453), accumulated in float64 and
    stored float32."""
    B, T, C = x.shape
    xd = x.astype(np.float64)
    spec = xd.mean(axis=1)
    var = np.maximum((xd * xd).mean(axis=1) - spec * spec, 0.0)
    mx = x.max(axis=1).astype(np.float64)
    nb = T // tbin
    if nb > 0:
        bm = xd[:, :nb * tbin].reshape(B, nb, tbin, C).sum(axis=2) / tbin
        pp = bm.max(axis=1) - bm.min(axis=1)
    else:
        pp = np.zeros((B, C))
    ts = xd.mean(axis=2)
    f = np.float32
    return spec.astype(f), var.astype(f), mx.astype(f), pp.astype(f), ts.astype(f)


def test_statistics(x, p):
    """The plain flagger's test statistics scaled so that its rule fires at
    1 (src/gpu_flagger.cu:1340-1398): z[k][b][c] for channflag on the mean
    (Thr), variance (Thr + 0.5) and max (Thr): corr / (thr * MAD) after the
    forward filt-channel median detrend (:655-720; flag when |z| > 1, 0 in
    the guard band); simple_channflag on pp (:562-610): (mean of the next
    fbin pp values - median) / (Thr / sqrt(fbin) * MAD) (flag when z > 1);
    and simple_tsflag (:612-653): zt[b][t] = (ts - median) / (TsThr * MAD)
    over the first ts_base samples (flag when zt > 1; 0 when tsflag is off)."""
    B, T, C = x.shape
    G, F, FB = p.guard, p.filt, p.fbin
    spec, var, mx, pp, ts = flag_stats(x, p.tbin)
    if p.parity:
        mx = spec
    n = C - 2 * G
    z = np.zeros((4, B, C), np.float32)
    thrs = [p.thresh, p.thresh + p.var_add, p.thresh]
    for k, S in enumerate([spec, var, mx]):
        thr = np.float32(thrs[k])
        for b in range(B):
            sb = S[b]
            corr = np.zeros(n, np.float32)
            for j in range(G, C - G):
                w0 = j if C - G - j >= F else C - G - F
                corr[j - G] = sb[j] - _lower_median(sb[w0:w0 + F])
            med = _lower_median(corr)
            mad = _lower_median(np.abs(corr - med))
            for i in range(n):
                z[k, b, G + i] = _ratio(corr[i], thr * mad)
    mythr = np.float32(p.thresh) / np.sqrt(np.float32(FB))
    for b in range(B):
        sb = pp[b]
        med = _lower_median(sb[G:C - G])
        mad = _lower_median(np.abs(sb[G:C - G] - med))
        for j in range(G, C - G - FB):
            vv = np.float32(0.0)
            for k in range(FB):
                vv = np.float32(vv + (sb[j] if p.parity else sb[j + k]))
            vv = np.float32(vv / np.float32(FB)) - med
            z[3, b, j] = _ratio(vv, mythr * mad)
    zt = np.zeros((B, T), np.float32)
    if p.tsflag:
        for b in range(B):
            med = _lower_median(ts[b, :p.ts_base])
            mad = _lower_median(np.abs(ts[b, :p.ts_base] - med))
            den = np.float32(p.ts_thresh) * mad
            vv = (ts[b] - med).astype(np.float32)
            zt[b] = (vv / den if den > 0 else np.float32(1e6) * np.sign(vv)).astype(np.float32)
    return z, zt, spec, var


MARGIN_SCALE = 10.0


def features(x: np.ndarray, tds: int, p) -> np.ndarray:
    """x [B][T][C] -> [B][H = T/tds][C][8], slog(v) = sign(v) log(1 + |v|):
    f0 (pixel mean - mu) / sigma * sqrt(tds), f1 (pixel max - mu) / sigma,
    f2 = 10 (max over the pixel's samples of zt - 1), f3..f5 = 10 (|z| - 1)
    for the mean, variance and max statistics, f6 = 10 (z_pp - 1), f7 the
    mean over the pixel's samples of zt (z, zt from test_statistics; each
    margin is positive exactly where the plain rule fires); mu and sigma are
    the beam's sample mean and standard deviation, from the per-channel
    mean and variance.  p: the plain flagger's parameters (guard, filt,
    tbin, fbin, ts_base, tsflag, parity, thresh, var_add, ts_thresh)."""
    B, T, C = x.shape
    H = T // tds
    z, zt, spec, var = test_statistics(x, p)
    f = np.empty((B, H, C, 8))
    blk = x[:, :H * tds].reshape(B, H, tds, C)
    pm = blk.astype(np.float64).sum(axis=2) / tds
    px = blk.max(axis=2).astype(np.float64)
    mu = spec.astype(np.float64).mean(axis=1)
    ex2 = (var.astype(np.float64) + spec.astype(np.float64) ** 2).mean(axis=1)
    sd = np.sqrt(np.maximum(ex2 - mu * mu, 1e-30))
    m = mu[:, None, None]
    s = sd[:, None, None]
    ztp = zt[:, :H * tds].reshape(B, H, tds).astype(np.float64)
    ones_c = np.ones((1, 1, C))
    ones_h = np.ones((1, H, 1))
    km = MARGIN_SCALE
    f[..., 0] = _slog((pm - m) / s * np.sqrt(tds))
    f[..., 1] = _slog((px - m) / s)
    f[..., 2] = _slog(km * (ztp.max(axis=2)[:, :, None] * ones_c - 1.0))
    for k in range(3):
        f[..., 3 + k] = _slog(km * (np.abs(z[k].astype(np.float64))[:, None, :] * ones_h - 1.0))
    f[..., 6] = _slog(km * (z[3].astype(np.float64)[:, None, :] * ones_h - 1.0))
    f[..., 7] = _slog(ztp.mean(axis=2)[:, :, None] * ones_c)
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


def to_bf16(v):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    u = np.asarray(v, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward_bf16(params, f):
    """The tensor-core inference path: BF16 features, weights of layers 1-3
    and activations of layers 1-2 (round to nearest even), wide
    accumulation, layer-3 activations and the last layer in FP32.
    Returns logits [B][H][W]."""
    h = to_bf16(f)
    for li in range(3):
        w, b = params[li]
        z = conv3x3(h, to_bf16(w), b)
        h = np.maximum(z, 0.0)
        if li < 2:
            h = to_bf16(h)
    w, b = params[3]
    return conv3x3(h, w, b)[..., 0]


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
