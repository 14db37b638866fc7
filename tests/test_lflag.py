"""Learned RFI flagger: the numpy oracle's gradients (CPU), the CUDA
features and gradients against the oracle (GPU), and training on the plain
flagger's masks (GPU) with the F1 it reaches and what it gains over the
method without training."""
import numpy as np
import pytest

import lflag_oracle as LO


def test_oracle_gradients_finite_difference():
    rng = np.random.default_rng(0)
    params = LO.init_params(1)
    f = rng.standard_normal((1, 5, 8, 8))
    y = rng.random((1, 5, 8)) < 0.3
    valid = np.ones((1, 5, 8))
    valid[..., :1] = 0
    acts = LO.forward(params, f)
    loss, dl = LO.bce_loss_grad(acts[-1], y, valid, 2.0)
    grads = LO.backward(params, acts, dl)
    eps = 1e-6
    for li, (gw, gb) in enumerate(grads):
        w, b = params[li]
        for idx in [(0, 1, 2, 0), (w.shape[0] - 1, 0, 0, w.shape[3] - 1)]:
            old = w[idx]
            w[idx] = old + eps
            lp = LO.bce_loss_grad(LO.forward(params, f)[-1], y, valid, 2.0)[0]
            w[idx] = old - eps
            lm = LO.bce_loss_grad(LO.forward(params, f)[-1], y, valid, 2.0)[0]
            w[idx] = old
            assert abs((lp - lm) / (2 * eps) - gw[idx]) < 1e-5 * max(1.0, abs(gw[idx]))
        old = b[0]
        b[0] = old + eps
        lp = LO.bce_loss_grad(LO.forward(params, f)[-1], y, valid, 2.0)[0]
        b[0] = old - eps
        lm = LO.bce_loss_grad(LO.forward(params, f)[-1], y, valid, 2.0)[0]
        b[0] = old
        assert abs((lp - lm) / (2 * eps) - gb[0]) < 1e-5 * max(1.0, abs(gb[0]))


def test_oracle_features_encode_plain_rule(oracle):
    """The channel and time features are margins of the plain flagger's own
    test statistics: "any margin > 0" reproduces the C oracle's masks
    exactly, so a net can reach F1 = 1 from them."""
    from types import SimpleNamespace
    B, T, C, tds = 12, 4096, 48, 32
    x, _ = oracle.gen_filterbank(1000, nbeam=B)
    po = oracle.flag_params(B, T, C, guard=6, filt=21, tbin=128, fbin=8, ts_base=T // 16,
                            tsflag=1, parity=0, thresh=5.0, var_add=0.5, ts_thresh=10.0, perm=[])
    p = SimpleNamespace(guard=6, filt=21, tbin=128, fbin=8, ts_base=T // 16, tsflag=1, parity=0,
                        thresh=5.0, var_add=0.5, ts_thresh=10.0)
    cm, tm, _, _, _ = oracle.plain_flag(x, po, None)
    f = LO.features(x, tds, p)
    y = LO.labels(cm, tm, tds, 6)
    pred = (f[..., 2] > 0) | (f[..., 3] > 0) | (f[..., 4] > 0) | (f[..., 5] > 0) | (f[..., 6] > 0)
    pred[..., :6] = False
    pred[..., C - 6:] = False
    assert y.sum() > 0
    assert np.array_equal(pred, y)


def test_param_count():
    assert LO.n_params() == 58337


def _flat(params):
    return np.concatenate([np.concatenate([w.reshape(-1), b]) for w, b in params]).astype(np.float32)


def _unflat(v):
    out, o = [], 0
    for ci, co in LO.LAYERS:
        w = v[o:o + co * 9 * ci].reshape(co, 3, 3, ci).astype(np.float64)
        o += co * 9 * ci
        b = v[o:o + co].astype(np.float64)
        o += co
        out.append((w, b))
    return out


@pytest.mark.gpu
def test_features_match_oracle(dsax, oracle):
    import torch
    x, _ = oracle.gen_filterbank(11, nbeam=4, ntime=1024, nchan=48)
    p = dsax.flag_params(4, 1024, 48)
    with dsax.Context(dsax.default_config(npkt=16, nchan=8)) as ctx:
        F = torch.zeros(4 * 32 * 48 * 8, dtype=torch.float32, device="cuda")
        xd = torch.from_numpy(x).cuda()
        torch.cuda.synchronize()
        ctx.lf_features(p, xd, F, tds=32)
        ctx.sync()
        got = F.cpu().numpy().reshape(4, 32, 48, 8)
    want = LO.features(x, 32, p)
    np.testing.assert_allclose(got, want, rtol=2e-4, atol=2e-4)


@pytest.mark.gpu
@pytest.mark.parametrize("B", [6, 40])
def test_tensor_core_inference_matches_oracle(dsax, oracle, B):
    """dsax_flag_learned (tcgen05 BF16 implicit-GEMM convolutions, the
    64-channel layers TMA-fed from zero-bordered grids) against the oracle's
    restatement of the same arithmetic (BF16 operands, wide accumulation):
    logits within 5e-3 of their scale, the mask identical away from the
    decision boundary.  40 beams: several 128-pixel tiles per CTA."""
    import torch
    T, C, tds = 1024, 48, 32
    x, _ = oracle.gen_filterbank(21, nbeam=B, ntime=T, nchan=C)
    p = dsax.flag_params(B, T, C)
    rng = np.random.default_rng(9)
    params = LO.init_params(4)
    for i, (w, b) in enumerate(params):
        params[i] = (w, rng.normal(scale=0.1, size=b.shape))
    H = T // tds
    with dsax.Context(dsax.default_config(npkt=16, nchan=8)) as ctx:
        ctx.lf_set_params(_flat(params))
        xd = torch.from_numpy(x).cuda()
        mask = torch.zeros(B * H * C, dtype=torch.uint8, device="cuda")
        logit = torch.zeros(B * H * C, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        ctx.flag_learned(p, xd, mask, logits=logit, tds=tds)
        ctx.sync()
        got = logit.cpu().numpy().reshape(B, H, C)
        gmask = mask.cpu().numpy().reshape(B, H, C).astype(bool)
    pw = _unflat(_flat(params))
    want = LO.forward_bf16(pw, LO.features(x, tds, p))
    scale = np.abs(want).max()
    err = np.abs(got - want)
    assert err.max() < 5e-3 * scale, (err.max(), scale)
    assert err.mean() < 5e-4 * scale
    inside = np.zeros(C, bool)
    inside[p.guard:C - p.guard] = True
    wmask = (want > 0) & inside
    sure = np.abs(want) > 1e-2 * scale
    assert np.array_equal(gmask[sure], wmask[sure])


@pytest.mark.gpu
def test_gradients_match_oracle(dsax, oracle):
    """Loss and every parameter gradient of one step against the FP64
    oracle (FP32 kernels: relative 2e-3 of each layer's gradient scale)."""
    import torch
    B, T, C, tds = 2, 256, 16, 32
    x, _ = oracle.gen_filterbank(12, nbeam=B, ntime=T, nchan=C, n_tones=2, n_bursts=2, n_drift=1)
    p = dsax.flag_params(B, T, C, guard=2, filt=9)
    rng = np.random.default_rng(5)
    cm = (rng.random((B, C)) < 0.2).astype(np.uint8)
    tm = (rng.random((B, T)) < 0.02).astype(np.uint8)
    params = LO.init_params(3)
    for i, (w, b) in enumerate(params):
        params[i] = (w, rng.normal(scale=0.1, size=b.shape))
    with dsax.Context(dsax.default_config(npkt=16, nchan=8)) as ctx:
        ctx.lf_set_params(_flat(params))
        loss, g = ctx.lf_train_step(p, torch.from_numpy(x).cuda(), torch.from_numpy(cm).cuda(),
                                    torch.from_numpy(tm).cuda(), tds=tds, pos_weight=2.0,
                                    update=False, want_grads=True)
    f = LO.features(x, tds, p)
    y = LO.labels(cm, tm, tds, 2)
    valid = np.zeros(y.shape)
    valid[..., 2:C - 2] = 1
    pw = _unflat(_flat(params))                   # the FP32-rounded parameters
    acts = LO.forward(pw, f)
    wloss, dl = LO.bce_loss_grad(acts[-1], y, valid, 2.0)
    wg = LO.backward(pw, acts, dl)
    assert abs(loss - wloss) < 1e-4 * max(1.0, abs(wloss))
    gg = _unflat(g)
    for (gw, gb), (ow, ob) in zip(gg, wg):
        scale = max(np.abs(ow).max(), 1e-12)
        assert np.abs(gw - ow).max() < 2e-3 * scale
        assert np.abs(gb - ob).max() < 2e-3 * max(np.abs(ob).max(), 1e-12)


@pytest.mark.gpu
def test_inference_context_reuse(dsax, oracle):
    """One context, calls with new parameters and changing geometry (40
    beams, then 6, then 40 again inside the same allocation): the cached
    weight images follow the parameters and the zero-bordered grids follow
    the geometry; each call matches the oracle."""
    import torch
    T, C, tds = 1024, 48, 32
    rng = np.random.default_rng(17)
    nets = []
    for k in range(2):
        params = LO.init_params(40 + k)
        nets.append([(w, rng.normal(scale=0.1, size=b.shape)) for w, b in params])
    with dsax.Context(dsax.default_config(npkt=16, nchan=8)) as ctx:
        for B, k in ((40, 0), (6, 1), (40, 1)):
            x, _ = oracle.gen_filterbank(50 + B + k, nbeam=B, ntime=T, nchan=C)
            p = dsax.flag_params(B, T, C)
            ctx.lf_set_params(_flat(nets[k]))
            H = T // tds
            xd = torch.from_numpy(x).cuda()
            mask = torch.zeros(B * H * C, dtype=torch.uint8, device="cuda")
            logit = torch.zeros(B * H * C, dtype=torch.float32, device="cuda")
            torch.cuda.synchronize()
            ctx.flag_learned(p, xd, mask, logits=logit, tds=tds)
            ctx.sync()
            got = logit.cpu().numpy().reshape(B, H, C)
            want = LO.forward_bf16(_unflat(_flat(nets[k])), LO.features(x, tds, p))
            scale = np.abs(want).max()
            assert np.abs(got - want).max() < 5e-3 * scale, (B, k)


@pytest.mark.gpu
def test_training_reaches_plain_flagger_masks(dsax, oracle):
    """Train on 4 synthetic blocks labelled by the GPU plain flagger, test on
    2 held-out blocks: report P/R/F1 per block; the trained net must beat
    the untrained net and the best single-feature threshold rule."""
    import torch
    from dsax import lflag
    B, T, C, tds = 64, 4096, 48, 32
    train_blocks = [torch.from_numpy(oracle.gen_filterbank(1000 + k, nbeam=B)[0]).cuda()
                    for k in range(4)]
    test_blocks = [torch.from_numpy(oracle.gen_filterbank(2000 + k, nbeam=B)[0]).cuda()
                   for k in range(2)]
    with dsax.Context(dsax.default_config(npkt=16, nchan=8)) as ctx:
        ctx.lf_init(7)
        untrained = [LO.prf1(*lflag.evaluate(ctx, xb, tds)) for xb in test_blocks]
        losses = lflag.train(ctx, train_blocks, steps=2000, beams_per_step=16, tds=tds)
        print("loss first/last", losses[0], losses[-1])
        trained = [LO.prf1(*lflag.evaluate(ctx, xb, tds)) for xb in test_blocks]
        # threshold rule on one feature (no learning): best over features and cuts
        p = dsax.flag_params(B, T, C)
        best_rule = 0.0
        for xb in test_blocks:
            F = torch.zeros(B * (T // tds) * C * 8, device="cuda")
            torch.cuda.synchronize()
            ctx.lf_features(p, xb, F, tds=tds)
            ctx.sync()
            F = F.cpu().numpy().reshape(B, T // tds, C, 8)
            _, ref = lflag.evaluate(ctx, xb, tds)
            inside = np.zeros(C, bool)
            inside[p.guard:C - p.guard] = True
            for k in range(8):
                for cut in np.linspace(0.25, 6.0, 24):
                    best_rule = max(best_rule, LO.prf1((F[..., k] > cut) & inside, ref)[2],
                                    LO.prf1((np.abs(F[..., k]) > cut) & inside, ref)[2])
    print("untrained P/R/F1", untrained)
    print("trained   P/R/F1", trained)
    print("best single-feature threshold F1", best_rule)
    f1 = min(t[2] for t in trained)
    assert f1 > max(u[2] for u in untrained) + 0.2
    assert f1 > best_rule
    assert f1 >= 0.98
