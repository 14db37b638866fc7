"""Batches of blocks with mixed subband widths (16 blocks of 192 / 384 / 768 channels):
the batch API, with and without graph capture, must reproduce the per-block
entry points exactly, and the beam flags must equal the plain flagger run
on the beamformer's FP32 filterbank."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(dsax, oracle, widths, npkt=256):
    import torch
    cfg = dsax.default_config(npkt=npkt, nant_in=63, nchan=max(widths), bf_scale=1e-4)
    ctx = dsax.Context(cfg)
    wre, wim = oracle.random_phase_weights(5, max(widths) // 8, 256)
    ctx.set_weights(wre, wim)
    blocks, descs = [], []
    for k, w in enumerate(widths):
        blk = oracle.gen_block(900 + k, npkt, 63, w, "gauss")
        d = {"blk": torch.from_numpy(blk.reshape(-1)).cuda(), "nchan": w,
             "vis": torch.zeros(2 * w * 2080 * 8, dtype=torch.float32, device="cuda"),
             "beams": torch.zeros((npkt // 16) * 256 * (w // 8), dtype=torch.uint8, device="cuda"),
             "chanmask": torch.zeros(256 * (w // 8), dtype=torch.uint8, device="cuda"),
             "tsmask": torch.zeros(256 * (npkt // 16), dtype=torch.uint8, device="cuda")}
        blocks.append(blk)
        descs.append(d)
    torch.cuda.synchronize()
    return ctx, blocks, descs, (wre, wim)


def test_batch_matches_per_block_calls(dsax, oracle):
    import torch
    widths = [192, 384, 192, 768]
    ctx, blocks, descs, (wre, wim) = _setup(dsax, oracle, widths)
    try:
        ctx.run_batch(descs, use_graph=False)
        ctx.sync()
        first = [{k: v.clone() for k, v in d.items() if torch.is_tensor(v) and k != "blk"}
                 for d in descs]
        for d in descs:
            for k in ("vis", "beams", "chanmask", "tsmask"):
                d[k].zero_()
        torch.cuda.synchronize()
        ctx.run_batch(descs, use_graph=True)     # capture + launch
        ctx.run_batch(descs, use_graph=True)     # replay
        ctx.sync()
        for d, f in zip(descs, first):
            for k in f:
                assert torch.equal(d[k], f[k]), k
        # each block against the single-block entry points
        for k, (blk, w) in enumerate(zip(blocks, widths)):
            vis = descs[k]["vis"].cpu().numpy().reshape(2 * w, 2080, 4, 2)
            for c in (0, w // 2, w - 1):
                np.testing.assert_array_equal(vis[2 * c:2 * c + 2], oracle.correlate(blk, c, 1))
            cfg = dsax.default_config(npkt=256, nant_in=63, nchan=w, bf_scale=1e-4)
            with dsax.Context(cfg) as c1:
                c1.set_weights(wre[:w // 8], wim[:w // 8])
                u8 = torch.zeros((256 // 16) * 256 * (w // 8), dtype=torch.uint8, device="cuda")
                f32 = torch.zeros(u8.numel(), dtype=torch.float32, device="cuda")
                c1.beamform(descs[k]["blk"], u8, f32)
                c1.sync()
                assert torch.equal(u8, descs[k]["beams"])
                fb = f32.view(256 // 16, 256, w // 8).permute(1, 0, 2).contiguous()
                p = dsax.flag_params(256, 256 // 16, w // 8, tbin=4)
                p.filt = min(p.filt, w // 8 - 2 * p.guard)
                cm = torch.zeros(256 * (w // 8), dtype=torch.uint8, device="cuda")
                tm = torch.zeros(256 * (256 // 16), dtype=torch.uint8, device="cuda")
                c1.flag(p, fb, cm, tm)
                c1.sync()
                assert torch.equal(cm, descs[k]["chanmask"])
                assert torch.equal(tm, descs[k]["tsmask"])
    finally:
        ctx.close()
