"""Training and evaluation driver of the learned RFI flagger, on top of the
C-ABI (dsax_flag for labels, dsax_lf_train_step, dsax_flag_learned).
Device buffers are torch tensors; all compute runs in libdsax.so."""
from __future__ import annotations

import numpy as np

from . import FlagParams, flag_params


def plain_masks(ctx, x_dev, params: FlagParams):
    """GPU plain flagger on a device filterbank -> (chanmask, tsmask) device."""
    import torch
    B, T, C = params.nbeam, params.ntime, params.nchan
    cm = torch.zeros(B * C, dtype=torch.uint8, device=x_dev.device)
    tm = torch.zeros(B * T, dtype=torch.uint8, device=x_dev.device)
    torch.cuda.synchronize(x_dev.device)   # inputs ready before the library stream reads them
    ctx.flag(params, x_dev, cm, tm)
    ctx.sync()                             # masks complete before torch or the host reads them
    return cm, tm


def pixel_labels(cm, tm, B, T, C, tds, guard):
    """Pixel mask the plain flagger applies, on the downsampled grid (host)."""
    cm = cm.reshape(B, C).astype(bool)
    ts = tm.reshape(B, T)[:, :(T // tds) * tds].reshape(B, T // tds, tds).any(axis=2)
    inside = np.zeros(C, bool)
    inside[guard:C - guard] = True
    return cm[:, None, :] | (ts[:, :, None] & inside[None, None, :])


def train(ctx, blocks, steps: int = 1000, beams_per_step: int = 16, tds: int = 32,
          lr: float = 3e-3, pos_weight: float = 3.0, seed: int = 0, log=None):
    """blocks: list of device filterbanks [B][T][C] (torch float32).  Labels
    come from the GPU plain flagger on each whole block.  Adam with a cosine
    learning-rate decay from lr to lr/20."""
    import torch
    rng = np.random.default_rng(seed)
    B, T, C = blocks[0].shape
    pfull = flag_params(B, T, C)
    labels = [plain_masks(ctx, x, pfull) for x in blocks]
    pb = flag_params(beams_per_step, T, C)
    torch.cuda.synchronize(blocks[0].device)
    losses = []
    for it in range(steps):
        k = int(rng.integers(len(blocks)))
        b0 = int(rng.integers(0, B - beams_per_step + 1))
        x = blocks[k][b0:b0 + beams_per_step]
        cm = labels[k][0].view(B, C)[b0:b0 + beams_per_step]
        tm = labels[k][1].view(B, T)[b0:b0 + beams_per_step]
        lr_t = lr * (0.05 + 0.95 * 0.5 * (1.0 + np.cos(np.pi * it / max(steps - 1, 1))))
        loss = ctx.lf_train_step(pb, x.contiguous(), cm.contiguous(), tm.contiguous(), tds=tds,
                                 lr=lr_t, pos_weight=pos_weight)
        losses.append(loss)
        if log and (it % 50 == 0 or it == steps - 1):
            log(f"step {it} loss {loss:.4f}")
    return losses


def evaluate(ctx, x_dev, tds: int = 32):
    """Returns (learned mask, plain-flagger pixel mask) as host bool arrays."""
    import torch
    B, T, C = x_dev.shape
    p = flag_params(B, T, C)
    cm, tm = plain_masks(ctx, x_dev, p)
    ref = pixel_labels(cm.cpu().numpy(), tm.cpu().numpy(), B, T, C, tds, p.guard)
    mask = torch.zeros(B * (T // tds) * C, dtype=torch.uint8, device=x_dev.device)
    torch.cuda.synchronize(x_dev.device)
    ctx.flag_learned(p, x_dev, mask, tds=tds)
    ctx.sync()
    return mask.cpu().numpy().reshape(B, T // tds, C).astype(bool), ref


def prf1(pred, truth):
    """Precision, recall and F1 of a boolean mask against a reference mask."""
    pred = np.asarray(pred, bool)
    truth = np.asarray(truth, bool)
    tp = int((pred & truth).sum())
    fp = int((pred & ~truth).sum())
    fn = int((~pred & truth).sum())
    p = tp / (tp + fp) if tp + fp else 1.0
    r = tp / (tp + fn) if tp + fn else 1.0
    f1 = 2 * p * r / (p + r) if p + r else 0.0
    return p, r, f1
