"""Multi-GPU plumbing: one process per GPU.  For the correlator, blocks
shard over ranks with no collective on the data path (each rank correlates
its own blocks) and timings reduce as the max over ranks.  The one real
exchange of the pipeline is the beam corner turn (corner_turn_beams): every
rank beamforms its own subband, then an all-to-all gives each rank a group
of beams across all subbands for the search stage.  torch.distributed
carries it (NCCL over NVLink on GPUs, gloo in the CPU tests)."""
from __future__ import annotations

import datetime
import os


def world():
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(n_items: int, rank: int, world_size: int) -> range:
    """Contiguous, balanced share of n_items for `rank`."""
    lo = n_items * rank // world_size
    hi = n_items * (rank + 1) // world_size
    return range(lo, hi)


def init(backend: str, timeout_s: int = 120):
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank timing over all ranks (identity without a group)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def corner_turn_beams(local, group=None):
    """Beam corner turn of the dsaX_dbnic -> dsaX_nicdb stage
    (src/dsaX_dbnic.c:84-152, src/dsaX_nicdb.c:180-196) as one all-to-all.

    local: this rank's beamformer output for its subband, a tensor
    [T][NB][C] (time, beam, channel; uint8 or float) with NB divisible by the
    world size W.  Returns [NB/W][T][W*C]: beams NB/W*r .. NB/W*(r+1)-1 of
    rank r, with the channel axis ordered by source rank (subband), i.e. the
    filterbank the flagger of that beam group reads."""
    import torch
    import torch.distributed as dist
    W = dist.get_world_size(group)
    T, NB, C = local.shape
    if NB % W:
        raise ValueError("beam count must divide by the world size")
    nb = NB // W
    # [W dest][nb][T][C], contiguous per destination
    send = local.reshape(T, W, nb, C).permute(1, 2, 0, 3).contiguous()
    recv = torch.empty_like(send)
    dist.all_to_all_single(recv.view(-1), send.view(-1), group=group)
    # recv[src][nb][T][C] -> [nb][T][src][C] -> [nb][T][W*C]
    return recv.permute(1, 2, 0, 3).reshape(nb, T, W * C)


def beam_corner_turn(ctx, beams, fil, t0: int = 0, ch0: int = 0, group=None):
    """The beam corner turn through the library: this rank's beamformer
    output beams [T][NB][C] (uint8, device) is packed per destination on the
    GPU (dsax_ct_pack), exchanged with one all-to-all (NCCL), and the
    received subbands are placed into this rank's search filterbank
    fil [NB/W][fil_T][fil_C] at sample t0 and channel ch0 + src * C
    (dsax_ct_unpack).  Rank r receives beams NB/W * r .. NB/W * (r + 1) - 1 of
    every rank's subband, ordered by source rank."""
    import torch
    import torch.distributed as dist
    W = dist.get_world_size(group)
    T, NB, C = beams.shape
    nbl = NB // W
    if NB % W:
        raise ValueError("beam count must divide by the world size")
    send = torch.empty(W * nbl * T * C, dtype=torch.uint8, device=beams.device)
    recv = torch.empty_like(send)
    ctx.ct_pack(beams, T, NB, C, W, send)
    # the collective runs on torch's current stream: order it after the pack
    torch.cuda.ExternalStream(ctx.stream).synchronize()
    dist.all_to_all_single(recv, send, group=group)
    torch.cuda.current_stream(beams.device).synchronize()
    ctx.ct_unpack(recv, W, nbl, T, C, fil, fil.shape[1], fil.shape[2], t0, ch0)
    return fil
